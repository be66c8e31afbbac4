// Darcy fluxes, flow-balance error, CFL / Neumann limits, L2 norm, field
// statistics, Peclet diagnostics and the declared linear EOS.
// FP64, reference operation order, compiled with --fmad=false.
#include "tse_common.cuh"

namespace tse {

constexpr int kRedBlocks = 1024;   // fixed partial count: deterministic reductions

__device__ __forceinline__ void decode(long long t, int ny, int nz, int& i, int& j, int& k) {
    long long row;
    grid_coords(t, ny, nz, i, j, k, row);
}

// compute_q (tse.py:744-780); q on the last plane of each axis is not written
__global__ void compute_q_kernel(TseGrid g, const double* P, const double* BP, const double* Kx,
                                 const double* Ky, const double* Kz, double* qx, double* qy,
                                 double* qz, const double* nue, const double* rho) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int nx = g.nx, ny = g.ny, nz = g.nz;
    if (t >= (long long)nx * ny * nz) return;
    int i, j, k;
    decode(t, ny, nz, i, j, k);
    const double *dx = g.dx, *dy = g.dy, *dz = g.dz;
    if (i < nx - 1) {
        const long long o = t + (long long)ny * nz;
        if (!(BP[t] != 0 && BP[o] != 0))
            qx[t] = (-harm2(Kx[o], Kx[t], dx[i + 1], dx[i]) / harm2(nue[o], nue[t], dx[i + 1], dx[i]) *
                     ((P[o] - P[t]) / (0.5 * (dx[i + 1] + dx[i])) +
                      amean2(rho[o], rho[t], dx[i + 1], dx[i]) * g.g * g.sin_beta));
        else
            qx[t] = 0.0;
    }
    if (j < ny - 1) {
        const long long o = t + nz;
        if (!(BP[t] != 0 && BP[o] != 0))
            qy[t] = (-harm2(Ky[o], Ky[t], dy[j + 1], dy[j]) / harm2(nue[o], nue[t], dy[j + 1], dy[j]) *
                     (P[o] - P[t]) / (0.5 * (dy[j + 1] + dy[j])));
        else
            qy[t] = 0.0;
    }
    if (k < nz - 1) {
        const long long o = t + 1;
        if (!(BP[t] != 0 && BP[o] != 0))
            qz[t] = (-harm2(Kz[o], Kz[t], dz[k + 1], dz[k]) / harm2(nue[o], nue[t], dz[k + 1], dz[k]) *
                     ((P[o] - P[t]) / (0.5 * (dz[k + 1] + dz[k])) +
                      amean2(rho[o], rho[t], dz[k + 1], dz[k]) * g.g * g.cos_beta));
        else
            qz[t] = 0.0;
    }
}

// flow_error (tse.py:409-446)
__global__ void flow_error_kernel(TseGrid g, const double* P, const double* Pn, const double* qx,
                                  const double* qy, const double* qz, const double* WP,
                                  const double* phi, const double* c_f, const double* c_r,
                                  const double* rho, double dt_P, double* e) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int nx = g.nx, ny = g.ny, nz = g.nz;
    if (t >= (long long)nx * ny * nz) return;
    int i, j, k;
    decode(t, ny, nz, i, j, k);
    const double *dx = g.dx, *dy = g.dy, *dz = g.dz;
    const long long sx = (long long)ny * nz;
    double v = 0.0;
    if (i != nx - 1) v -= (qx[t] / dx[i] * harm2(rho[t + sx], rho[t], dx[i + 1], dx[i]));
    if (i != 0) v += (qx[t - sx] / dx[i] * harm2(rho[t - sx], rho[t], dx[i - 1], dx[i]));
    if (j != ny - 1) v -= (qy[t] / dy[j] * harm2(rho[t + nz], rho[t], dy[j + 1], dy[j]));
    if (j != 0) v += (qy[t - nz] / dy[j] * harm2(rho[t - nz], rho[t], dy[j - 1], dy[j]));
    if (k != nz - 1) v -= (qz[t] / dz[k] * harm2(rho[t + 1], rho[t], dz[k + 1], dz[k]));
    if (k != 0) v += (qz[t - 1] / dz[k] * harm2(rho[t - 1], rho[t], dz[k - 1], dz[k]));
    const double por = phi[t];
    v += (WP[t] + ((1 - por) * c_r[t] + por * c_f[t]) * (P[t] - Pn[t]) * rho[t] / dt_P);
    e[t] = v;
}

// ---------------------------------------------------------------- reduces
enum RedOp { R_SUM = 0, R_MAX = 1, R_MIN = 2 };

__device__ __forceinline__ double red_init(int op) {
    return op == R_SUM ? 0.0 : (op == R_MAX ? -__longlong_as_double(0x7ff0000000000000LL)
                                            : __longlong_as_double(0x7ff0000000000000LL));
}
__device__ __forceinline__ double red_combine(int op, double a, double b) {
    return op == R_SUM ? a + b : (op == R_MAX ? nmax(a, b) : nmin(a, b));
}

template <int NT>
__device__ __forceinline__ double block_red(int op, double v, double* sh) {
    if (op == R_SUM) return block_sum<NT>(v, sh);
    if (op == R_MAX) return block_nmax<NT>(v, sh);
    return block_nmin<NT>(v, sh);
}

struct Ops {
    int op[4];
};

// Final pass: one block folds `nparts` partials per output (fixed order).
__global__ void finish_kernel(const double* parts, int nparts, int nout, Ops ops, double* out,
                              int post) {
    __shared__ double sh[kBlock / 32];
    for (int q = 0; q < nout; ++q) {
        const int op = ops.op[q];
        double v = red_init(op);
        for (int b = threadIdx.x; b < nparts; b += blockDim.x) v = red_combine(op, v, parts[q * nparts + b]);
        double r = block_red<kBlock>(op, v, sh);
        if (threadIdx.x == 0) out[q] = r;
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        if (post == 1) {          // l2_norm: out = {sum d^2, sum old^2} -> l2
            double l2 = sqrt(out[0]) / sqrt(out[1] + 1e-200);
            out[0] = (l2 != l2) ? 1.0 : l2;
        } else if (post == 2) {   // CFL: out = {max x, max y, max z} -> dt_CFL
            out[0] = 0.9 / (out[0] + out[1] + out[2]);
        }
    }
}

__global__ void l2_partial_kernel(const double* New, const double* Old, long long n, double* parts) {
    __shared__ double sh[kBlock / 32];
    double s1 = 0.0, s2 = 0.0;
    for (long long f = (long long)blockIdx.x * blockDim.x + threadIdx.x; f < n;
         f += (long long)gridDim.x * blockDim.x) {
        const double d = New[f] - Old[f];
        s1 = s1 + d * d;
        s2 = s2 + Old[f] * Old[f];
    }
    double r1 = block_sum<kBlock>(s1, sh);
    double r2 = block_sum<kBlock>(s2, sh);
    if (threadIdx.x == 0) {
        parts[blockIdx.x] = r1;
        parts[gridDim.x + blockIdx.x] = r2;
    }
}

// dt_CFL (tse.py:1241-1246): element f of reshape(|qx|/phi, (ny,nz,nx)) / dx
// is divided by dx[f % nx]; likewise dy[f % ny]; qz uses dz[k].
__global__ void cfl_partial_kernel(TseGrid g, const double* qx, const double* qy, const double* qz,
                                   const double* phi, double* parts) {
    __shared__ double sh[kBlock / 32];
    const long long n = (long long)g.nx * g.ny * g.nz;
    const double ninf = -__longlong_as_double(0x7ff0000000000000LL);
    double a = ninf, b = ninf, c = ninf;
    for (long long f = (long long)blockIdx.x * blockDim.x + threadIdx.x; f < n;
         f += (long long)gridDim.x * blockDim.x) {
        const double p = phi[f];
        a = nmax(a, fabs(qx[f]) / p / g.dx[f % g.nx]);
        b = nmax(b, fabs(qy[f]) / p / g.dy[f % g.ny]);
        c = nmax(c, fabs(qz[f]) / p / g.dz[f % g.nz]);
    }
    double ra = block_nmax<kBlock>(a, sh);
    double rb = block_nmax<kBlock>(b, sh);
    double rc = block_nmax<kBlock>(c, sh);
    if (threadIdx.x == 0) {
        parts[blockIdx.x] = ra;
        parts[gridDim.x + blockIdx.x] = rb;
        parts[2 * gridDim.x + blockIdx.x] = rc;
    }
}

// explicit_C (tse.py:385-396); per-cell max over species, NaN propagating
struct SpeciesPtrs {
    const double* p[8];
};

__global__ void explicit_c_partial_kernel(TseGrid g, SpeciesPtrs D, int ns, const double* phi,
                                          double* parts) {
    __shared__ double sh[kBlock / 32];
    const long long n = (long long)g.nx * g.ny * g.nz;
    double m = 1e100;
    for (long long f = (long long)blockIdx.x * blockDim.x + threadIdx.x; f < n;
         f += (long long)gridDim.x * blockDim.x) {
        int i, j, k;
        decode(f, g.ny, g.nz, i, j, k);
        double dmax = D.p[0][f];
        for (int s = 1; s < ns; ++s) dmax = nmax(dmax, D.p[s][f]);
        const double dxi = g.dx[i], dyj = g.dy[j], dzk = g.dz[k];
        const double v = 0.45 * dmax / phi[f] / (1 / (dxi * dxi) + 1 / (dyj * dyj) + 1 / (dzk * dzk));
        m = pymin(m, v);
    }
    double r = block_nmin<kBlock>(m, sh);
    if (threadIdx.x == 0) parts[blockIdx.x] = r;
}

__global__ void stats_partial_kernel(const double* x, long long n, double* parts) {
    __shared__ double sh[kBlock / 32];
    const double inf = __longlong_as_double(0x7ff0000000000000LL);
    double s = 0.0, mx = -inf, mn = inf;
    for (long long f = (long long)blockIdx.x * blockDim.x + threadIdx.x; f < n;
         f += (long long)gridDim.x * blockDim.x) {
        const double v = x[f];
        s = s + v;
        mx = nmax(mx, v);
        mn = nmin(mn, v);
    }
    double r1 = block_sum<kBlock>(s, sh);
    double r2 = block_nmax<kBlock>(mx, sh);
    double r3 = block_nmin<kBlock>(mn, sh);
    if (threadIdx.x == 0) {
        parts[blockIdx.x] = r1;
        parts[gridDim.x + blockIdx.x] = r2;
        parts[2 * gridDim.x + blockIdx.x] = r3;
    }
}

// peclet_C (tse.py:331-354): non-boundary cells get |q| / max_s D * d (NaN
// when max_s D == 0); boundary cells keep the zero the reference's PeC array
// was initialised with.
__global__ void peclet_c_partial_kernel(TseGrid g, const double* qx, const double* qy,
                                        const double* qz, SpeciesPtrs Dx, SpeciesPtrs Dy,
                                        SpeciesPtrs Dz, int ns, const double* BC, double* parts) {
    __shared__ double sh[kBlock / 32];
    const long long n = (long long)g.nx * g.ny * g.nz;
    double a = 0.0, b = 0.0, c = 0.0;   // max over a zero-initialised array
    const double nan = __longlong_as_double(0x7ff8000000000000LL);
    for (long long f = (long long)blockIdx.x * blockDim.x + threadIdx.x; f < n;
         f += (long long)gridDim.x * blockDim.x) {
        if (BC[f] == 0) {
            int i, j, k;
            decode(f, g.ny, g.nz, i, j, k);
            double mx = Dx.p[0][f], my = Dy.p[0][f], mz = Dz.p[0][f];
            for (int s = 1; s < ns; ++s) {
                mx = nmax(mx, Dx.p[s][f]);
                my = nmax(my, Dy.p[s][f]);
                mz = nmax(mz, Dz.p[s][f]);
            }
            a = nmax(a, mx != 0 ? fabs(qx[f]) / mx * g.dx[i] : nan);
            b = nmax(b, my != 0 ? fabs(qy[f]) / my * g.dy[j] : nan);
            c = nmax(c, mz != 0 ? fabs(qz[f]) / mz * g.dz[k] : nan);
        }
    }
    double ra = block_nmax<kBlock>(a, sh);
    double rb = block_nmax<kBlock>(b, sh);
    double rc = block_nmax<kBlock>(c, sh);
    if (threadIdx.x == 0) {
        parts[blockIdx.x] = ra;
        parts[gridDim.x + blockIdx.x] = rb;
        parts[2 * gridDim.x + blockIdx.x] = rc;
    }
}

// peclet_T (tse.py:357-383)
__global__ void peclet_t_partial_kernel(TseGrid g, const double* qx, const double* qy,
                                        const double* qz, const double* rho, const double* cp,
                                        const double* phi, const double* l_r, const double* l_f,
                                        const double* BT, double* parts) {
    __shared__ double sh[kBlock / 32];
    const long long n = (long long)g.nx * g.ny * g.nz;
    double a = 0.0, b = 0.0, c = 0.0;
    for (long long f = (long long)blockIdx.x * blockDim.x + threadIdx.x; f < n;
         f += (long long)gridDim.x * blockDim.x) {
        if (BT[f] == 0) {
            int i, j, k;
            decode(f, g.ny, g.nz, i, j, k);
            const double den = (1 - phi[f]) * l_r[f] + phi[f] * l_f[f];
            a = nmax(a, fabs(qx[f]) * rho[f] * cp[f] / den * g.dx[i]);
            b = nmax(b, fabs(qy[f]) * rho[f] * cp[f] / den * g.dy[j]);
            c = nmax(c, fabs(qz[f]) * rho[f] * cp[f] / den * g.dz[k]);
        }
    }
    double ra = block_nmax<kBlock>(a, sh);
    double rb = block_nmax<kBlock>(b, sh);
    double rc = block_nmax<kBlock>(c, sh);
    if (threadIdx.x == 0) {
        parts[blockIdx.x] = ra;
        parts[gridDim.x + blockIdx.x] = rb;
        parts[2 * gridDim.x + blockIdx.x] = rc;
    }
}

// Mass-balance totals in FP64 (cell volume V = dx dy dz):
//   water  sum phi rho V             species s  sum RC phi C_s V
//   heat   sum (phi rho cp_f + (1-phi) rho_r cp_r) T V
//   source rates  sum WP V, sum WC_s V, sum WT V
// out (per block partial q): 0 water, 1..ns species, ns+1 heat, ns+2 WP,
// ns+3..2ns+2 WC, 2ns+3 WT
struct MassArgs {
    const double *phi, *rho, *RC, *T, *cp_f, *rho_r, *cp_r, *WP, *WT;
    const double* C[8];
    const double* WC[8];
    int ns;
};

__global__ void mass_partial_kernel(TseGrid g, MassArgs a, double* parts) {
    __shared__ double sh[kBlock / 32];
    const long long n = (long long)g.nx * g.ny * g.nz;
    const int nq = 2 * a.ns + 4;
    double acc[20];
    for (int q = 0; q < 20; ++q) acc[q] = 0.0;
    for (long long f = (long long)blockIdx.x * blockDim.x + threadIdx.x; f < n;
         f += (long long)gridDim.x * blockDim.x) {
        int i, j, k;
        decode(f, g.ny, g.nz, i, j, k);
        const double V = g.dx[i] * g.dy[j] * g.dz[k];
        const double ph = a.phi[f];
        acc[0] += ph * a.rho[f] * V;
        for (int s = 0; s < a.ns; ++s) {
            acc[1 + s] += a.RC[f] * ph * a.C[s][f] * V;
            acc[a.ns + 3 + s] += a.WC[s][f] * V;
        }
        acc[a.ns + 1] += (ph * a.rho[f] * a.cp_f[f] + (1 - ph) * a.rho_r[f] * a.cp_r[f]) * a.T[f] * V;
        acc[a.ns + 2] += a.WP[f] * V;
        acc[2 * a.ns + 3] += a.WT[f] * V;
    }
    for (int q = 0; q < nq; ++q) {
        const double r = block_sum<kBlock>(acc[q], sh);
        if (threadIdx.x == 0) parts[q * gridDim.x + blockIdx.x] = r;
    }
}

__global__ void mass_finish_kernel(const double* parts, int nparts, int nq, double* out) {
    __shared__ double sh[kBlock / 32];
    for (int q = 0; q < nq; ++q) {
        double v = 0.0;
        for (int b = threadIdx.x; b < nparts; b += blockDim.x) v = v + parts[q * nparts + b];
        const double r = block_sum<kBlock>(v, sh);
        if (threadIdx.x == 0) out[q] = r;
        __syncthreads();
    }
}

// Declared linear EOS: rho = rho0 + a0*C[s0] + ... - tcoef*(T - T0)
struct EosLinear {
    const double* C[8];
    double a[8];
    int m;
    double rho0, tcoef, T0;
};

__global__ void eos_linear_kernel(EosLinear E, const double* T, double* rho, long long n) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    double r = E.rho0;
    for (int q = 0; q < E.m; ++q) r = r + E.a[q] * E.C[q][t];
    r = r - E.tcoef * (T[t] - E.T0);
    rho[t] = r;
}

// Declared per-cell property forms (constant, fourth-order polynomial in T),
// optionally guarded: cells whose guard species equals guard_value keep their
// value, as `if C[s] != v:` in a config callback does.
struct EosForm {
    int kind;
    const double* guard;
    double guard_value;
    double c[5];
};

__global__ void eos_form_kernel(EosForm E, const double* T, double* out, long long n) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    if (E.guard && !(E.guard[t] != E.guard_value)) return;
    double r;
    if (E.kind == TSE_EOS_CONSTANT) {
        r = E.c[0];
    } else {
        // c[4] + c[3]*T + c[2]*T**2 + c[1]*T**3 + c[0]*T**4, left to right,
        // powers by repeated squaring: T**3 = T*(T*T), T**4 = (T*T)*(T*T) --
        // the products numba emits for a literal integer exponent
        const double x = T[t];
        const double x2 = x * x;
        const double x3 = x * x2;
        const double x4 = x2 * x2;
        r = E.c[4] + E.c[3] * x;
        r = r + E.c[2] * x2;
        r = r + E.c[1] * x3;
        r = r + E.c[0] * x4;
    }
    out[t] = r;
}

inline unsigned grid_for(long long n) {
    long long b = (n + kBlock - 1) / kBlock;
    return (unsigned)(b < 1 ? 1 : b);
}

inline unsigned red_blocks(long long n) {
    long long b = (n + kBlock - 1) / kBlock;
    if (b > kRedBlocks) b = kRedBlocks;
    return (unsigned)(b < 1 ? 1 : b);
}

// reduce workspace: up to 8 outputs x kRedBlocks partials
size_t reduce_ws_bytes() { return align256(sizeof(double) * 8 * kRedBlocks); }

static int finish(double* parts, unsigned nparts, int nout, const int* h_ops, double* out, int post,
                  void*, cudaStream_t s) {
    Ops ops;
    for (int q = 0; q < 4; ++q) ops.op[q] = q < nout ? h_ops[q] : 0;
    finish_kernel<<<1, kBlock, 0, s>>>(parts, (int)nparts, nout, ops, out, post);
    return cudaGetLastError() == cudaSuccess ? TSE_OK : TSE_ERR_LAUNCH;
}

}  // namespace tse

using namespace tse;

extern "C" int32_t tse_compute_q(const TseGrid* grid, const double* P, const double* BP,
                                 const double* Kx, const double* Ky, const double* Kz, double* qx,
                                 double* qy, double* qz, const double* nue, const double* rho_f,
                                 void* stream) {
    if (!grid || !P || !BP || !Kx || !Ky || !Kz || !qx || !qy || !qz || !nue || !rho_f) return TSE_ERR_ARG;
    const long long n = (long long)grid->nx * grid->ny * grid->nz;
    if (n <= 0) return TSE_ERR_ARG;
    compute_q_kernel<<<grid_for(n), kBlock, 0, (cudaStream_t)stream>>>(*grid, P, BP, Kx, Ky, Kz, qx,
                                                                       qy, qz, nue, rho_f);
    return cudaGetLastError() == cudaSuccess ? TSE_OK : TSE_ERR_LAUNCH;
}

extern "C" int32_t tse_flow_error(const TseGrid* grid, const double* P, const double* Pn,
                                  const double* qx, const double* qy, const double* qz,
                                  const double* WP, const double* phi, const double* c_f,
                                  const double* c_r, const double* rho_f, double dt_P, double* e,
                                  void* stream) {
    if (!grid || !P || !Pn || !qx || !qy || !qz || !WP || !phi || !c_f || !c_r || !rho_f || !e)
        return TSE_ERR_ARG;
    const long long n = (long long)grid->nx * grid->ny * grid->nz;
    if (n <= 0) return TSE_ERR_ARG;
    flow_error_kernel<<<grid_for(n), kBlock, 0, (cudaStream_t)stream>>>(*grid, P, Pn, qx, qy, qz, WP,
                                                                        phi, c_f, c_r, rho_f, dt_P, e);
    return cudaGetLastError() == cudaSuccess ? TSE_OK : TSE_ERR_LAUNCH;
}

extern "C" int32_t tse_l2_norm(const double* New, const double* Old, int64_t n, double* d_out,
                               void* ws, size_t ws_bytes, void* stream) {
    if (!New || !Old || !d_out || !ws || n <= 0) return TSE_ERR_ARG;
    if (ws_bytes < reduce_ws_bytes()) return TSE_ERR_WORKSPACE;
    cudaStream_t s = (cudaStream_t)stream;
    double* parts = (double*)ws;
    const unsigned nb = red_blocks(n);
    l2_partial_kernel<<<nb, kBlock, 0, s>>>(New, Old, n, parts);
    if (cudaGetLastError() != cudaSuccess) return TSE_ERR_LAUNCH;
    static const int ops[2] = {R_SUM, R_SUM};
    return finish(parts, nb, 2, ops, d_out, 1, ws, s);
}

extern "C" int32_t tse_dt_cfl(const TseGrid* grid, const double* qx, const double* qy,
                              const double* qz, const double* phi, double* d_out, void* ws,
                              size_t ws_bytes, void* stream) {
    if (!grid || !qx || !qy || !qz || !phi || !d_out || !ws) return TSE_ERR_ARG;
    if (ws_bytes < reduce_ws_bytes()) return TSE_ERR_WORKSPACE;
    const long long n = (long long)grid->nx * grid->ny * grid->nz;
    if (n <= 0) return TSE_ERR_ARG;
    cudaStream_t s = (cudaStream_t)stream;
    double* parts = (double*)ws;
    const unsigned nb = red_blocks(n);
    cfl_partial_kernel<<<nb, kBlock, 0, s>>>(*grid, qx, qy, qz, phi, parts);
    if (cudaGetLastError() != cudaSuccess) return TSE_ERR_LAUNCH;
    static const int ops[3] = {R_MAX, R_MAX, R_MAX};
    return finish(parts, nb, 3, ops, d_out, 2, ws, s);
}

extern "C" int32_t tse_explicit_C(const TseGrid* grid, const double* const* h_D, int32_t nspec,
                                  const double* phi, double* d_out, void* ws, size_t ws_bytes,
                                  void* stream) {
    if (!grid || !h_D || nspec < 1 || nspec > 8 || !phi || !d_out || !ws) return TSE_ERR_ARG;
    if (ws_bytes < reduce_ws_bytes()) return TSE_ERR_WORKSPACE;
    const long long n = (long long)grid->nx * grid->ny * grid->nz;
    cudaStream_t s = (cudaStream_t)stream;
    SpeciesPtrs D;
    for (int q = 0; q < 8; ++q) D.p[q] = q < nspec ? h_D[q] : nullptr;
    double* parts = (double*)ws;
    const unsigned nb = red_blocks(n);
    explicit_c_partial_kernel<<<nb, kBlock, 0, s>>>(*grid, D, nspec, phi, parts);
    if (cudaGetLastError() != cudaSuccess) return TSE_ERR_LAUNCH;
    static const int ops[1] = {R_MIN};
    return finish(parts, nb, 1, ops, d_out, 0, ws, s);
}

extern "C" int32_t tse_field_stats(const double* x, int64_t n, double* d_out, void* ws,
                                   size_t ws_bytes, void* stream) {
    if (!x || n <= 0 || !d_out || !ws) return TSE_ERR_ARG;
    if (ws_bytes < reduce_ws_bytes()) return TSE_ERR_WORKSPACE;
    cudaStream_t s = (cudaStream_t)stream;
    double* parts = (double*)ws;
    const unsigned nb = red_blocks(n);
    stats_partial_kernel<<<nb, kBlock, 0, s>>>(x, n, parts);
    if (cudaGetLastError() != cudaSuccess) return TSE_ERR_LAUNCH;
    static const int ops[3] = {R_SUM, R_MAX, R_MIN};
    return finish(parts, nb, 3, ops, d_out, 0, ws, s);
}

extern "C" int32_t tse_peclet_C(const TseGrid* grid, const double* qx, const double* qy,
                                const double* qz, const double* const* h_Dx,
                                const double* const* h_Dy, const double* const* h_Dz, int32_t ns,
                                const double* BC, double* d_out, void* ws, size_t ws_bytes,
                                void* stream) {
    if (!grid || !qx || !qy || !qz || !h_Dx || !h_Dy || !h_Dz || ns < 1 || ns > 8 || !BC || !d_out || !ws)
        return TSE_ERR_ARG;
    if (ws_bytes < reduce_ws_bytes()) return TSE_ERR_WORKSPACE;
    const long long n = (long long)grid->nx * grid->ny * grid->nz;
    cudaStream_t s = (cudaStream_t)stream;
    SpeciesPtrs X, Y, Z;
    for (int q = 0; q < 8; ++q) {
        X.p[q] = q < ns ? h_Dx[q] : nullptr;
        Y.p[q] = q < ns ? h_Dy[q] : nullptr;
        Z.p[q] = q < ns ? h_Dz[q] : nullptr;
    }
    double* parts = (double*)ws;
    const unsigned nb = red_blocks(n);
    peclet_c_partial_kernel<<<nb, kBlock, 0, s>>>(*grid, qx, qy, qz, X, Y, Z, ns, BC, parts);
    if (cudaGetLastError() != cudaSuccess) return TSE_ERR_LAUNCH;
    static const int ops[3] = {R_MAX, R_MAX, R_MAX};
    return finish(parts, nb, 3, ops, d_out, 0, ws, s);
}

extern "C" int32_t tse_peclet_T(const TseGrid* grid, const double* qx, const double* qy,
                                const double* qz, const double* rho_f, const double* cp_f,
                                const double* phi, const double* l_r, const double* l_f,
                                const double* BT, double* d_out, void* ws, size_t ws_bytes,
                                void* stream) {
    if (!grid || !qx || !qy || !qz || !rho_f || !cp_f || !phi || !l_r || !l_f || !BT || !d_out || !ws)
        return TSE_ERR_ARG;
    if (ws_bytes < reduce_ws_bytes()) return TSE_ERR_WORKSPACE;
    const long long n = (long long)grid->nx * grid->ny * grid->nz;
    cudaStream_t s = (cudaStream_t)stream;
    double* parts = (double*)ws;
    const unsigned nb = red_blocks(n);
    peclet_t_partial_kernel<<<nb, kBlock, 0, s>>>(*grid, qx, qy, qz, rho_f, cp_f, phi, l_r, l_f, BT,
                                                 parts);
    if (cudaGetLastError() != cudaSuccess) return TSE_ERR_LAUNCH;
    static const int ops[3] = {R_MAX, R_MAX, R_MAX};
    return finish(parts, nb, 3, ops, d_out, 0, ws, s);
}

extern "C" int32_t tse_mass_totals(const TseGrid* grid, const double* phi, const double* rho_f,
                                   const double* RC, const double* const* h_C,
                                   const double* const* h_WC, int32_t nspec, const double* T,
                                   const double* cp_f, const double* rho_r, const double* cp_r,
                                   const double* WP, const double* WT, double* d_out, void* ws,
                                   size_t ws_bytes, void* stream) {
    if (!grid || !phi || !rho_f || !RC || !T || !cp_f || !rho_r || !cp_r || !WP || !WT || !d_out ||
        !ws || nspec < 0 || nspec > 8 || (nspec > 0 && (!h_C || !h_WC)))
        return TSE_ERR_ARG;
    const long long n = (long long)grid->nx * grid->ny * grid->nz;
    const int nq = 2 * nspec + 4;
    const unsigned nb = red_blocks(n) > 256 ? 256 : red_blocks(n);
    if (ws_bytes < reduce_ws_bytes() || (size_t)nq * nb > (size_t)8 * kRedBlocks) return TSE_ERR_WORKSPACE;
    MassArgs a;
    a.phi = phi;
    a.rho = rho_f;
    a.RC = RC;
    a.T = T;
    a.cp_f = cp_f;
    a.rho_r = rho_r;
    a.cp_r = cp_r;
    a.WP = WP;
    a.WT = WT;
    a.ns = nspec;
    for (int s = 0; s < 8; ++s) {
        a.C[s] = s < nspec ? h_C[s] : nullptr;
        a.WC[s] = s < nspec ? h_WC[s] : nullptr;
    }
    cudaStream_t s = (cudaStream_t)stream;
    double* parts = (double*)ws;
    mass_partial_kernel<<<nb, kBlock, 0, s>>>(*grid, a, parts);
    if (cudaGetLastError() != cudaSuccess) return TSE_ERR_LAUNCH;
    mass_finish_kernel<<<1, kBlock, 0, s>>>(parts, (int)nb, nq, d_out);
    return cudaGetLastError() == cudaSuccess ? TSE_OK : TSE_ERR_LAUNCH;
}

extern "C" int32_t tse_eos_linear(const TseGrid* grid, const double* const* h_C,
                                  const int32_t* h_sidx, const double* h_coef, int32_t m,
                                  const double* T, double rho0, double tcoef, double T0,
                                  double* rho_f, void* stream) {
    if (!grid || !T || !rho_f || m < 0 || m > 8 || (m > 0 && (!h_C || !h_sidx || !h_coef)))
        return TSE_ERR_ARG;
    const long long n = (long long)grid->nx * grid->ny * grid->nz;
    EosLinear E;
    for (int q = 0; q < 8; ++q) {
        E.C[q] = q < m ? h_C[h_sidx[q]] : nullptr;
        E.a[q] = q < m ? h_coef[q] : 0.0;
    }
    E.m = m;
    E.rho0 = rho0;
    E.tcoef = tcoef;
    E.T0 = T0;
    eos_linear_kernel<<<grid_for(n), kBlock, 0, (cudaStream_t)stream>>>(E, T, rho_f, n);
    return cudaGetLastError() == cudaSuccess ? TSE_OK : TSE_ERR_LAUNCH;
}

extern "C" int32_t tse_eos_form(const TseGrid* grid, const TseEosForm* form, const double* T,
                                const double* guard, double* out, void* stream) {
    if (!grid || !form || !out) return TSE_ERR_ARG;
    if (form->kind != TSE_EOS_CONSTANT && form->kind != TSE_EOS_POLY4_T) return TSE_ERR_ARG;
    if (form->kind == TSE_EOS_POLY4_T && !T) return TSE_ERR_ARG;
    const long long n = (long long)grid->nx * grid->ny * grid->nz;
    if (n <= 0) return TSE_ERR_ARG;
    EosForm E;
    E.kind = form->kind;
    E.guard = guard;
    E.guard_value = form->guard_value;
    for (int q = 0; q < 5; ++q) E.c[q] = form->coef[q];
    eos_form_kernel<<<grid_for(n), kBlock, 0, (cudaStream_t)stream>>>(E, T, out, n);
    return cudaGetLastError() == cudaSuccess ? TSE_OK : TSE_ERR_LAUNCH;
}
