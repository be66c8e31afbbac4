// FP64 red-black SOR pressure solve, compute_P (tse.py:647-742).
//
// The reference recomputes six transmissibilities (alpha, tse.py:249-260)
// and four buoyancy terms (beta_g, tse.py:263-271) for every cell in every
// sweep.  They do not change during a solve, so one assembly pass computes
// them once, with the reference's operation order, and stores them per
// colour in the compact colour-split layout; the persistent loop then
// streams 11-13 coefficient words per cell-update and evaluates the update
//   P = (1-SOR) P + SOR (Anew + A B + Cnew - C D + Enew + Gnew + Inew + I J
//                        + Knew - K L + R Pn + WP) / (R + M)       (tse.py:691-695)
// term by term in the same order, so each cell-update is bit-identical to the
// reference's.  Compiled with --fmad=false.
#include <atomic>

#include "tse_dc.cuh"
#include "tse_forms.cuh"
#include "tse_rbsolve.cuh"
#include "tse_rbsolve_tma.cuh"

namespace tse {

// alpha (tse.py:249-260) for the face between cells o (first) and c
__device__ __forceinline__ double alpha_(double K1, double K2, double n1, double n2, double r1,
                                         double r2, double d1, double d2, double dden1,
                                         double dden2) {
    return harm2(K1, K2, d1, d2) / harm2(n1, n2, d1, d2) / (dden2 * (dden1 + dden2) * 0.5) *
           harm2(r1, r2, d1, d2);
}

// One cell of the pressure assembly (cell t of the padded natural order);
// with fz, also the mixed-precision form's first cycle (DcFuse): K'_q =
// k_q / Den and r' = (sum(Pn) - Den Pn) / Den with sum() of PressureForm over
// the neighbours' Pn; returns Pn^2 (0 for padding).
template <bool DC>
__device__ __forceinline__ double assemble_p_cell(const TseGrid& g, const TsePressureArgs& a,
                                                  const PressureForm& F, uint8_t* mask0,
                                                  uint8_t* mask1, const Layout& L, long long t,
                                                  const DcFuse& fz) {
    const int nx = L.nx, ny = L.ny, nz = L.nz;
    int i, j, k;
    long long row;
    grid_coords(t, ny, L.nzp, i, j, k, row);
    const long long m = t >> 1;
    const int col = (i + j + k) & 1;
    double* b = F.arr[col];
    const long long N = F.Ncal;
    uint8_t* msk = col ? mask1 : mask0;
    if (k >= nz) {
        for (int q = 0; q < PA_COUNT; ++q) b[q * N + m] = 0.0;
        msk[m] = 0;
        if (DC) {
            float2* rec = reinterpret_cast<float2*>(fz.K[col] + 6 * m);
            for (int q = 0; q < 3; ++q) rec[q] = make_float2(0.0f, 0.0f);
            fz.K[col][6 * fz.Ncal + m] = 0.0f;
        }
        return 0.0;
    }
    const long long c = row * nz + k;
    const long long sx = (long long)ny * nz;
    const double *dx = g.dx, *dy = g.dy, *dz = g.dz;
    const double *Kx = a.Kx, *Ky = a.Ky, *Kz = a.Kz, *nue = a.nue, *rho = a.rho_f;
    double A_ = 0, B_ = 0, C_ = 0, D_ = 0, E_ = 0, G_ = 0, I_ = 0, J_ = 0, K_ = 0, L_ = 0;
    if (i != nx - 1) {
        const long long o = c + sx;
        A_ = alpha_(Kx[o], Kx[c], nue[o], nue[c], rho[o], rho[c], dx[i + 1], dx[i], dx[i + 1], dx[i]);
        B_ = amean2(rho[o], rho[c], dx[i + 1], dx[i]) * g.g * 0.5 * (dx[i + 1] + dx[i]) * g.sin_beta;
    }
    if (i != 0) {
        const long long o = c - sx;
        C_ = alpha_(Kx[c], Kx[o], nue[c], nue[o], rho[c], rho[o], dx[i], dx[i - 1], dx[i - 1], dx[i]);
        D_ = amean2(rho[c], rho[o], dx[i], dx[i - 1]) * g.g * 0.5 * (dx[i] + dx[i - 1]) * g.sin_beta;
    }
    if (j != ny - 1) {
        const long long o = c + nz;
        E_ = alpha_(Ky[o], Ky[c], nue[o], nue[c], rho[o], rho[c], dy[j + 1], dy[j], dy[j + 1], dy[j]);
    }
    if (j != 0) {
        const long long o = c - nz;
        G_ = alpha_(Ky[c], Ky[o], nue[c], nue[o], rho[c], rho[o], dy[j], dy[j - 1], dy[j - 1], dy[j]);
    }
    if (k != nz - 1) {
        const long long o = c + 1;
        I_ = alpha_(Kz[o], Kz[c], nue[o], nue[c], rho[o], rho[c], dz[k + 1], dz[k], dz[k + 1], dz[k]);
        J_ = amean2(rho[o], rho[c], dz[k + 1], dz[k]) * g.g * 0.5 * (dz[k + 1] + dz[k]) * g.cos_beta;
    }
    if (k != 0) {
        const long long o = c - 1;
        K_ = alpha_(Kz[c], Kz[o], nue[c], nue[o], rho[c], rho[o], dz[k], dz[k - 1], dz[k - 1], dz[k]);
        L_ = amean2(rho[c], rho[o], dz[k], dz[k - 1]) * g.g * 0.5 * (dz[k] + dz[k - 1]) * g.cos_beta;
    }
    const double por = a.phi[c];
    const double S = rho[c] * ((1 - por) * a.c_r[c] + por * a.c_f[c]);
    const double R = S / a.dt_P;
    const double M = A_ + C_ + E_ + G_ + I_ + K_;
    const double pn = a.P[c];
    const double AB = A_ * B_, CD = C_ * D_, IJ = I_ * J_, KL = K_ * L_, RPN = R * pn, WP = a.WP[c];
    const double DEN = R + M;
    a.Pn[c] = pn;
    b[PA_A * N + m] = A_;
    b[PA_C * N + m] = C_;
    b[PA_E * N + m] = E_;
    b[PA_G * N + m] = G_;
    b[PA_I * N + m] = I_;
    b[PA_K * N + m] = K_;
    b[PA_AB * N + m] = AB;
    b[PA_CD * N + m] = CD;
    b[PA_IJ * N + m] = IJ;
    b[PA_KL * N + m] = KL;
    b[PA_RPN * N + m] = RPN;
    b[PA_WP * N + m] = WP;
    b[PA_DEN * N + m] = DEN;
    b[PA_S * N + m] = S;
    b[PA_M * N + m] = M;
    b[PA_PN * N + m] = pn;
    b[PA_P * N + m] = pn;
    uint8_t f = neighbour_flags(i, j, k, nx, ny, nz);
    const bool active = !(a.BP[c] != 0.0);
    if (active) f |= F_ACTIVE;
    msk[m] = f;
    if (DC) {
        float2* rec = reinterpret_cast<float2*>(fz.K[col] + 6 * m);
        float rp = 0.0f;
        if (active) {
            const double rden = 1.0 / DEN;
            rec[0] = make_float2((float)(A_ * rden), (float)(C_ * rden));
            rec[1] = make_float2((float)(E_ * rden), (float)(G_ * rden));
            rec[2] = make_float2((float)(I_ * rden), (float)(K_ * rden));
            const double* P = a.P;
            const double s = F.sum_with(
                [&](int q) -> double {
                    switch (q) {
                        case PA_A: return A_;
                        case PA_C: return C_;
                        case PA_E: return E_;
                        case PA_G: return G_;
                        case PA_I: return I_;
                        case PA_K: return K_;
                        case PA_AB: return AB;
                        case PA_CD: return CD;
                        case PA_IJ: return IJ;
                        case PA_KL: return KL;
                        case PA_RPN: return RPN;
                        default: return WP;
                    }
                },
                [&](int q) -> double {
                    return q == 0 ? P[c + sx] : q == 1 ? P[c - sx] : q == 2 ? P[c + nz]
                         : q == 3 ? P[c - nz] : q == 4 ? P[c + 1] : P[c - 1];
                },
                f);
            rp = (float)((s - DEN * pn) * rden);
        } else {
            for (int q = 0; q < 3; ++q) rec[q] = make_float2(0.0f, 0.0f);
        }
        fz.K[col][6 * fz.Ncal + m] = rp;
    }
    return pn * pn;
}

template <bool DC>
__global__ void assemble_p_kernel(TseGrid g, TsePressureArgs a, PressureForm F, uint8_t* mask0,
                                  uint8_t* mask1, Layout L, DcFuse fz) {
    const long long total = (long long)L.nx * L.ny * L.nzp;
    if (!DC) {
        const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
        if (t < total) assemble_p_cell<false>(g, a, F, mask0, mask1, L, t, fz);
        return;
    }
    __shared__ double sh[kBlock / 32];
    double x2 = 0.0;
    for (int s = 0; s < fz.per_thread; ++s) {
        const long long t = ((long long)blockIdx.x * fz.per_thread + s) * kBlock + threadIdx.x;
        if (t >= total) break;
        x2 = x2 + assemble_p_cell<true>(g, a, F, mask0, mask1, L, t, fz);
    }
    const double bs = block_sum<kBlock>(x2, sh);
    if (threadIdx.x == 0) fz.partials[blockIdx.x] = bs;
}

// compact colour arrays -> natural (nx, ny, nz) layout
__global__ void unpack_kernel(double* out, const double* X0, const double* X1, Layout L) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long total = (long long)L.nx * L.ny * L.nz;
    if (t >= total) return;
    int i, j, k;
    long long row;
    grid_coords(t, L.ny, L.nz, i, j, k, row);
    const long long m = (row * L.nzp + k) >> 1;
    out[t] = ((i + j + k) & 1) ? X1[m] : X0[m];
}

size_t pressure_ws_bytes(const Layout& L, long long* Ncal_out) {
    long long Ncal = (L.Nc + 31) & ~31LL;
    if (Ncal_out) *Ncal_out = Ncal;
    size_t b = 0;
    b += align256(sizeof(GridBarrier));
    b += align256((size_t)2 * kMaxBlocks * sizeof(double));
    b += 2 * align256((size_t)Ncal);                               // masks
    b += 2 * (size_t)PA_COUNT * Ncal * sizeof(double);            // arrays
    return b;
}

// Carve the workspace and launch the assembly (shared by the exact and the
// defect-correction pressure solves).  The bytes after the exact form's
// arrays are returned in `tail` for the caller's own use.
static int carve_pressure(const TseGrid* grid, const TsePressureArgs* args, void* d_ws,
                          size_t ws_bytes, cudaStream_t stream, PressureSetup& S) {
    S.L = make_layout(grid->nx, grid->ny, grid->nz);
    const size_t need = pressure_ws_bytes(S.L, &S.Ncal);
    if (need > ws_bytes) return TSE_ERR_WORKSPACE;
    char* p = (char*)d_ws;
    S.bar = (GridBarrier*)p;
    p += align256(sizeof(GridBarrier));
    S.partials = (double*)p;
    p += align256((size_t)2 * kMaxBlocks * sizeof(double));
    S.mask[0] = (uint8_t*)p;
    p += align256((size_t)S.Ncal);
    S.mask[1] = (uint8_t*)p;
    p += align256((size_t)S.Ncal);
    double* arr0 = (double*)p;
    S.F.arr[0] = arr0;
    S.F.arr[1] = arr0 + (size_t)PA_COUNT * S.Ncal;
    S.F.Ncal = S.Ncal;
    S.F.SX = S.L.SX;
    S.F.H = S.L.H;
    S.F.xgrav = grid->sin_beta != 0.0;
    S.F.zgrav = grid->cos_beta != 0.0;
    S.F.SOR = args->SOR;
    S.tail = (char*)d_ws + need;
    S.tail_bytes = ws_bytes - need;
    if (cudaMemsetAsync(S.bar, 0, sizeof(GridBarrier), stream) != cudaSuccess) return TSE_ERR_LAUNCH;
    return TSE_OK;
}

int setup_pressure(const TseGrid* grid, const TsePressureArgs* args, void* d_ws, size_t ws_bytes,
                   cudaStream_t stream, PressureSetup& S) {
    int rc = carve_pressure(grid, args, d_ws, ws_bytes, stream, S);
    if (rc != TSE_OK) return rc;
    const long long total = (long long)S.L.nx * S.L.ny * S.L.nzp;
    assemble_p_kernel<false><<<(unsigned)((total + kBlock - 1) / kBlock), kBlock, 0, stream>>>(
        *grid, *args, S.F, S.mask[0], S.mask[1], S.L, DcFuse{});
    return cudaGetLastError() == cudaSuccess ? TSE_OK : TSE_ERR_LAUNCH;
}

int setup_pressure_dc(const TseGrid* grid, const TsePressureArgs* args, void* d_ws, size_t ws_bytes,
                      cudaStream_t stream, PressureSetup& S, int* nparts) {
    int rc = carve_pressure(grid, args, d_ws, ws_bytes, stream, S);
    if (rc != TSE_OK) return rc;
    if (S.tail_bytes < dc_extra_bytes(S.L)) return TSE_ERR_WORKSPACE;
    DcCtl c;
    dc_carve(S, c, PA_P);
    long long per, nb;
    dc_fuse_grid(S.L, per, nb);
    DcFuse fz;
    fz.K[0] = c.K[0];
    fz.K[1] = c.K[1];
    fz.Ncal = c.Ncal;
    fz.partials = S.partials;
    fz.per_thread = (int)per;
    assemble_p_kernel<true><<<(unsigned)nb, kBlock, 0, stream>>>(*grid, *args, S.F, S.mask[0],
                                                                  S.mask[1], S.L, fz);
    *nparts = (int)nb;
    return cudaGetLastError() == cudaSuccess ? TSE_OK : TSE_ERR_LAUNCH;
}

int launch_unpack(double* out, const double* X0, const double* X1, const Layout& L,
                  cudaStream_t stream) {
    const long long nat = (long long)L.nx * L.ny * L.nz;
    unpack_kernel<<<(unsigned)((nat + kBlock - 1) / kBlock), kBlock, 0, stream>>>(out, X0, X1, L);
    return cudaGetLastError() == cudaSuccess ? TSE_OK : TSE_ERR_LAUNCH;
}

}  // namespace tse

using namespace tse;

extern "C" int32_t tse_compute_P(const TseGrid* grid, const TsePressureArgs* args,
                                 TseSolveStatus* d_status, void* d_ws, size_t ws_bytes,
                                 void* stream_) {
    if (!grid || !args || !d_status || !d_ws) return TSE_ERR_ARG;
    if (grid->nx < 1 || grid->ny < 1 || grid->nz < 1) return TSE_ERR_ARG;
    if (!args->P || !args->Pn || !args->c_f || !args->nue || !args->rho_f || !args->phi ||
        !args->Kx || !args->Ky || !args->Kz || !args->c_r || !args->BP || !args->WP)
        return TSE_ERR_ARG;
    if (args->max_it < 1) return TSE_ERR_ARG;
    cudaStream_t stream = (cudaStream_t)stream_;
    PressureSetup S;
    int rc = setup_pressure(grid, args, d_ws, ws_bytes, stream, S);
    if (rc != TSE_OK) return rc;
    const Layout L = S.L;
    const long long Ncal = S.Ncal;

    SolveCtl ctl;
    ctl.L = L;
    ctl.Ncal = Ncal;
    ctl.plain_sweep = args->sweep == 1;
    ctl.dt = args->dt_P;
    ctl.inc_it = args->inc_it;
    ctl.max_dt = args->max_dt;
    ctl.min_dt = args->min_dt;
    ctl.conv = args->P_conv;
    ctl.max_it = args->max_it;
    ctl.pressure_schedule = 1;
    ctl.stop_on_first = 0;
    ctl.X[0] = S.F.arr[0] + (size_t)PA_P * Ncal;
    ctl.X[1] = S.F.arr[1] + (size_t)PA_P * Ncal;
    ctl.mask[0] = S.mask[0];
    ctl.mask[1] = S.mask[1];
    ctl.partials = S.partials;
    ctl.bar = S.bar;
    ctl.status = d_status;
    rc = launch_rb_solve_tma(S.F, ctl, stream);
    if (rc == 1) rc = launch_rb_solve(S.F, ctl, stream);
    if (rc != TSE_OK) return rc;
    return launch_unpack(args->P, ctl.X[0], ctl.X[1], L, stream);
}

// ----------------------------------------------------------------------------
// Pressure solve without any allocation.
//
// Some host programs cannot hand this library a workspace: their device
// memory belongs to an allocator they do not control (a plugin host that
// passes in only the field buffers, a process held to a fixed memory budget),
// or their time loop must never stall on cudaMalloc, which can synchronise
// the whole device.  tse_compute_P_noalloc serves them: its scratch lives in
// the fixed device array below, which the driver reserves when the library's
// code is loaded on a GPU and keeps until the process exits.  The array is
// shared by every call on that GPU, so calls whose execution overlaps on the
// GPU (different streams, or host threads) corrupt each other; the barrier
// words the solve needs zeroed are cleared by every call, everything else is
// rewritten before it is read.
static __device__ __align__(256) unsigned char g_noalloc_scratch[TSE_NOALLOC_SCRATCH_BYTES];

namespace {
constexpr int kNoallocMaxDevices = 64;
std::atomic<void*> g_noalloc_addr[kNoallocMaxDevices];
}  // namespace

extern "C" int32_t tse_compute_P_noalloc(const TseGrid* grid, const TsePressureArgs* args,
                                         TseSolveStatus* d_status, void* stream) {
    if (!grid || !args || !d_status) return TSE_ERR_ARG;
    if (grid->nx < 1 || grid->ny < 1 || grid->nz < 1) return TSE_ERR_ARG;
    const Layout L = make_layout(grid->nx, grid->ny, grid->nz);
    if (pressure_ws_bytes(L, nullptr) > (size_t)TSE_NOALLOC_SCRATCH_BYTES) return TSE_ERR_WORKSPACE;
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kNoallocMaxDevices)
        return TSE_ERR_DEVICE;
    void* scratch = g_noalloc_addr[dev].load();
    if (!scratch) {
        // first call on this device (the device must be current): host code
        // only knows the array through its device address
        if (cudaGetSymbolAddress(&scratch, g_noalloc_scratch) != cudaSuccess || !scratch)
            return TSE_ERR_DEVICE;
        g_noalloc_addr[dev].store(scratch);
    }
    return tse_compute_P(grid, args, d_status, scratch, (size_t)TSE_NOALLOC_SCRATCH_BYTES, stream);
}
