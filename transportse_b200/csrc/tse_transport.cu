// FP64 species and heat transport solves, compute_C (tse.py:783-916) and
// compute_T (tse.py:919-1081), plus the dispersion coefficients
// (dispersivity, tse.py:460-644).
//
// Within a solve the upwind/diffusive/dispersive neighbour coefficients, the
// explicit (1-omega) part, R*Xn, the source and the IMBLFLO term are fixed,
// so one assembly pass computes them in the reference's operation order and
// the persistent red-black loop evaluates
//   X = (1-SOR) X + SOR (omega (Mnew+Nnew+Onew+Pnew+Qnew+Rnew)
//                        + (1-omega) (...) + R Xn + W - E) / (R - omega M)
// (tse.py:870-875, 1038-1043) term by term.  Compiled with --fmad=false.
#include "tse_forms.cuh"
#include "tse_rbsolve.cuh"
#include "tse_rbsolve_tma.cuh"

namespace tse {

// dispersivity (tse.py:460-644); D = {xl, yl, zl, xr, yr, zr}
__device__ void dispersivity_dev(const double* qx, const double* qy, const double* qz,
                                 const double* l_l, const double* l_t, const double* B, int i,
                                 int j, int k, int nx, int ny, int nz, double* D) {
    const long long sx = (long long)ny * nz, sy = nz;
    const long long c = ((long long)i * ny + j) * nz + k;
#define IX3(ii, jj, kk) (c + (long long)((ii) - i) * sx + (long long)((jj) - j) * sy + ((kk) - k))
    double qxl = 0, qyl = 0, qzl = 0, qxr = 0, qyr = 0, qzr = 0;
    double qxyl = 0, qxzl = 0, qyxl = 0, qyzl = 0, qzxl = 0, qzyl = 0;
    double qxyr = 0, qxzr = 0, qyxr = 0, qyzr = 0, qzxr = 0, qzyr = 0;
    double q1, q2, q3, q4, cnt;
    if (i != 0) {
        qxl = qx[IX3(i - 1, j, k)];
        q1 = qy[IX3(i - 1, j, k)]; q2 = qy[c]; q3 = q4 = 0; cnt = 2;
        if (j != 0) { q3 = qy[IX3(i, j - 1, k)]; q4 = qy[IX3(i - 1, j - 1, k)]; cnt += 2; }
        if (!(B[IX3(i - 1, j, k)] != 0)) qxyl = (q1 + q2 + q3 + q4) / cnt;
        q1 = qz[IX3(i - 1, j, k)]; q2 = qz[c]; q3 = q4 = 0; cnt = 2;
        if (k != 0) { q3 = qz[IX3(i, j, k - 1)]; q4 = qz[IX3(i - 1, j, k - 1)]; cnt += 2; }
        if (!(B[IX3(i - 1, j, k)] != 0)) qxzl = (q1 + q2 + q3 + q4) / cnt;
    }
    if (i != nx - 1) {
        qxr = qx[c];
        q1 = qy[c]; q2 = qy[IX3(i + 1, j, k)]; q3 = q4 = 0; cnt = 2;
        if (j != 0) { q3 = qy[IX3(i + 1, j - 1, k)]; q4 = qy[IX3(i, j - 1, k)]; cnt += 2; }
        if (!(B[IX3(i + 1, j, k)] != 0)) qxyr = (q1 + q2 + q3 + q4) / cnt;
        q1 = qz[c]; q2 = qz[IX3(i + 1, j, k)]; q3 = q4 = 0; cnt = 2;
        if (k != 0) { q3 = qz[IX3(i + 1, j, k - 1)]; q4 = qz[IX3(i, j, k - 1)]; cnt += 2; }
        if (!(B[IX3(i + 1, j, k)] != 0)) qxzr = (q1 + q2 + q3 + q4) / cnt;
    }
    if (j != 0) {
        qyl = qy[IX3(i, j - 1, k)];
        q1 = qx[c]; q2 = qx[IX3(i, j - 1, k)]; q3 = q4 = 0; cnt = 2;
        if (i != 0) { q3 = qx[IX3(i - 1, j - 1, k)]; q4 = qx[IX3(i - 1, j, k)]; cnt += 2; }
        if (!(B[IX3(i, j - 1, k)] != 0)) qyxl = (q1 + q2 + q3 + q4) / cnt;
        q1 = qz[IX3(i, j - 1, k)]; q2 = qz[c]; q3 = q4 = 0; cnt = 2;
        if (k != 0) { q3 = qz[IX3(i, j, k - 1)]; q4 = qz[IX3(i, j - 1, k - 1)]; cnt += 2; }
        if (!(B[IX3(i, j - 1, k)] != 0)) qyzl = (q1 + q2 + q3 + q4) / cnt;
    }
    if (j != ny - 1) {
        qyr = qy[c];
        q1 = qx[IX3(i, j + 1, k)]; q2 = qx[c]; q3 = q4 = 0; cnt = 2;
        if (i != 0) { q3 = qx[IX3(i - 1, j, k)]; q4 = qx[IX3(i - 1, j + 1, k)]; cnt += 2; }
        if (!(B[IX3(i, j + 1, k)] != 0)) qyxr = (q1 + q2 + q3 + q4) / cnt;
        q1 = qz[c]; q2 = qz[IX3(i, j + 1, k)]; q3 = q4 = 0; cnt = 2;
        if (k != 0) { q3 = qz[IX3(i, j + 1, k - 1)]; q4 = qz[IX3(i, j, k - 1)]; cnt += 2; }
        if (!(B[IX3(i, j + 1, k)] != 0)) qyzr = (q1 + q2 + q3 + q4) / cnt;
    }
    if (k != 0) {
        qzl = qz[IX3(i, j, k - 1)];
        q1 = qx[c]; q2 = qx[IX3(i, j, k - 1)]; q3 = q4 = 0; cnt = 2;
        if (i != 0) { q3 = qx[IX3(i - 1, j, k - 1)]; q4 = qx[IX3(i - 1, j, k)]; cnt += 2; }
        if (!(B[IX3(i, j, k - 1)] != 0)) qzxl = (q1 + q2 + q3 + q4) / cnt;
        q1 = qy[c]; q2 = qy[IX3(i, j, k - 1)]; q3 = q4 = 0; cnt = 2;
        if (j != 0) { q3 = qy[IX3(i, j - 1, k - 1)]; q4 = qy[IX3(i, j - 1, k)]; cnt += 2; }
        if (!(B[IX3(i, j, k - 1)] != 0)) qzyl = (q1 + q2 + q3 + q4) / cnt;
    }
    if (k != nz - 1) {
        qzr = qz[c];
        q1 = qx[IX3(i, j, k + 1)]; q2 = qx[c]; q3 = q4 = 0; cnt = 2;
        if (i != 0) { q3 = qx[IX3(i - 1, j, k)]; q4 = qx[IX3(i - 1, j, k + 1)]; cnt += 2; }
        if (!(B[IX3(i, j, k + 1)] != 0)) qzxr = (q1 + q2 + q3 + q4) / cnt;
        q1 = qy[IX3(i, j, k + 1)]; q2 = qy[c]; q3 = q4 = 0; cnt = 2;
        if (j != 0) { q3 = qy[IX3(i, j - 1, k)]; q4 = qy[IX3(i, j - 1, k + 1)]; cnt += 2; }
        if (!(B[IX3(i, j, k + 1)] != 0)) qzyr = (q1 + q2 + q3 + q4) / cnt;
    }
#undef IX3
    const double ll = l_l[c], lt = l_t[c];
    D[0] = ll * fabs(qxl) + lt * (fabs(qxyl) + fabs(qxzl));
    D[1] = ll * fabs(qyl) + lt * (fabs(qyxl) + fabs(qyzl));
    D[2] = ll * fabs(qzl) + lt * (fabs(qzxl) + fabs(qzyl));
    D[3] = ll * fabs(qxr) + lt * (fabs(qxyr) + fabs(qxzr));
    D[4] = ll * fabs(qyr) + lt * (fabs(qyxr) + fabs(qyzr));
    D[5] = ll * fabs(qzr) + lt * (fabs(qzxr) + fabs(qzyr));
}

struct CellIdx {
    int i, j, k, col;
    long long m, c;
    bool pad;
};

__device__ __forceinline__ bool decode_padded(long long t, const Layout& L, CellIdx& x) {
    const long long total = (long long)L.nx * L.ny * L.nzp;
    if (t >= total) return false;
    long long row;
    grid_coords(t, L.ny, L.nzp, x.i, x.j, x.k, row);
    x.m = t >> 1;
    x.col = (x.i + x.j + x.k) & 1;
    x.pad = x.k >= L.nz;
    x.c = row * L.nz + x.k;
    return true;
}

// Shared tail of both assemblies: store the per-cell terms.
__device__ __forceinline__ void store_transport(const TransportForm& F, uint8_t* msk, const CellIdx& x,
                                                const double* co, double Mo, double Xn,
                                                double Rnum, double R, double M, double W,
                                                double EX, double omega, bool active, int nx,
                                                int ny, int nz) {
    double* b = F.arr[x.col];
    const long long N = F.Ncal, m = x.m;
    for (int q = 0; q < 6; ++q) b[q * N + m] = co[q];
    b[TA_Y * N + m] = (1 - omega) * Mo;
    b[TA_RXN * N + m] = R * Xn;
    b[TA_W * N + m] = W;
    b[TA_EX * N + m] = EX;
    b[TA_DEN * N + m] = R - omega * M;
    b[TA_RNUM * N + m] = Rnum;
    b[TA_M * N + m] = M;
    b[TA_XN * N + m] = Xn;
    b[TA_X * N + m] = Xn;
    uint8_t f = neighbour_flags(x.i, x.j, x.k, nx, ny, nz);
    if (active) f |= F_ACTIVE;
    msk[m] = f;
}

__device__ __forceinline__ void store_padding(const TransportForm& F, uint8_t* msk, const CellIdx& x) {
    double* b = F.arr[x.col];
    for (int q = 0; q < TA_COUNT; ++q) b[q * F.Ncal + x.m] = 0.0;
    msk[x.m] = 0;
}

// Both assemblies run one thread per cell and are latency-bound (many FP64
// divisions and neighbour loads per cell).  Three 256-thread blocks per SM
// (80 registers, a few bytes spilled) rather than the two that 96-98
// registers allow: measured on the 256 x 256 x 128 reservoir, species solves
// 13.6 -> 16.2 and heat solves 9.1 -> 11.5 G cell-updates/s.
constexpr int kAssembleMinBlocks = 3;

// coefficient part of compute_C.solve (tse.py:795-868)
__global__ void __launch_bounds__(kBlock, kAssembleMinBlocks) assemble_c_kernel(TseGrid g, TseSpeciesArgs a, TransportForm F, uint8_t* mask0,
                                  uint8_t* mask1, Layout L) {
    CellIdx x;
    if (!decode_padded((long long)blockIdx.x * blockDim.x + threadIdx.x, L, x)) return;
    uint8_t* msk = x.col ? mask1 : mask0;
    if (x.pad) { store_padding(F, msk, x); return; }
    const int nx = L.nx, ny = L.ny, nz = L.nz, i = x.i, j = x.j, k = x.k;
    const long long c = x.c, sx = (long long)ny * nz;
    const double *dx = g.dx, *dy = g.dy, *dz = g.dz, *phi = a.phi, *Cn = a.C;
    double A_ = 0, B_ = 0, C_ = 0, D_ = 0, E_ = 0, F_ = 0, G_ = 0, H_ = 0, I_ = 0, J_ = 0, K_ = 0,
           L_ = 0, M_ = 0, N_ = 0, O_ = 0, P_ = 0, Q_ = 0, R_ = 0, EC = 0;
    double Mold = 0, Nold = 0, Oold = 0, Pold = 0, Qold = 0, Rold = 0;
    double Dd[6] = {0, 0, 0, 0, 0, 0};
    double dd, dd2, ph;
    if (a.l_l[c] != 0 || a.l_t[c] != 0)
        dispersivity_dev(a.qx, a.qy, a.qz, a.l_l, a.l_t, a.BC, i, j, k, nx, ny, nz, Dd);
    double co[6] = {0, 0, 0, 0, 0, 0};
    if (i != nx - 1) {
        const long long o = c + sx;
        dd = dx[i];
        dd2 = (0.5 * (dx[i + 1] + dx[i])) * dd;
        ph = amean2(phi[o], phi[c], dx[i + 1], dx[i]);
        A_ = (harm2(a.D_fx[o], a.D_fx[c], dx[i + 1], dx[i]) * ph + Dd[3]) / dd2;
        N_ = min0(a.qx[c]) / dd;
        H_ = max0(a.qx[c]) / dd;
        co[0] = A_ - N_;
        Mold = co[0] * Cn[o];
    }
    if (i != 0) {
        const long long o = c - sx;
        dd = dx[i];
        dd2 = (0.5 * (dx[i - 1] + dx[i])) * dd;
        ph = amean2(phi[o], phi[c], dx[i - 1], dx[i]);
        B_ = (harm2(a.D_fx[o], a.D_fx[c], dx[i - 1], dx[i]) * ph + Dd[0]) / dd2;
        M_ = max0(a.qx[o]) / dd;
        G_ = min0(a.qx[o]) / dd;
        co[1] = B_ + M_;
        Nold = co[1] * Cn[o];
    }
    if (j != ny - 1) {
        const long long o = c + nz;
        dd = dy[j];
        dd2 = (0.5 * (dy[j + 1] + dy[j])) * dd;
        ph = amean2(phi[o], phi[c], dy[j + 1], dy[j]);
        C_ = (harm2(a.D_fy[o], a.D_fy[c], dy[j + 1], dy[j]) * ph + Dd[4]) / dd2;
        P_ = min0(a.qy[c]) / dd;
        J_ = max0(a.qy[c]) / dd;
        co[2] = C_ - P_;
        Oold = co[2] * Cn[o];
    }
    if (j != 0) {
        const long long o = c - nz;
        dd = dy[j];
        dd2 = (0.5 * (dy[j - 1] + dy[j])) * dd;
        ph = amean2(phi[o], phi[c], dy[j - 1], dy[j]);
        D_ = (harm2(a.D_fy[o], a.D_fy[c], dy[j - 1], dy[j]) * ph + Dd[1]) / dd2;
        O_ = max0(a.qy[o]) / dd;
        I_ = min0(a.qy[o]) / dd;
        co[3] = D_ + O_;
        Pold = co[3] * Cn[o];
    }
    if (k != nz - 1) {
        const long long o = c + 1;
        dd = dz[k];
        dd2 = (0.5 * (dz[k + 1] + dz[k])) * dd;
        ph = amean2(phi[o], phi[c], dz[k + 1], dz[k]);
        E_ = (harm2(a.D_fz[o], a.D_fz[c], dz[k + 1], dz[k]) * ph + Dd[5]) / dd2;
        R_ = min0(a.qz[c]) / dd;
        L_ = max0(a.qz[c]) / dd;
        co[4] = E_ - R_;
        Qold = co[4] * Cn[o];
    }
    if (k != 0) {
        const long long o = c - 1;
        dd = dz[k];
        dd2 = (0.5 * (dz[k - 1] + dz[k])) * dd;
        ph = amean2(phi[o], phi[c], dz[k - 1], dz[k]);
        F_ = (harm2(a.D_fz[o], a.D_fz[c], dz[k - 1], dz[k]) * ph + Dd[2]) / dd2;
        Q_ = max0(a.qz[o]) / dd;
        K_ = min0(a.qz[o]) / dd;
        co[5] = F_ + Q_;
        Rold = co[5] * Cn[o];
    }
    const double Rnum = a.RC[c] * phi[c];
    const double R = Rnum / a.dt;
    const double M = -A_ - B_ - C_ - D_ - E_ - F_ + G_ - H_ + I_ - J_ + K_ - L_;
    if (a.imblflo) EC = Cn[c] / a.rho_f[c] * a.e[c];
    const double Xn = Cn[c];
    const double Mo = Xn * M + Mold + Nold + Oold + Pold + Qold + Rold;
    store_transport(F, msk, x, co, Mo, Xn, Rnum, R, M, a.WC[c], EC, a.omega, !(a.BC[c] != 0.0),
                    nx, ny, nz);
}

// coefficient part of compute_T.solve (tse.py:930-1036)
__global__ void __launch_bounds__(kBlock, kAssembleMinBlocks) assemble_t_kernel(TseGrid g, TseHeatArgs a, TransportForm F, uint8_t* mask0,
                                  uint8_t* mask1, Layout L) {
    CellIdx x;
    if (!decode_padded((long long)blockIdx.x * blockDim.x + threadIdx.x, L, x)) return;
    uint8_t* msk = x.col ? mask1 : mask0;
    if (x.pad) { store_padding(F, msk, x); return; }
    const int nx = L.nx, ny = L.ny, nz = L.nz, i = x.i, j = x.j, k = x.k;
    const long long c = x.c, sx = (long long)ny * nz;
    const double *dx = g.dx, *dy = g.dy, *dz = g.dz, *phi = a.phi, *Tn = a.T;
    double A_ = 0, B_ = 0, C_ = 0, D_ = 0, E_ = 0, F_ = 0, G_ = 0, H_ = 0, I_ = 0, J_ = 0, K_ = 0,
           L_ = 0, S_ = 0, M_ = 0, N_ = 0, O_ = 0, P_ = 0, Q_ = 0, R_ = 0, ET = 0;
    double Mold = 0, Nold = 0, Oold = 0, Pold = 0, Qold = 0, Rold = 0;
    double Dd[6] = {0, 0, 0, 0, 0, 0};
    double dd, dd2, por, lf, lr, cpf, rhocpf;
    if (a.l_l[c] != 0 || a.l_t[c] != 0)
        dispersivity_dev(a.qx, a.qy, a.qz, a.l_l, a.l_t, a.BT, i, j, k, nx, ny, nz, Dd);
    double co[6] = {0, 0, 0, 0, 0, 0};
#define TFACE(o, d1, d2)                                   \
    por = amean2(phi[c], phi[o], d1, d2);                  \
    lf = harm2(a.l_f[c], a.l_f[o], d1, d2);                \
    lr = harm2(a.l_r[c], a.l_r[o], d1, d2);                \
    cpf = harm2(a.cp_f[c], a.cp_f[o], d1, d2);             \
    rhocpf = harm2(a.rho_f[c], a.rho_f[o], d1, d2) * cpf;
    if (i != nx - 1) {
        const long long o = c + sx;
        dd = dx[i];
        dd2 = (0.5 * (dx[i + 1] + dx[i])) * dd;
        TFACE(o, dx[i], dx[i + 1]);
        A_ = ((1 - por) * lr + por * lf + Dd[3] * rhocpf) / dd2;
        S_ = rhocpf / dd;
        N_ = min0(a.qx[c]) * S_;
        H_ = max0(a.qx[c]) * S_;
        co[0] = A_ - N_;
        Mold = co[0] * Tn[o];
    }
    if (i != 0) {
        const long long o = c - sx;
        dd = dx[i];
        dd2 = (0.5 * (dx[i - 1] + dx[i])) * dd;
        TFACE(o, dx[i], dx[i - 1]);
        B_ = ((1 - por) * lr + por * lf + Dd[0] * rhocpf) / dd2;
        S_ = rhocpf / dd;
        M_ = max0(a.qx[o]) * S_;
        G_ = min0(a.qx[o]) * S_;
        co[1] = B_ + M_;
        Nold = co[1] * Tn[o];
    }
    if (j != ny - 1) {
        const long long o = c + nz;
        dd = dy[j];
        dd2 = (0.5 * (dy[j + 1] + dy[j])) * dd;
        TFACE(o, dy[j], dy[j + 1]);
        C_ = ((1 - por) * lr + por * lf + Dd[4] * rhocpf) / dd2;
        S_ = rhocpf / dd;
        P_ = min0(a.qy[c]) * S_;
        J_ = max0(a.qy[c]) * S_;
        co[2] = C_ - P_;
        Oold = co[2] * Tn[o];
    }
    if (j != 0) {
        const long long o = c - nz;
        dd = dy[j];
        dd2 = (0.5 * (dy[j - 1] + dy[j])) * dd;
        TFACE(o, dy[j], dy[j - 1]);
        D_ = ((1 - por) * lr + por * lf + Dd[1] * rhocpf) / dd2;
        S_ = rhocpf / dd;
        O_ = max0(a.qy[o]) * S_;
        I_ = min0(a.qy[o]) * S_;
        co[3] = D_ + O_;
        Pold = co[3] * Tn[o];
    }
    if (k != nz - 1) {
        const long long o = c + 1;
        dd = dz[k];
        dd2 = (0.5 * (dz[k + 1] + dz[k])) * dd;
        TFACE(o, dz[k], dz[k + 1]);
        E_ = ((1 - por) * lr + por * lf + Dd[5] * rhocpf) / dd2;
        S_ = rhocpf / dd;
        R_ = min0(a.qz[c]) * S_;
        L_ = max0(a.qz[c]) * S_;
        co[4] = E_ - R_;
        Qold = co[4] * Tn[o];
    }
    if (k != 0) {
        const long long o = c - 1;
        dd = dz[k];
        dd2 = (0.5 * (dz[k - 1] + dz[k])) * dd;
        TFACE(o, dz[k], dz[k - 1]);
        F_ = ((1 - por) * lr + por * lf + Dd[2] * rhocpf) / dd2;
        S_ = rhocpf / dd;
        Q_ = max0(a.qz[o]) * S_;
        K_ = min0(a.qz[o]) * S_;
        co[5] = F_ + Q_;
        Rold = co[5] * Tn[o];
    }
#undef TFACE
    (void)S_;
    const double por_ = phi[c];
    const double Rnum = por_ * a.rho_f[c] * a.cp_f[c] + (1 - por_) * a.rho_r[c] * a.cp_r[c];
    const double R = Rnum / a.dt;
    const double M = -A_ - B_ - C_ - D_ - E_ - F_ + G_ - H_ + I_ - J_ + K_ - L_;
    if (a.imblflo) ET = a.cp_f[c] * Tn[c] * a.e[c];
    const double Xn = Tn[c];
    const double Mo = Xn * M + Mold + Nold + Oold + Pold + Qold + Rold;
    store_transport(F, msk, x, co, Mo, Xn, Rnum, R, M, a.WT[c], ET, a.omega, !(a.BT[c] != 0.0),
                    nx, ny, nz);
}

__global__ void unpack_t_kernel(double* out, const double* X0, const double* X1, Layout L) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long total = (long long)L.nx * L.ny * L.nz;
    if (t >= total) return;
    int i, j, k;
    long long row;
    grid_coords(t, L.ny, L.nz, i, j, k, row);
    const long long m = (row * L.nzp + k) >> 1;
    out[t] = ((i + j + k) & 1) ? X1[m] : X0[m];
}

size_t transport_ws_bytes(const Layout& L, long long* Ncal_out) {
    long long Ncal = (L.Nc + 31) & ~31LL;
    if (Ncal_out) *Ncal_out = Ncal;
    size_t b = 0;
    b += align256(sizeof(GridBarrier));
    b += align256((size_t)2 * kMaxBlocks * sizeof(double));
    b += 2 * align256((size_t)Ncal);
    b += 2 * (size_t)TA_COUNT * Ncal * sizeof(double);
    return b;
}

// Carve the workspace and launch the assembly (shared by the exact and the
// defect-correction transport solves).
template <class Args, class AssembleK>
static int setup_transport(const TseGrid* grid, const Args* a, void* d_ws, size_t ws_bytes,
                           cudaStream_t stream, AssembleK kernel, int imbl, TransportSetup& S) {
    S.L = make_layout(grid->nx, grid->ny, grid->nz);
    const size_t need = transport_ws_bytes(S.L, &S.Ncal);
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
    S.F.arr[0] = (double*)p;
    S.F.arr[1] = S.F.arr[0] + (size_t)TA_COUNT * S.Ncal;
    S.F.Ncal = S.Ncal;
    S.F.SX = S.L.SX;
    S.F.H = S.L.H;
    S.F.omega = a->omega;
    S.F.SOR = a->SOR;
    S.F.useY = a->omega != 1.0;
    S.F.useEX = imbl != 0;
    S.tail = (char*)d_ws + need;
    S.tail_bytes = ws_bytes - need;
    if (cudaMemsetAsync(S.bar, 0, sizeof(GridBarrier), stream) != cudaSuccess) return TSE_ERR_LAUNCH;
    const long long total = (long long)S.L.nx * S.L.ny * S.L.nzp;
    kernel<<<(unsigned)((total + kBlock - 1) / kBlock), kBlock, 0, stream>>>(*grid, *a, S.F, S.mask[0],
                                                                              S.mask[1], S.L);
    return cudaGetLastError() == cudaSuccess ? TSE_OK : TSE_ERR_LAUNCH;
}

int setup_species(const TseGrid* grid, const TseSpeciesArgs* a, void* d_ws, size_t ws_bytes,
                  cudaStream_t stream, TransportSetup& S) {
    return setup_transport(grid, a, d_ws, ws_bytes, stream, assemble_c_kernel, a->imblflo, S);
}

int setup_heat(const TseGrid* grid, const TseHeatArgs* a, void* d_ws, size_t ws_bytes,
               cudaStream_t stream, TransportSetup& S) {
    return setup_transport(grid, a, d_ws, ws_bytes, stream, assemble_t_kernel, a->imblflo, S);
}

template <class Args, class AssembleK>
static int run_transport(const TseGrid* grid, const Args* a, double* X, TseSolveStatus* d_status,
                         void* d_ws, size_t ws_bytes, void* stream_, AssembleK kernel, int imbl) {
    cudaStream_t stream = (cudaStream_t)stream_;
    TransportSetup S;
    int rc = setup_transport(grid, a, d_ws, ws_bytes, stream, kernel, imbl, S);
    if (rc != TSE_OK) return rc;
    const Layout L = S.L;
    TransportForm F = S.F;
    struct {
        GridBarrier* bar;
        double* partials;
        uint8_t* mask[2];
        double* arr[2];
        long long Ncal;
    } w = {S.bar, S.partials, {S.mask[0], S.mask[1]}, {S.F.arr[0], S.F.arr[1]}, S.Ncal};
    SolveCtl ctl;
    ctl.L = L;
    ctl.Ncal = w.Ncal;
    ctl.plain_sweep = a->sweep == 1;
    ctl.dt = a->dt;
    ctl.inc_it = a->inc_it;
    ctl.max_dt = a->max_dt;
    ctl.min_dt = a->min_dt;
    ctl.conv = a->conv;
    ctl.max_it = a->max_it;
    ctl.pressure_schedule = 0;
    ctl.stop_on_first = a->omega == 0.0;
    ctl.X[0] = w.arr[0] + (size_t)TA_X * w.Ncal;
    ctl.X[1] = w.arr[1] + (size_t)TA_X * w.Ncal;
    ctl.mask[0] = w.mask[0];
    ctl.mask[1] = w.mask[1];
    ctl.partials = w.partials;
    ctl.bar = w.bar;
    ctl.status = d_status;
    rc = launch_rb_solve_tma(F, ctl, stream);
    if (rc == 1) rc = launch_rb_solve(F, ctl, stream);
    if (rc != TSE_OK) return rc;
    const long long nat = (long long)L.nx * L.ny * L.nz;
    unpack_t_kernel<<<(unsigned)((nat + kBlock - 1) / kBlock), kBlock, 0, stream>>>(X, ctl.X[0],
                                                                                     ctl.X[1], L);
    if (cudaGetLastError() != cudaSuccess) return TSE_ERR_LAUNCH;
    return TSE_OK;
}

// smolarkiewicz (tse.py:1083-1116)
__global__ void smolarkiewicz_kernel(TseGrid g, const double* C, const double* qx, const double* qy,
                                     const double* qz, double* vx, double* vy, double* vz,
                                     double dt, double eps, double Sc) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int nx = g.nx, ny = g.ny, nz = g.nz;
    const long long total = (long long)nx * ny * nz;
    if (t >= total) return;
    const int k = (int)(t % nz);
    const long long row = t / nz;
    const int j = (int)(row % ny);
    const int i = (int)(row / ny);
    const double c0 = C[t];
    if (c0 > 0) {
        double dd;
        if (i < nx - 1) {
            const double c1 = C[t + (long long)ny * nz];
            const double q = qx[t];
            dd = 0.5 * (g.dx[i + 1] + g.dx[i]);
            vx[t] = (Sc * (fabs(q) * dd - dt * (q * q)) * (c1 - c0) / ((c0 + c1 + eps) * dd));
        }
        if (j < ny - 1) {
            const double c1 = C[t + nz];
            const double q = qy[t];
            dd = 0.5 * (g.dy[j + 1] + g.dy[j]);
            vy[t] = (Sc * (fabs(q) * dd - dt * (q * q)) * (c1 - c0) / ((c0 + c1 + eps) * dd));
        }
        if (k < nz - 1) {
            const double c1 = C[t + 1];
            const double q = qz[t];
            dd = 0.5 * (g.dz[k + 1] + g.dz[k]);
            vz[t] = (Sc * (fabs(q) * dd - dt * (q * q)) * (c1 - c0) / ((c0 + c1 + eps) * dd));
        }
    } else {
        vx[t] = 0.0;
        vy[t] = 0.0;
        vz[t] = 0.0;
    }
}

}  // namespace tse

using namespace tse;

extern "C" int32_t tse_compute_C(const TseGrid* grid, const TseSpeciesArgs* a,
                                 TseSolveStatus* d_status, void* d_ws, size_t ws_bytes,
                                 void* stream) {
    if (!grid || !a || !d_status || !d_ws) return TSE_ERR_ARG;
    if (grid->nx < 1 || grid->ny < 1 || grid->nz < 1 || a->max_it < 1) return TSE_ERR_ARG;
    if (!a->C || !a->D_fx || !a->D_fy || !a->D_fz || !a->phi || !a->rho_f || !a->qx || !a->qy ||
        !a->qz || !a->BC || !a->WC || !a->RC || !a->e || !a->l_l || !a->l_t)
        return TSE_ERR_ARG;
    return run_transport(grid, a, a->C, d_status, d_ws, ws_bytes, stream, assemble_c_kernel,
                         a->imblflo);
}

extern "C" int32_t tse_compute_T(const TseGrid* grid, const TseHeatArgs* a,
                                 TseSolveStatus* d_status, void* d_ws, size_t ws_bytes,
                                 void* stream) {
    if (!grid || !a || !d_status || !d_ws) return TSE_ERR_ARG;
    if (grid->nx < 1 || grid->ny < 1 || grid->nz < 1 || a->max_it < 1) return TSE_ERR_ARG;
    if (!a->T || !a->l_f || !a->cp_f || !a->rho_f || !a->phi || !a->qx || !a->qy || !a->qz ||
        !a->BT || !a->WT || !a->e || !a->l_r || !a->rho_r || !a->cp_r || !a->l_l || !a->l_t)
        return TSE_ERR_ARG;
    return run_transport(grid, a, a->T, d_status, d_ws, ws_bytes, stream, assemble_t_kernel,
                         a->imblflo);
}

extern "C" int32_t tse_smolarkiewicz(const TseGrid* grid, const double* C, const double* qx,
                                     const double* qy, const double* qz, double* vx, double* vy,
                                     double* vz, double dt, double eps, double Sc, void* stream) {
    if (!grid || !C || !qx || !qy || !qz || !vx || !vy || !vz) return TSE_ERR_ARG;
    const long long n = (long long)grid->nx * grid->ny * grid->nz;
    if (n <= 0) return TSE_ERR_ARG;
    smolarkiewicz_kernel<<<(unsigned)((n + kBlock - 1) / kBlock), kBlock, 0, (cudaStream_t)stream>>>(
        *grid, C, qx, qy, qz, vx, vy, vz, dt, eps, Sc);
    return cudaGetLastError() == cudaSuccess ? TSE_OK : TSE_ERR_LAUNCH;
}
