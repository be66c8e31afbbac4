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
#include "tse_dc.cuh"
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
    // cnt: 1/2 or 1/4 -- dividing by 2 or 4 and multiplying by 0.5 or 0.25
    // round the same exact quotient, so the results are identical
    double q1, q2, q3, q4, cnt;
    if (i != 0) {
        qxl = qx[IX3(i - 1, j, k)];
        q1 = qy[IX3(i - 1, j, k)]; q2 = qy[c]; q3 = q4 = 0; cnt = 0.5;
        if (j != 0) { q3 = qy[IX3(i, j - 1, k)]; q4 = qy[IX3(i - 1, j - 1, k)]; cnt = 0.25; }
        if (!(B[IX3(i - 1, j, k)] != 0)) qxyl = (q1 + q2 + q3 + q4) * cnt;
        q1 = qz[IX3(i - 1, j, k)]; q2 = qz[c]; q3 = q4 = 0; cnt = 0.5;
        if (k != 0) { q3 = qz[IX3(i, j, k - 1)]; q4 = qz[IX3(i - 1, j, k - 1)]; cnt = 0.25; }
        if (!(B[IX3(i - 1, j, k)] != 0)) qxzl = (q1 + q2 + q3 + q4) * cnt;
    }
    if (i != nx - 1) {
        qxr = qx[c];
        q1 = qy[c]; q2 = qy[IX3(i + 1, j, k)]; q3 = q4 = 0; cnt = 0.5;
        if (j != 0) { q3 = qy[IX3(i + 1, j - 1, k)]; q4 = qy[IX3(i, j - 1, k)]; cnt = 0.25; }
        if (!(B[IX3(i + 1, j, k)] != 0)) qxyr = (q1 + q2 + q3 + q4) * cnt;
        q1 = qz[c]; q2 = qz[IX3(i + 1, j, k)]; q3 = q4 = 0; cnt = 0.5;
        if (k != 0) { q3 = qz[IX3(i + 1, j, k - 1)]; q4 = qz[IX3(i, j, k - 1)]; cnt = 0.25; }
        if (!(B[IX3(i + 1, j, k)] != 0)) qxzr = (q1 + q2 + q3 + q4) * cnt;
    }
    if (j != 0) {
        qyl = qy[IX3(i, j - 1, k)];
        q1 = qx[c]; q2 = qx[IX3(i, j - 1, k)]; q3 = q4 = 0; cnt = 0.5;
        if (i != 0) { q3 = qx[IX3(i - 1, j - 1, k)]; q4 = qx[IX3(i - 1, j, k)]; cnt = 0.25; }
        if (!(B[IX3(i, j - 1, k)] != 0)) qyxl = (q1 + q2 + q3 + q4) * cnt;
        q1 = qz[IX3(i, j - 1, k)]; q2 = qz[c]; q3 = q4 = 0; cnt = 0.5;
        if (k != 0) { q3 = qz[IX3(i, j, k - 1)]; q4 = qz[IX3(i, j - 1, k - 1)]; cnt = 0.25; }
        if (!(B[IX3(i, j - 1, k)] != 0)) qyzl = (q1 + q2 + q3 + q4) * cnt;
    }
    if (j != ny - 1) {
        qyr = qy[c];
        q1 = qx[IX3(i, j + 1, k)]; q2 = qx[c]; q3 = q4 = 0; cnt = 0.5;
        if (i != 0) { q3 = qx[IX3(i - 1, j, k)]; q4 = qx[IX3(i - 1, j + 1, k)]; cnt = 0.25; }
        if (!(B[IX3(i, j + 1, k)] != 0)) qyxr = (q1 + q2 + q3 + q4) * cnt;
        q1 = qz[c]; q2 = qz[IX3(i, j + 1, k)]; q3 = q4 = 0; cnt = 0.5;
        if (k != 0) { q3 = qz[IX3(i, j + 1, k - 1)]; q4 = qz[IX3(i, j, k - 1)]; cnt = 0.25; }
        if (!(B[IX3(i, j + 1, k)] != 0)) qyzr = (q1 + q2 + q3 + q4) * cnt;
    }
    if (k != 0) {
        qzl = qz[IX3(i, j, k - 1)];
        q1 = qx[c]; q2 = qx[IX3(i, j, k - 1)]; q3 = q4 = 0; cnt = 0.5;
        if (i != 0) { q3 = qx[IX3(i - 1, j, k - 1)]; q4 = qx[IX3(i - 1, j, k)]; cnt = 0.25; }
        if (!(B[IX3(i, j, k - 1)] != 0)) qzxl = (q1 + q2 + q3 + q4) * cnt;
        q1 = qy[c]; q2 = qy[IX3(i, j, k - 1)]; q3 = q4 = 0; cnt = 0.5;
        if (j != 0) { q3 = qy[IX3(i, j - 1, k - 1)]; q4 = qy[IX3(i, j - 1, k)]; cnt = 0.25; }
        if (!(B[IX3(i, j, k - 1)] != 0)) qzyl = (q1 + q2 + q3 + q4) * cnt;
    }
    if (k != nz - 1) {
        qzr = qz[c];
        q1 = qx[IX3(i, j, k + 1)]; q2 = qx[c]; q3 = q4 = 0; cnt = 0.5;
        if (i != 0) { q3 = qx[IX3(i - 1, j, k)]; q4 = qx[IX3(i - 1, j, k + 1)]; cnt = 0.25; }
        if (!(B[IX3(i, j, k + 1)] != 0)) qzxr = (q1 + q2 + q3 + q4) * cnt;
        q1 = qy[IX3(i, j, k + 1)]; q2 = qy[c]; q3 = q4 = 0; cnt = 0.5;
        if (j != 0) { q3 = qy[IX3(i, j - 1, k)]; q4 = qy[IX3(i, j - 1, k + 1)]; cnt = 0.25; }
        if (!(B[IX3(i, j, k + 1)] != 0)) qzyr = (q1 + q2 + q3 + q4) * cnt;
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

// The assemblies below keep the reference's operations and their order for
// every value they produce, and drop only work whose result is already
// known:
//  - each face's means are formed once, by the face pass, rather than by
//    both cells that share the face (see species_face);
//  - min0(q) / d and max0(q) / d: one of the two is 0 / d, so q / d is formed
//    once and 0 / d (+0 for d > 0) is selected for the other.
// harm2w is harm2(H1, H2, d1, d2) = (d1 + d2) / (d1 / H1 + d2 / H2) with the
// quotients w1 = d1 / H1, w2 = d2 / H2 passed in.
__device__ __forceinline__ double harm2w(double H1, double H2, double d1, double d2, double w1,
                                         double w2) {
    if (H1 != 0.0 && H2 != 0.0) return (d1 + d2) / (w1 + w2);
    return 0.0;
}
__device__ __forceinline__ double zero_over(double d) { return d > 0.0 ? 0.0 : 0.0 / d; }

// One axis of a transport assembly: the + face (toward the next cell along
// the axis) and the - face.  dP/dM: diffusive (and dispersive) coefficients,
// minP/maxP: min0/max0 of the cell's own face flux (scaled), maxM/minM: the
// same for the - neighbour's face flux, coP/coM: upwinded neighbour
// coefficients, oldP/oldM: coP * Xn(+ neighbour), coM * Xn(- neighbour).
struct AxisTerms {
    double dP, dM, minP, maxP, maxM, minM, coP, coM, oldP, oldM;
};

// The means both cells of a face form alike, computed once a face by a pass
// before the assembly (faces_kernel): for a species harm2(D) * amean2(phi),
// the face's value of A (tse.py:811-861); for heat the conductivity mix
// (1 - por) lr + por lf and the mean of rho_f times that of cp_f
// (tse.py:952-1027).  The cell on the + side forms them with the operands
// swapped -- (d1 + d2) / (d1/H1 + d2/H2) and (X1 d1 + X2 d2) / (d1 + d2) --
// and IEEE addition and multiplication commute, so the values are the ones
// each cell would form itself, bit for bit.  Stored per axis for the face
// toward the + neighbour (0 where there is none).
__device__ __forceinline__ void species_face(const double* __restrict__ Df, const double* __restrict__ phi,
                                             const double* __restrict__ d, long long c, long long st,
                                             int ii, bool hp, double phic, double* __restrict__ out) {
    double v = 0.0;
    if (hp) {
        const long long o = c + st;
        const double dd = d[ii], dp = d[ii + 1];
        const double Dc = Df[c], Dp = Df[o];
        v = harm2w(Dp, Dc, dp, dd, dp / Dp, dd / Dc) * amean2(phi[o], phic, dp, dd);
    }
    out[c] = v;
}

__device__ __forceinline__ void heat_face(const TseHeatArgs& a, const double* __restrict__ d, long long c,
                                          long long st, int ii, bool hp, double* __restrict__ k1_out,
                                          double* __restrict__ rc_out) {
    double k1 = 0.0, rc = 0.0;
    if (hp) {
        const long long o = c + st;
        const double dd = d[ii], dp = d[ii + 1];
        const double phic = a.phi[c], lfc = a.l_f[c], lrc = a.l_r[c], cpc = a.cp_f[c], rhc = a.rho_f[c];
        const double php = a.phi[o], lfp = a.l_f[o], lrp = a.l_r[o], cpp = a.cp_f[o], rhp = a.rho_f[o];
        const double por = amean2(phic, php, dd, dp);
        const double lf = harm2w(lfc, lfp, dd, dp, dd / lfc, dp / lfp);
        const double lr = harm2w(lrc, lrp, dd, dp, dd / lrc, dp / lrp);
        const double cpf = harm2w(cpc, cpp, dd, dp, dd / cpc, dp / cpp);
        rc = harm2w(rhc, rhp, dd, dp, dd / rhc, dp / rhp) * cpf;
        k1 = (1 - por) * lr + por * lf;
    }
    k1_out[c] = k1;
    rc_out[c] = rc;
}

// compute_C, one axis (tse.py:811-861): x -> (A, B, N, H, M, G), y -> (C, D,
// P, J, O, I), z -> (E, F, R, L, Q, K); Pf: this axis's face values
__device__ __forceinline__ AxisTerms species_axis(const double* __restrict__ Pf,
                                                  const double* __restrict__ Xn,
                                                  const double* __restrict__ q,
                                                  const double* __restrict__ d, long long c,
                                                  long long st, int ii, bool hp, bool hm,
                                                  double DdP, double DdM) {
    AxisTerms r = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
    const long long op = hp ? c + st : c, om = hm ? c - st : c;
    const double dd = d[ii], dp = d[hp ? ii + 1 : ii], dm = d[hm ? ii - 1 : ii];
    const double xp = Xn[op], xm = Xn[om];
    const double qc = q[c], qm = q[om];
    const double fp = Pf[c], fm = Pf[om];
    const double z = zero_over(dd);
    if (hp) {
        const double dd2 = (0.5 * (dp + dd)) * dd;
        r.dP = (fp + DdP) / dd2;
        const double qd = qc / dd;
        r.minP = (0.0 < qc) ? z : qd;
        r.maxP = (0.0 > qc) ? z : qd;
        r.coP = r.dP - r.minP;
        r.oldP = r.coP * xp;
    }
    if (hm) {
        const double dd2 = (0.5 * (dm + dd)) * dd;
        r.dM = (fm + DdM) / dd2;
        const double qd = qm / dd;
        r.maxM = (0.0 > qm) ? z : qd;
        r.minM = (0.0 < qm) ? z : qd;
        r.coM = r.dM + r.maxM;
        r.oldM = r.coM * xm;
    }
    return r;
}

// compute_T, one axis (tse.py:952-1027); K1, RC: this axis's face values
// (conductivity mix, rho_f cp_f mean)
__device__ __forceinline__ AxisTerms heat_axis(const double* __restrict__ K1, const double* __restrict__ RC,
                                               const double* __restrict__ Xn,
                                               const double* __restrict__ q,
                                               const double* __restrict__ d, long long c,
                                               long long st, int ii, bool hp, bool hm,
                                               double DdP, double DdM) {
    AxisTerms r = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
    const long long op = hp ? c + st : c, om = hm ? c - st : c;
    const double dd = d[ii], dp = d[hp ? ii + 1 : ii], dm = d[hm ? ii - 1 : ii];
    const double qc = q[c], qm = q[om];
    if (hp) {
        const double dd2 = (0.5 * (dp + dd)) * dd;
        const double rhocpf = RC[c];
        r.dP = (K1[c] + DdP * rhocpf) / dd2;
        const double S = rhocpf / dd;
        r.minP = min0(qc) * S;
        r.maxP = max0(qc) * S;
        r.coP = r.dP - r.minP;
        r.oldP = r.coP * Xn[op];
    }
    if (hm) {
        const double dd2 = (0.5 * (dm + dd)) * dd;
        const double rhocpf = RC[om];
        r.dM = (K1[om] + DdM * rhocpf) / dd2;
        const double S = rhocpf / dd;
        r.maxM = max0(qm) * S;
        r.minM = min0(qm) * S;
        r.coM = r.dM + r.maxM;
        r.oldM = r.coM * Xn[om];
    }
    return r;
}

// The per-cell terms of a transport solve: the six neighbour coefficients
// (x+, x-, y+, y-, z+, z-), M, (1-omega)-part Mo, R and its numerator, source,
// IMBLFLO term and the neighbour sum of the initial iterate in sum()'s order.
struct TransportTerms {
    double co[6];
    double s, Mo, Xn, Rnum, R, M, W, EX;
    bool active;
};

__device__ __forceinline__ void combine_axes(const AxisTerms& X, const AxisTerms& Y,
                                             const AxisTerms& Z, double Xn, TransportTerms& T) {
    T.co[0] = X.coP;
    T.co[1] = X.coM;
    T.co[2] = Y.coP;
    T.co[3] = Y.coM;
    T.co[4] = Z.coP;
    T.co[5] = Z.coM;
    // M = -A - B - C - D - E - F + G - H + I - J + K - L (tse.py:863, 1029)
    T.M = -X.dP - X.dM - Y.dP - Y.dM - Z.dP - Z.dM + X.minM - X.maxP + Y.minM - Y.maxP + Z.minM -
          Z.maxP;
    T.Xn = Xn;
    T.Mo = Xn * T.M + X.oldP + X.oldM + Y.oldP + Y.oldM + Z.oldP + Z.oldM;
    double s = X.oldP;
    s = s + X.oldM;
    s = s + Y.oldP;
    s = s + Y.oldM;
    s = s + Z.oldP;
    s = s + Z.oldM;
    T.s = s;
}

// coefficient part of compute_C.solve (tse.py:795-868)
__device__ __forceinline__ void species_terms(const TseGrid& g, const TseSpeciesArgs& a,
                                              const CellIdx& x, const Layout& L,
                                              const double* __restrict__ faces, TransportTerms& T) {
    const int nx = L.nx, ny = L.ny, nz = L.nz, i = x.i, j = x.j, k = x.k;
    const long long c = x.c;
    double Dd[6] = {0, 0, 0, 0, 0, 0};
    if (a.l_l[c] != 0 || a.l_t[c] != 0)
        dispersivity_dev(a.qx, a.qy, a.qz, a.l_l, a.l_t, a.BC, i, j, k, nx, ny, nz, Dd);
    const long long n = (long long)nx * ny * nz;
    const AxisTerms X = species_axis(faces, a.C, a.qx, g.dx, c, (long long)ny * nz, i, i != nx - 1,
                                     i != 0, Dd[3], Dd[0]);
    const AxisTerms Y = species_axis(faces + n, a.C, a.qy, g.dy, c, nz, j, j != ny - 1, j != 0,
                                     Dd[4], Dd[1]);
    const AxisTerms Z = species_axis(faces + 2 * n, a.C, a.qz, g.dz, c, 1, k, k != nz - 1, k != 0,
                                     Dd[5], Dd[2]);
    const double phic = a.phi[c];
    const double Xn = a.C[c];
    combine_axes(X, Y, Z, Xn, T);
    T.Rnum = a.RC[c] * phic;
    T.R = T.Rnum / a.dt;
    T.EX = a.imblflo ? Xn / a.rho_f[c] * a.e[c] : 0.0;
    T.W = a.WC[c];
    T.active = !(a.BC[c] != 0.0);
}

// coefficient part of compute_T.solve (tse.py:930-1036)
__device__ __forceinline__ void heat_terms(const TseGrid& g, const TseHeatArgs& a, const CellIdx& x,
                                           const Layout& L, const double* __restrict__ faces,
                                           TransportTerms& T) {
    const int nx = L.nx, ny = L.ny, nz = L.nz, i = x.i, j = x.j, k = x.k;
    const long long c = x.c;
    double Dd[6] = {0, 0, 0, 0, 0, 0};
    if (a.l_l[c] != 0 || a.l_t[c] != 0)
        dispersivity_dev(a.qx, a.qy, a.qz, a.l_l, a.l_t, a.BT, i, j, k, nx, ny, nz, Dd);
    const long long n = (long long)nx * ny * nz;
    const AxisTerms X = heat_axis(faces, faces + 3 * n, a.T, a.qx, g.dx, c, (long long)ny * nz, i,
                                  i != nx - 1, i != 0, Dd[3], Dd[0]);
    const AxisTerms Y = heat_axis(faces + n, faces + 4 * n, a.T, a.qy, g.dy, c, nz, j, j != ny - 1,
                                  j != 0, Dd[4], Dd[1]);
    const AxisTerms Z = heat_axis(faces + 2 * n, faces + 5 * n, a.T, a.qz, g.dz, c, 1, k, k != nz - 1,
                                  k != 0, Dd[5], Dd[2]);
    const double Xn = a.T[c];
    combine_axes(X, Y, Z, Xn, T);
    const double por_ = a.phi[c];
    T.Rnum = por_ * a.rho_f[c] * a.cp_f[c] + (1 - por_) * a.rho_r[c] * a.cp_r[c];
    T.R = T.Rnum / a.dt;
    T.EX = a.imblflo ? a.cp_f[c] * Xn * a.e[c] : 0.0;
    T.W = a.WT[c];
    T.active = !(a.BT[c] != 0.0);
}

// The exact form's per-cell arrays (TransportForm) and the flag byte.
__device__ __forceinline__ void store_terms(const TransportForm& F, uint8_t* msk, const CellIdx& x,
                                            const TransportTerms& T, int nx, int ny, int nz) {
    double* b = F.arr[x.col];
    const long long N = F.Ncal, m = x.m;
    const double omega = F.omega;
    for (int q = 0; q < 6; ++q) b[q * N + m] = T.co[q];
    // the (1-omega) part and the IMBLFLO term are read only where the form
    // uses them (TransportForm::useY / useEX)
    if (F.useY) b[TA_Y * N + m] = (1 - omega) * T.Mo;
    b[TA_RXN * N + m] = T.R * T.Xn;
    b[TA_W * N + m] = T.W;
    if (F.useEX) b[TA_EX * N + m] = T.EX;
    b[TA_DEN * N + m] = T.R - omega * T.M;
    b[TA_RNUM * N + m] = T.Rnum;
    b[TA_M * N + m] = T.M;
    b[TA_XN * N + m] = T.Xn;
    b[TA_X * N + m] = T.Xn;
    uint8_t f = neighbour_flags(x.i, x.j, x.k, nx, ny, nz);
    if (T.active) f |= F_ACTIVE;
    msk[m] = f;
}

__device__ __forceinline__ void store_padding(const TransportForm& F, uint8_t* msk, const CellIdx& x) {
    double* b = F.arr[x.col];
    for (int q = 0; q < TA_COUNT; ++q) b[q * F.Ncal + x.m] = 0.0;
    msk[x.m] = 0;
}

// The first correction cycle of the mixed-precision form (DcFuse): K'_q =
// omega co_q / Den, and r' with sum() of TransportForm, whose neighbour
// products are the assembly's own co_q * Xn_q.
__device__ __forceinline__ void store_dc(const TransportForm& F, const DcFuse& fz, const CellIdx& x,
                                         const TransportTerms* T) {
    float* Kc = fz.K[x.col];
    float2* rec = reinterpret_cast<float2*>(Kc + 6 * x.m);
    float rp = 0.0f;
    if (T && T->active) {
        const double omega = F.omega;
        const double den = T->R - omega * T->M;
        const double rden = 1.0 / den;
#pragma unroll
        for (int q = 0; q < 3; ++q)
            rec[q] = make_float2((float)(omega * T->co[2 * q] * rden),
                                 (float)(omega * T->co[2 * q + 1] * rden));
        double num = omega * T->s;
        if (F.useY) num = num + (1 - omega) * T->Mo;
        num = num + T->R * T->Xn;
        num = num + T->W;
        num = num - (F.useEX ? T->EX : 0.0);
        rp = (float)((num - den * T->Xn) * rden);
    } else {
#pragma unroll
        for (int q = 0; q < 3; ++q) rec[q] = make_float2(0.0f, 0.0f);
    }
    Kc[6 * fz.Ncal + x.m] = rp;
}

struct SpeciesKind {
    using Args = TseSpeciesArgs;
    static __device__ __forceinline__ void terms(const TseGrid& g, const Args& a, const CellIdx& x,
                                                 const Layout& L, const double* faces,
                                                 TransportTerms& T) {
        species_terms(g, a, x, L, faces, T);
    }
    // the face pass, one cell (natural order)
    static __device__ __forceinline__ void faces(const TseGrid& g, const Args& a, const Layout& L,
                                                 long long c, int i, int j, int k, double* out) {
        const long long n = (long long)L.nx * L.ny * L.nz;
        const double phic = a.phi[c];
        species_face(a.D_fx, a.phi, g.dx, c, (long long)L.ny * L.nz, i, i != L.nx - 1, phic, out);
        species_face(a.D_fy, a.phi, g.dy, c, L.nz, j, j != L.ny - 1, phic, out + n);
        species_face(a.D_fz, a.phi, g.dz, c, 1, k, k != L.nz - 1, phic, out + 2 * n);
    }
};
struct HeatKind {
    using Args = TseHeatArgs;
    static __device__ __forceinline__ void terms(const TseGrid& g, const Args& a, const CellIdx& x,
                                                 const Layout& L, const double* faces,
                                                 TransportTerms& T) {
        heat_terms(g, a, x, L, faces, T);
    }
    static __device__ __forceinline__ void faces(const TseGrid& g, const Args& a, const Layout& L,
                                                 long long c, int i, int j, int k, double* out) {
        const long long n = (long long)L.nx * L.ny * L.nz;
        heat_face(a, g.dx, c, (long long)L.ny * L.nz, i, i != L.nx - 1, out, out + 3 * n);
        heat_face(a, g.dy, c, L.nz, j, j != L.ny - 1, out + n, out + 4 * n);
        heat_face(a, g.dz, c, 1, k, k != L.nz - 1, out + 2 * n, out + 5 * n);
    }
};

// Both assemblies are bound by the latency of their loads (15 input arrays,
// neighbours included).  Four 256-thread blocks per SM (64 registers, some
// spilled): with the face values read from the face pass, measured on the
// 256 x 256 x 128 reservoir (whole calls, one box, one call each), a species
// solve of 5 iterations took 1.65 ms at four blocks, 1.89 at three and 2.09 at
// two (heat, 3 iterations: 1.39, 1.51, 1.65 ms).
#ifndef TSE_ASM_MINB
#define TSE_ASM_MINB 4
#endif
constexpr int kAssembleMinBlocks = TSE_ASM_MINB;

// One thread per cell of the padded natural order (DC: per_thread
// consecutive blocks of kBlock cells each, so the x^2 partials stay few).
template <class Kind, bool DC>
__device__ __forceinline__ void assemble_body(const TseGrid& g, const typename Kind::Args& a,
                                              const TransportForm& F, uint8_t* mask0,
                                              uint8_t* mask1, const Layout& L,
                                              const double* __restrict__ faces, const DcFuse& fz) {
    __shared__ double sh[kBlock / 32];
    double x2 = 0.0;
    const int per = DC ? fz.per_thread : 1;
    for (int s = 0; s < per; ++s) {
        CellIdx x;
        const long long t = ((long long)blockIdx.x * per + s) * kBlock + threadIdx.x;
        if (!decode_padded(t, L, x)) break;
        uint8_t* msk = x.col ? mask1 : mask0;
        if (x.pad) {
            store_padding(F, msk, x);
            if (DC) store_dc(F, fz, x, nullptr);
            continue;
        }
        TransportTerms T;
        Kind::terms(g, a, x, L, faces, T);
        store_terms(F, msk, x, T, L.nx, L.ny, L.nz);
        if (DC) {
            store_dc(F, fz, x, &T);
            x2 = x2 + T.Xn * T.Xn;
        }
    }
    if (DC) {
        const double b = block_sum<kBlock>(x2, sh);
        if (threadIdx.x == 0) fz.partials[blockIdx.x] = b;
    }
}

// coefficient part of compute_C.solve (tse.py:795-868)
template <bool DC>
__global__ void __launch_bounds__(kBlock, kAssembleMinBlocks)
    assemble_c_kernel(TseGrid g, TseSpeciesArgs a, TransportForm F, uint8_t* mask0, uint8_t* mask1,
                      Layout L, const double* faces, DcFuse fz) {
    assemble_body<SpeciesKind, DC>(g, a, F, mask0, mask1, L, faces, fz);
}

// coefficient part of compute_T.solve (tse.py:930-1036)
template <bool DC>
__global__ void __launch_bounds__(kBlock, kAssembleMinBlocks)
    assemble_t_kernel(TseGrid g, TseHeatArgs a, TransportForm F, uint8_t* mask0, uint8_t* mask1,
                      Layout L, const double* faces, DcFuse fz) {
    assemble_body<HeatKind, DC>(g, a, F, mask0, mask1, L, faces, fz);
}

// the face pass before an assembly: one thread per cell, natural order
template <class Kind>
__global__ void faces_kernel(TseGrid g, typename Kind::Args a, Layout L, double* faces) {
    const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= (long long)L.nx * L.ny * L.nz) return;
    int i, j, k;
    long long row;
    grid_coords(c, L.ny, L.nz, i, j, k, row);
    Kind::faces(g, a, L, c, i, j, k, faces);
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

// face values a cell: 3 for a species, 6 for heat
constexpr int kTransportFaceWords = 6;

size_t transport_ws_bytes(const Layout& L, long long* Ncal_out) {
    long long Ncal = (L.Nc + 31) & ~31LL;
    if (Ncal_out) *Ncal_out = Ncal;
    size_t b = 0;
    b += align256(sizeof(GridBarrier));
    b += align256((size_t)2 * kMaxBlocks * sizeof(double));
    b += 2 * align256((size_t)Ncal);
    b += 2 * (size_t)TA_COUNT * Ncal * sizeof(double);
    b += align256((size_t)kTransportFaceWords * L.nx * L.ny * L.nz * sizeof(double));   // face pass
    return b;
}

// Carve the workspace (shared by the exact and the defect-correction
// transport solves) and reset the grid barrier.
template <class Args>
static int carve_transport(const TseGrid* grid, const Args* a, void* d_ws, size_t ws_bytes,
                           cudaStream_t stream, int imbl, TransportSetup& S) {
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
    S.faces = S.F.arr[1] + (size_t)TA_COUNT * S.Ncal;
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
    return TSE_OK;
}

// carve + the exact form's assembly
// the face pass of a transport setup
template <class Args, class FacesK>
static void launch_faces(const TseGrid* grid, const Args* a, const TransportSetup& S, FacesK fk,
                         cudaStream_t stream) {
    const long long n = (long long)S.L.nx * S.L.ny * S.L.nz;
    fk<<<(unsigned)((n + kBlock - 1) / kBlock), kBlock, 0, stream>>>(*grid, *a, S.L, S.faces);
}

// carve + the face pass + the exact form's assembly
template <class Args, class FacesK, class AssembleK>
static int setup_transport(const TseGrid* grid, const Args* a, void* d_ws, size_t ws_bytes,
                           cudaStream_t stream, FacesK fk, AssembleK kernel, int imbl,
                           TransportSetup& S) {
    int rc = carve_transport(grid, a, d_ws, ws_bytes, stream, imbl, S);
    if (rc != TSE_OK) return rc;
    launch_faces(grid, a, S, fk, stream);
    const long long total = (long long)S.L.nx * S.L.ny * S.L.nzp;
    kernel<<<(unsigned)((total + kBlock - 1) / kBlock), kBlock, 0, stream>>>(
        *grid, *a, S.F, S.mask[0], S.mask[1], S.L, S.faces, DcFuse{});
    return cudaGetLastError() == cudaSuccess ? TSE_OK : TSE_ERR_LAUNCH;
}

// carve + the assembly that also writes the mixed-precision form's first
// cycle (records, r', x^2 partials); *nparts: the number of partials
template <class Args, class FacesK, class AssembleK>
static int setup_transport_dc(const TseGrid* grid, const Args* a, void* d_ws, size_t ws_bytes,
                              cudaStream_t stream, FacesK fk, AssembleK kernel, int imbl,
                              TransportSetup& S, int* nparts) {
    int rc = carve_transport(grid, a, d_ws, ws_bytes, stream, imbl, S);
    if (rc != TSE_OK) return rc;
    if (S.tail_bytes < dc_extra_bytes(S.L)) return TSE_ERR_WORKSPACE;
    launch_faces(grid, a, S, fk, stream);
    DcCtl c;
    dc_carve(S, c, TA_X);
    long long per, nb;
    dc_fuse_grid(S.L, per, nb);
    DcFuse fz;
    fz.K[0] = c.K[0];
    fz.K[1] = c.K[1];
    fz.Ncal = c.Ncal;
    fz.partials = S.partials;
    fz.per_thread = (int)per;
    kernel<<<(unsigned)nb, kBlock, 0, stream>>>(*grid, *a, S.F, S.mask[0], S.mask[1], S.L, S.faces,
                                                 fz);
    *nparts = (int)nb;
    return cudaGetLastError() == cudaSuccess ? TSE_OK : TSE_ERR_LAUNCH;
}

int setup_species(const TseGrid* grid, const TseSpeciesArgs* a, void* d_ws, size_t ws_bytes,
                  cudaStream_t stream, TransportSetup& S) {
    return setup_transport(grid, a, d_ws, ws_bytes, stream, faces_kernel<SpeciesKind>,
                           assemble_c_kernel<false>, a->imblflo, S);
}

int setup_heat(const TseGrid* grid, const TseHeatArgs* a, void* d_ws, size_t ws_bytes,
               cudaStream_t stream, TransportSetup& S) {
    return setup_transport(grid, a, d_ws, ws_bytes, stream, faces_kernel<HeatKind>,
                           assemble_t_kernel<false>, a->imblflo, S);
}

int setup_species_dc(const TseGrid* grid, const TseSpeciesArgs* a, void* d_ws, size_t ws_bytes,
                     cudaStream_t stream, TransportSetup& S, int* nparts) {
    return setup_transport_dc(grid, a, d_ws, ws_bytes, stream, faces_kernel<SpeciesKind>,
                              assemble_c_kernel<true>, a->imblflo, S, nparts);
}

int setup_heat_dc(const TseGrid* grid, const TseHeatArgs* a, void* d_ws, size_t ws_bytes,
                  cudaStream_t stream, TransportSetup& S, int* nparts) {
    return setup_transport_dc(grid, a, d_ws, ws_bytes, stream, faces_kernel<HeatKind>,
                              assemble_t_kernel<true>, a->imblflo, S, nparts);
}

template <class Args, class FacesK, class AssembleK>
static int run_transport(const TseGrid* grid, const Args* a, double* X, TseSolveStatus* d_status,
                         void* d_ws, size_t ws_bytes, void* stream_, FacesK fk, AssembleK kernel,
                         int imbl) {
    cudaStream_t stream = (cudaStream_t)stream_;
    TransportSetup S;
    int rc = setup_transport(grid, a, d_ws, ws_bytes, stream, fk, kernel, imbl, S);
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
    return run_transport(grid, a, a->C, d_status, d_ws, ws_bytes, stream, faces_kernel<SpeciesKind>,
                         assemble_c_kernel<false>, a->imblflo);
}

extern "C" int32_t tse_compute_T(const TseGrid* grid, const TseHeatArgs* a,
                                 TseSolveStatus* d_status, void* d_ws, size_t ws_bytes,
                                 void* stream) {
    if (!grid || !a || !d_status || !d_ws) return TSE_ERR_ARG;
    if (grid->nx < 1 || grid->ny < 1 || grid->nz < 1 || a->max_it < 1) return TSE_ERR_ARG;
    if (!a->T || !a->l_f || !a->cp_f || !a->rho_f || !a->phi || !a->qx || !a->qy || !a->qz ||
        !a->BT || !a->WT || !a->e || !a->l_r || !a->rho_r || !a->cp_r || !a->l_l || !a->l_t)
        return TSE_ERR_ARG;
    return run_transport(grid, a, a->T, d_status, d_ws, ws_bytes, stream, faces_kernel<HeatKind>,
                         assemble_t_kernel<false>, a->imblflo);
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
