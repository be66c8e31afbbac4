/*
 * tse_oracle.c -- THE ORACLE (test infrastructure, never the product).
 *
 * CPU FP64 restatement of the TRANSPORTSE time-step kernels of tse.py
 * (thkempka/transportse).  Each function keeps the reference's operation
 * order term by term (Python evaluates + - * / left to right) so that, built
 * with -ffp-contract=off (no FMA contraction, like numba with
 * fastmath=False), results agree bit for bit with the numba-compiled
 * reference on the same inputs.
 *
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU baseline / reference
 * arm load this library, and only as the checker or as the timed CPU baseline.
 *
 * Layout: every field is a C-order (nx, ny, nz) float64 array (k fastest), as
 * in tse.py:81-157; species fields are handed over one species at a time as
 * contiguous (nx, ny, nz) arrays.  The grid-wide globals that numba freezes at
 * first compilation (dx, dy, dz, g, beta, c_r, l_r, rho_r, cp_r, the
 * dispersivities and the IMBLFLO flags, tse.py:249-1116) are passed in
 * explicitly.
 *
 * Threading: the colour sweeps are parallel over i with OpenMP, like the
 * prange loops of the reference; the per-iteration copy and the L2 norm are
 * serial, as in tse.py:702, 880, 1048 and tse.py:273-281.
 */
#include <math.h>
#include <stddef.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

typedef struct {
    int nx, ny, nz;
    const double *dx, *dy, *dz;
    double g;
    double sinb, cosb;   /* numpy.sin(beta), numpy.cos(beta), evaluated by the caller */
} og_grid;

#define IX(i, j, k) ((((size_t)(i)) * (size_t)ny + (size_t)(j)) * (size_t)nz + (size_t)(k))

/* min(q, 0) / max(q, 0) with Python's builtin semantics (the first argument
 * is kept unless the second compares strictly smaller / larger). */
static inline double min0(double q) { return (0.0 < q) ? 0.0 : q; }
static inline double max0(double q) { return (0.0 > q) ? 0.0 : q; }

/* Python's min(a, b) for floats: b if b < a else a (dt clamps, explicit_C). */
static inline double pymin(double a, double b) { return (b < a) ? b : a; }

/* harm, tse.py:297-310: spacing-weighted harmonic mean, 0 if either is 0. */
static inline double harm2(double H1, double H2, double d1, double d2)
{
    if (H1 != 0 && H2 != 0)
        return (d1 + d2) / (d1 / H1 + d2 / H2);
    return 0.0;
}

/* amean, tse.py:284-294: spacing-weighted arithmetic mean. */
static inline double amean2(double X1, double X2, double d1, double d2)
{
    return (X1 * d1 + X2 * d2) / (d1 + d2);
}

/* l2_norm, tse.py:273-281 (serial sums in C order; NaN -> 1). */
double og_l2_norm(const double *New, const double *Old, size_t n)
{
    double s1 = 0.0, s2 = 0.0;
    for (size_t f = 0; f < n; ++f) {
        double d = New[f] - Old[f];
        s1 += d * d;
    }
    for (size_t f = 0; f < n; ++f)
        s2 += Old[f] * Old[f];
    double l2 = sqrt(s1) / sqrt(s2 + 1e-200);
    if (isnan(l2))
        return 1.0;
    return l2;
}

/* ------------------------------------------------------------------------ */
/* compute_P, tse.py:647-742                                                */
/* ------------------------------------------------------------------------ */

typedef struct {
    const double *c_f, *nue, *rho, *phi, *Kx, *Ky, *Kz, *c_r, *BP, *WP;
} og_pfields;

/* alpha, tse.py:249-260, with the d[d2] * (d[d1] + d[d2]) * 0.5 denominator */
static inline double alpha_(double K1, double K2, double n1, double n2,
                            double r1, double r2, double d1, double d2,
                            double dden1, double dden2)
{
    return harm2(K1, K2, d1, d2) / harm2(n1, n2, d1, d2)
           / (dden2 * (dden1 + dden2) * 0.5) * harm2(r1, r2, d1, d2);
}

static double solve_p(const og_grid *G, const og_pfields *F, double *P,
                      const double *Pn, double dt_P, double SOR,
                      int i, int j, int k)
{
    const int nx = G->nx, ny = G->ny, nz = G->nz;
    const double *dx = G->dx, *dy = G->dy, *dz = G->dz;
    const double *nue = F->nue, *rho = F->rho;
    const size_t c = IX(i, j, k);
    double A_ = 0, B_ = 0, C_ = 0, D_ = 0, E_ = 0, G_ = 0, I_ = 0, J_ = 0,
           K_ = 0, L_ = 0, Anew = 0, Cnew = 0, Enew = 0, Gnew = 0, Inew = 0,
           Knew = 0;
    if (i != nx - 1) {
        size_t o = IX(i + 1, j, k);
        /* alpha(i+1,j,k, i,j,k, ..., dx, i+1, i, 0) */
        A_ = alpha_(F->Kx[o], F->Kx[c], nue[o], nue[c], rho[o], rho[c],
                    dx[i + 1], dx[i], dx[i + 1], dx[i]);
        Anew = A_ * P[o];
        B_ = amean2(rho[o], rho[c], dx[i + 1], dx[i]) * G->g * 0.5
             * (dx[i + 1] + dx[i]) * G->sinb;
    }
    if (i != 0) {
        size_t o = IX(i - 1, j, k);
        /* alpha(i,j,k, i-1,j,k, ..., dx, i-1, i, 0) */
        C_ = alpha_(F->Kx[c], F->Kx[o], nue[c], nue[o], rho[c], rho[o],
                    dx[i], dx[i - 1], dx[i - 1], dx[i]);
        Cnew = C_ * P[o];
        D_ = amean2(rho[c], rho[o], dx[i], dx[i - 1]) * G->g * 0.5
             * (dx[i] + dx[i - 1]) * G->sinb;
    }
    if (j != ny - 1) {
        size_t o = IX(i, j + 1, k);
        E_ = alpha_(F->Ky[o], F->Ky[c], nue[o], nue[c], rho[o], rho[c],
                    dy[j + 1], dy[j], dy[j + 1], dy[j]);
        Enew = E_ * P[o];
    }
    if (j != 0) {
        size_t o = IX(i, j - 1, k);
        G_ = alpha_(F->Ky[c], F->Ky[o], nue[c], nue[o], rho[c], rho[o],
                    dy[j], dy[j - 1], dy[j - 1], dy[j]);
        Gnew = G_ * P[o];
    }
    if (k != nz - 1) {
        size_t o = IX(i, j, k + 1);
        I_ = alpha_(F->Kz[o], F->Kz[c], nue[o], nue[c], rho[o], rho[c],
                    dz[k + 1], dz[k], dz[k + 1], dz[k]);
        Inew = I_ * P[o];
        J_ = amean2(rho[o], rho[c], dz[k + 1], dz[k]) * G->g * 0.5
             * (dz[k + 1] + dz[k]) * G->cosb;
    }
    if (k != 0) {
        size_t o = IX(i, j, k - 1);
        K_ = alpha_(F->Kz[c], F->Kz[o], nue[c], nue[o], rho[c], rho[o],
                    dz[k], dz[k - 1], dz[k - 1], dz[k]);
        Knew = K_ * P[o];
        L_ = amean2(rho[c], rho[o], dz[k], dz[k - 1]) * G->g * 0.5
             * (dz[k] + dz[k - 1]) * G->cosb;
    }
    double por = F->phi[c];
    double R = (rho[c] * ((1 - por) * F->c_r[c] + por * F->c_f[c]) / dt_P);
    double M = A_ + C_ + E_ + G_ + I_ + K_;
    return (1 - SOR) * P[c] + SOR * (Anew + A_ * B_ + Cnew - C_ * D_ + Enew
                                     + Gnew + Inew + I_ * J_ + Knew - K_ * L_
                                     + R * Pn[c] + F->WP[c]) / (R + M);
}

static void sweep_p(const og_grid *G, const og_pfields *F, double *P,
                    const double *Pn, double dt_P, double SOR, int colour)
{
    const int nx = G->nx, ny = G->ny, nz = G->nz;
#pragma omp parallel for schedule(static)
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny; ++j)
            for (int k = ((i + j + colour) & 1); k < nz; k += 2) {
                size_t c = IX(i, j, k);
                if (!(F->BP[c] != 0))
                    P[c] = solve_p(G, F, P, Pn, dt_P, SOR, i, j, k);
            }
}

/* Outputs: out[0] = t_P, out[1] = dt_P, out[2] = converged, out[3] = num_it,
 * out[4] = last L2 diff, out[5] = number of dt halvings.  P is updated in
 * place (after a reset it holds the restarted iterate, as the rebinding at
 * tse.py:738 does); Pn receives the entry value of P. */
int og_compute_P(const og_grid *G, const og_pfields *F, double *P, double *Pn,
                 double dt_P, double SOR, int max_it, double inc_it,
                 double max_dt, double min_dt, double P_conv, double *out)
{
    const size_t n = (size_t)G->nx * G->ny * G->nz;
    double *Pold = (double *)malloc(n * sizeof(double));
    if (!Pold)
        return -1;
    double t_P = 0;
    int converged = 0, num_it = 0, num_sub_it = 0, halvings = 0;
    double diff = 1e100;
    memcpy(Pn, P, n * sizeof(double));
    while (!converged) {
        num_it += 1;
        num_sub_it += 1;
        memcpy(Pold, P, n * sizeof(double));
        sweep_p(G, F, P, Pn, dt_P, SOR, 0);
        sweep_p(G, F, P, Pn, dt_P, SOR, 1);
        diff = 1e100;
        if (num_it < 50)
            diff = og_l2_norm(P, Pold, n);
        else if (num_it % 10 == 0)
            diff = og_l2_norm(P, Pold, n);
        if (diff < P_conv) {
            converged = 1;
            t_P += dt_P;
            if (num_sub_it < max_it / 2.0)
                dt_P = pymin(dt_P * inc_it, max_dt);
        } else {
            converged = 0;
            if (num_sub_it >= max_it) {
                dt_P = dt_P / 2;
                num_sub_it = 0;
                halvings += 1;
                memcpy(P, Pn, n * sizeof(double));
            }
            if (dt_P <= min_dt)
                break;
        }
    }
    free(Pold);
    out[0] = t_P;
    out[1] = dt_P;
    out[2] = converged;
    out[3] = num_it;
    out[4] = diff;
    out[5] = halvings;
    return 0;
}

/* ------------------------------------------------------------------------ */
/* compute_q, tse.py:744-780 (the last plane of each component is untouched) */
/* ------------------------------------------------------------------------ */
void og_compute_q(const og_grid *G, const double *P, const double *BP,
                  const double *Kx, const double *Ky, const double *Kz,
                  double *qx, double *qy, double *qz, const double *nue,
                  const double *rho)
{
    const int nx = G->nx, ny = G->ny, nz = G->nz;
    const double *dx = G->dx, *dy = G->dy, *dz = G->dz;
#pragma omp parallel for schedule(static)
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny; ++j)
            for (int k = 0; k < nz; ++k) {
                size_t c = IX(i, j, k);
                if (i < nx - 1) {
                    size_t o = IX(i + 1, j, k);
                    if (!(BP[c] != 0 && BP[o] != 0))
                        qx[c] = (-harm2(Kx[o], Kx[c], dx[i + 1], dx[i])
                                 / harm2(nue[o], nue[c], dx[i + 1], dx[i])
                                 * ((P[o] - P[c]) / (0.5 * (dx[i + 1] + dx[i]))
                                    + amean2(rho[o], rho[c], dx[i + 1], dx[i])
                                      * G->g * G->sinb));
                    else
                        qx[c] = 0;
                }
                if (j < ny - 1) {
                    size_t o = IX(i, j + 1, k);
                    if (!(BP[c] != 0 && BP[o] != 0))
                        qy[c] = (-harm2(Ky[o], Ky[c], dy[j + 1], dy[j])
                                 / harm2(nue[o], nue[c], dy[j + 1], dy[j])
                                 * (P[o] - P[c]) / (0.5 * (dy[j + 1] + dy[j])));
                    else
                        qy[c] = 0;
                }
                if (k < nz - 1) {
                    size_t o = IX(i, j, k + 1);
                    if (!(BP[c] != 0 && BP[o] != 0))
                        qz[c] = (-harm2(Kz[o], Kz[c], dz[k + 1], dz[k])
                                 / harm2(nue[o], nue[c], dz[k + 1], dz[k])
                                 * ((P[o] - P[c]) / (0.5 * (dz[k + 1] + dz[k]))
                                    + amean2(rho[o], rho[c], dz[k + 1], dz[k])
                                      * G->g * G->cosb));
                    else
                        qz[c] = 0;
                }
            }
}

/* ------------------------------------------------------------------------ */
/* flow_error, tse.py:409-446                                               */
/* ------------------------------------------------------------------------ */
void og_flow_error(const og_grid *G, const double *P, const double *Pn,
                   const double *qx, const double *qy, const double *qz,
                   const double *WP, const double *phi, const double *c_f,
                   const double *c_r, const double *rho, double dt_P, double *e)
{
    const int nx = G->nx, ny = G->ny, nz = G->nz;
    const double *dx = G->dx, *dy = G->dy, *dz = G->dz;
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny; ++j)
            for (int k = 0; k < nz; ++k) {
                size_t c = IX(i, j, k);
                double v = 0.0;
                if (i != nx - 1)
                    v -= (qx[c] / dx[i] * harm2(rho[IX(i + 1, j, k)], rho[c], dx[i + 1], dx[i]));
                if (i != 0)
                    v += (qx[IX(i - 1, j, k)] / dx[i] * harm2(rho[IX(i - 1, j, k)], rho[c], dx[i - 1], dx[i]));
                if (j != ny - 1)
                    v -= (qy[c] / dy[j] * harm2(rho[IX(i, j + 1, k)], rho[c], dy[j + 1], dy[j]));
                if (j != 0)
                    v += (qy[IX(i, j - 1, k)] / dy[j] * harm2(rho[IX(i, j - 1, k)], rho[c], dy[j - 1], dy[j]));
                if (k != nz - 1)
                    v -= (qz[c] / dz[k] * harm2(rho[IX(i, j, k + 1)], rho[c], dz[k + 1], dz[k]));
                if (k != 0)
                    v += (qz[IX(i, j, k - 1)] / dz[k] * harm2(rho[IX(i, j, k - 1)], rho[c], dz[k - 1], dz[k]));
                double por = phi[c];
                v += (WP[c] + ((1 - por) * c_r[c] + por * c_f[c])
                      * (P[c] - Pn[c]) * rho[c] / dt_P);
                e[c] = v;
            }
}

/* ------------------------------------------------------------------------ */
/* dispersivity, tse.py:460-644                                             */
/* ------------------------------------------------------------------------ */
static void dispersivity_(const og_grid *G, const double *qx, const double *qy,
                          const double *qz, const double *l_l, const double *l_t,
                          const double *B, int i, int j, int k, double *Dout)
{
    const int nx = G->nx, ny = G->ny, nz = G->nz;
    double qxl = 0, qyl = 0, qzl = 0, qxr = 0, qyr = 0, qzr = 0;
    double qxyl = 0, qxzl = 0, qyxl = 0, qyzl = 0, qzxl = 0, qzyl = 0;
    double qxyr = 0, qxzr = 0, qyxr = 0, qyzr = 0, qzxr = 0, qzyr = 0;
    double q1, q2, q3, q4, cnt;
    if (i != 0) {
        qxl = qx[IX(i - 1, j, k)];
        q1 = qy[IX(i - 1, j, k)]; q2 = qy[IX(i, j, k)]; q3 = q4 = 0; cnt = 2;
        if (j != 0) { q3 = qy[IX(i, j - 1, k)]; q4 = qy[IX(i - 1, j - 1, k)]; cnt += 2; }
        if (!(B[IX(i - 1, j, k)] != 0)) qxyl = (q1 + q2 + q3 + q4) / cnt;
        q1 = qz[IX(i - 1, j, k)]; q2 = qz[IX(i, j, k)]; q3 = q4 = 0; cnt = 2;
        if (k != 0) { q3 = qz[IX(i, j, k - 1)]; q4 = qz[IX(i - 1, j, k - 1)]; cnt += 2; }
        if (!(B[IX(i - 1, j, k)] != 0)) qxzl = (q1 + q2 + q3 + q4) / cnt;
    }
    if (i != nx - 1) {
        qxr = qx[IX(i, j, k)];
        q1 = qy[IX(i, j, k)]; q2 = qy[IX(i + 1, j, k)]; q3 = q4 = 0; cnt = 2;
        if (j != 0) { q3 = qy[IX(i + 1, j - 1, k)]; q4 = qy[IX(i, j - 1, k)]; cnt += 2; }
        if (!(B[IX(i + 1, j, k)] != 0)) qxyr = (q1 + q2 + q3 + q4) / cnt;
        q1 = qz[IX(i, j, k)]; q2 = qz[IX(i + 1, j, k)]; q3 = q4 = 0; cnt = 2;
        if (k != 0) { q3 = qz[IX(i + 1, j, k - 1)]; q4 = qz[IX(i, j, k - 1)]; cnt += 2; }
        if (!(B[IX(i + 1, j, k)] != 0)) qxzr = (q1 + q2 + q3 + q4) / cnt;
    }
    if (j != 0) {
        qyl = qy[IX(i, j - 1, k)];
        q1 = qx[IX(i, j, k)]; q2 = qx[IX(i, j - 1, k)]; q3 = q4 = 0; cnt = 2;
        if (i != 0) { q3 = qx[IX(i - 1, j - 1, k)]; q4 = qx[IX(i - 1, j, k)]; cnt += 2; }
        if (!(B[IX(i, j - 1, k)] != 0)) qyxl = (q1 + q2 + q3 + q4) / cnt;
        q1 = qz[IX(i, j - 1, k)]; q2 = qz[IX(i, j, k)]; q3 = q4 = 0; cnt = 2;
        if (k != 0) { q3 = qz[IX(i, j, k - 1)]; q4 = qz[IX(i, j - 1, k - 1)]; cnt += 2; }
        if (!(B[IX(i, j - 1, k)] != 0)) qyzl = (q1 + q2 + q3 + q4) / cnt;
    }
    if (j != ny - 1) {
        qyr = qy[IX(i, j, k)];
        q1 = qx[IX(i, j + 1, k)]; q2 = qx[IX(i, j, k)]; q3 = q4 = 0; cnt = 2;
        if (i != 0) { q3 = qx[IX(i - 1, j, k)]; q4 = qx[IX(i - 1, j + 1, k)]; cnt += 2; }
        if (!(B[IX(i, j + 1, k)] != 0)) qyxr = (q1 + q2 + q3 + q4) / cnt;
        q1 = qz[IX(i, j, k)]; q2 = qz[IX(i, j + 1, k)]; q3 = q4 = 0; cnt = 2;
        if (k != 0) { q3 = qz[IX(i, j + 1, k - 1)]; q4 = qz[IX(i, j, k - 1)]; cnt += 2; }
        if (!(B[IX(i, j + 1, k)] != 0)) qyzr = (q1 + q2 + q3 + q4) / cnt;
    }
    if (k != 0) {
        qzl = qz[IX(i, j, k - 1)];
        q1 = qx[IX(i, j, k)]; q2 = qx[IX(i, j, k - 1)]; q3 = q4 = 0; cnt = 2;
        if (i != 0) { q3 = qx[IX(i - 1, j, k - 1)]; q4 = qx[IX(i - 1, j, k)]; cnt += 2; }
        if (!(B[IX(i, j, k - 1)] != 0)) qzxl = (q1 + q2 + q3 + q4) / cnt;
        q1 = qy[IX(i, j, k)]; q2 = qy[IX(i, j, k - 1)]; q3 = q4 = 0; cnt = 2;
        if (j != 0) { q3 = qy[IX(i, j - 1, k - 1)]; q4 = qy[IX(i, j - 1, k)]; cnt += 2; }
        if (!(B[IX(i, j, k - 1)] != 0)) qzyl = (q1 + q2 + q3 + q4) / cnt;
    }
    if (k != nz - 1) {
        qzr = qz[IX(i, j, k)];
        q1 = qx[IX(i, j, k + 1)]; q2 = qx[IX(i, j, k)]; q3 = q4 = 0; cnt = 2;
        if (i != 0) { q3 = qx[IX(i - 1, j, k)]; q4 = qx[IX(i - 1, j, k + 1)]; cnt += 2; }
        if (!(B[IX(i, j, k + 1)] != 0)) qzxr = (q1 + q2 + q3 + q4) / cnt;
        q1 = qy[IX(i, j, k + 1)]; q2 = qy[IX(i, j, k)]; q3 = q4 = 0; cnt = 2;
        if (j != 0) { q3 = qy[IX(i, j - 1, k)]; q4 = qy[IX(i, j - 1, k + 1)]; cnt += 2; }
        if (!(B[IX(i, j, k + 1)] != 0)) qzyr = (q1 + q2 + q3 + q4) / cnt;
    }
    size_t c = IX(i, j, k);
    double ll = l_l[c], lt = l_t[c];
    Dout[0] = ll * fabs(qxl) + lt * (fabs(qxyl) + fabs(qxzl)); /* D_xl */
    Dout[1] = ll * fabs(qyl) + lt * (fabs(qyxl) + fabs(qyzl)); /* D_yl */
    Dout[2] = ll * fabs(qzl) + lt * (fabs(qzxl) + fabs(qzyl)); /* D_zl */
    Dout[3] = ll * fabs(qxr) + lt * (fabs(qxyr) + fabs(qxzr)); /* D_xr */
    Dout[4] = ll * fabs(qyr) + lt * (fabs(qyxr) + fabs(qyzr)); /* D_yr */
    Dout[5] = ll * fabs(qzr) + lt * (fabs(qzxr) + fabs(qzyr)); /* D_zr */
}

/* ------------------------------------------------------------------------ */
/* compute_C, tse.py:783-916                                                */
/* ------------------------------------------------------------------------ */
typedef struct {
    const double *Dfx, *Dfy, *Dfz, *phi, *rho, *qx, *qy, *qz, *BC, *WC, *RC, *e;
    const double *l_l, *l_t;   /* frozen lf_l, lf_t */
    int imblflo;               /* frozen config.C_IMBLFLO */
} og_cfields;

static double solve_c(const og_grid *G, const og_cfields *F, double *C,
                      const double *Cn, double dt_C, double omega, double SOR,
                      int i, int j, int k)
{
    const int nx = G->nx, ny = G->ny, nz = G->nz;
    const double *dx = G->dx, *dy = G->dy, *dz = G->dz;
    const double *phi = F->phi;
    const size_t c = IX(i, j, k);
    double A_ = 0, B_ = 0, C_ = 0, D_ = 0, E_ = 0, F_ = 0, G_ = 0, H_ = 0,
           I_ = 0, J_ = 0, K_ = 0, L_ = 0, M_ = 0, N_ = 0, O_ = 0, P_ = 0,
           Q_ = 0, R_ = 0, EC = 0;
    double Mnew = 0, Nnew = 0, Onew = 0, Pnew = 0, Qnew = 0, Rnew = 0;
    double Mold = 0, Nold = 0, Oold = 0, Pold = 0, Qold = 0, Rold = 0;
    double Dd[6] = {0, 0, 0, 0, 0, 0}; /* xl yl zl xr yr zr */
    double dd, dd2, ph;
    if (F->l_l[c] != 0 || F->l_t[c] != 0)
        dispersivity_(G, F->qx, F->qy, F->qz, F->l_l, F->l_t, F->BC, i, j, k, Dd);
    if (i != nx - 1) {
        size_t o = IX(i + 1, j, k);
        dd = dx[i];
        dd2 = (0.5 * (dx[i + 1] + dx[i])) * dd;
        ph = amean2(phi[o], phi[c], dx[i + 1], dx[i]);
        A_ = (harm2(F->Dfx[o], F->Dfx[c], dx[i + 1], dx[i]) * ph + Dd[3]) / dd2;
        N_ = min0(F->qx[c]) / dd;
        H_ = max0(F->qx[c]) / dd;
        Mnew = (A_ - N_) * C[o];
        Mold = (A_ - N_) * Cn[o];
    }
    if (i != 0) {
        size_t o = IX(i - 1, j, k);
        dd = dx[i];
        dd2 = (0.5 * (dx[i - 1] + dx[i])) * dd;
        ph = amean2(phi[o], phi[c], dx[i - 1], dx[i]);
        B_ = (harm2(F->Dfx[o], F->Dfx[c], dx[i - 1], dx[i]) * ph + Dd[0]) / dd2;
        M_ = max0(F->qx[o]) / dd;
        G_ = min0(F->qx[o]) / dd;
        Nnew = (B_ + M_) * C[o];
        Nold = (B_ + M_) * Cn[o];
    }
    if (j != ny - 1) {
        size_t o = IX(i, j + 1, k);
        dd = dy[j];
        dd2 = (0.5 * (dy[j + 1] + dy[j])) * dd;
        ph = amean2(phi[o], phi[c], dy[j + 1], dy[j]);
        C_ = (harm2(F->Dfy[o], F->Dfy[c], dy[j + 1], dy[j]) * ph + Dd[4]) / dd2;
        P_ = min0(F->qy[c]) / dd;
        J_ = max0(F->qy[c]) / dd;
        Onew = (C_ - P_) * C[o];
        Oold = (C_ - P_) * Cn[o];
    }
    if (j != 0) {
        size_t o = IX(i, j - 1, k);
        dd = dy[j];
        dd2 = (0.5 * (dy[j - 1] + dy[j])) * dd;
        ph = amean2(phi[o], phi[c], dy[j - 1], dy[j]);
        D_ = (harm2(F->Dfy[o], F->Dfy[c], dy[j - 1], dy[j]) * ph + Dd[1]) / dd2;
        O_ = max0(F->qy[o]) / dd;
        I_ = min0(F->qy[o]) / dd;
        Pnew = (D_ + O_) * C[o];
        Pold = (D_ + O_) * Cn[o];
    }
    if (k != nz - 1) {
        size_t o = IX(i, j, k + 1);
        dd = dz[k];
        dd2 = (0.5 * (dz[k + 1] + dz[k])) * dd;
        ph = amean2(phi[o], phi[c], dz[k + 1], dz[k]);
        E_ = (harm2(F->Dfz[o], F->Dfz[c], dz[k + 1], dz[k]) * ph + Dd[5]) / dd2;
        R_ = min0(F->qz[c]) / dd;
        L_ = max0(F->qz[c]) / dd;
        Qnew = (E_ - R_) * C[o];
        Qold = (E_ - R_) * Cn[o];
    }
    if (k != 0) {
        size_t o = IX(i, j, k - 1);
        dd = dz[k];
        dd2 = (0.5 * (dz[k - 1] + dz[k])) * dd;
        ph = amean2(phi[o], phi[c], dz[k - 1], dz[k]);
        F_ = (harm2(F->Dfz[o], F->Dfz[c], dz[k - 1], dz[k]) * ph + Dd[2]) / dd2;
        Q_ = max0(F->qz[o]) / dd;
        K_ = min0(F->qz[o]) / dd;
        Rnew = (F_ + Q_) * C[o];
        Rold = (F_ + Q_) * Cn[o];
    }
    double R = F->RC[c] * phi[c] / dt_C;
    double M = -A_ - B_ - C_ - D_ - E_ - F_ + G_ - H_ + I_ - J_ + K_ - L_;
    if (F->imblflo)
        EC = Cn[c] / F->rho[c] * F->e[c];
    return ((1 - SOR) * C[c] + SOR * (omega * (Mnew + Nnew + Onew + Pnew + Qnew + Rnew)
                                      + (1 - omega) * (Cn[c] * M + Mold + Nold + Oold + Pold + Qold + Rold)
                                      + R * Cn[c] + F->WC[c] - EC)
                                   / (R - omega * M));
}

/* Shared transport driver loop (tse.py:877-914 for C, 1045-1079 for T).
 * out[] as for og_compute_P (out[0]=t, out[1]=dt, out[2]=converged,
 * out[3]=num_it, out[4]=diff, out[5]=halvings). */
typedef double (*solve_fn)(const og_grid *, const void *, double *, const double *,
                           double, double, double, int, int, int);

static int transport_loop(const og_grid *G, const void *F, const double *B,
                          solve_fn fn, double *X, double dt, double omega,
                          double SOR, int max_it, double inc_it, double max_dt,
                          double min_dt, double conv, double *out)
{
    const int nx = G->nx, ny = G->ny, nz = G->nz;
    const size_t n = (size_t)nx * ny * nz;
    double *Xn = (double *)malloc(n * sizeof(double));
    double *Xold = (double *)malloc(n * sizeof(double));
    if (!Xn || !Xold) {
        free(Xn);
        free(Xold);
        return -1;
    }
    double t = 0, diff = 1e100;
    int converged = 0, num_it = 0, num_sub_it = 0, halvings = 0;
    memcpy(Xn, X, n * sizeof(double));
    while (!converged) {
        num_it += 1;
        num_sub_it += 1;
        memcpy(Xold, X, n * sizeof(double));
        for (int colour = 0; colour < 2; ++colour) {
#pragma omp parallel for schedule(static)
            for (int i = 0; i < nx; ++i)
                for (int j = 0; j < ny; ++j)
                    for (int k = ((i + j + colour) & 1); k < nz; k += 2) {
                        size_t c = IX(i, j, k);
                        if (!(B[c] != 0))
                            X[c] = fn(G, F, X, Xn, dt, omega, SOR, i, j, k);
                    }
        }
        diff = og_l2_norm(X, Xold, n);
        if (diff < conv || omega == 0) {
            t += dt;
            if (num_sub_it < max_it / 2.0)
                dt = pymin(dt * inc_it, max_dt);
            converged = 1;
        } else {
            converged = 0;
            if (num_sub_it >= max_it) {
                dt = dt / 2;
                num_sub_it = 0;
                halvings += 1;
                memcpy(X, Xn, n * sizeof(double));
            }
            if (dt <= min_dt)
                break;
        }
    }
    free(Xn);
    free(Xold);
    out[0] = t;
    out[1] = dt;
    out[2] = converged;
    out[3] = num_it;
    out[4] = diff;
    out[5] = halvings;
    return 0;
}

static double solve_c_thunk(const og_grid *G, const void *F, double *X,
                            const double *Xn, double dt, double omega,
                            double SOR, int i, int j, int k)
{
    return solve_c(G, (const og_cfields *)F, X, Xn, dt, omega, SOR, i, j, k);
}

int og_compute_C(const og_grid *G, const og_cfields *F, double *C, double dt_C,
                 double omega, double SOR, int max_it, double inc_it,
                 double max_dt, double min_dt, double C_conv, double *out)
{
    return transport_loop(G, F, F->BC, solve_c_thunk, C, dt_C, omega, SOR,
                          max_it, inc_it, max_dt, min_dt, C_conv, out);
}

/* ------------------------------------------------------------------------ */
/* compute_T, tse.py:919-1081                                               */
/* ------------------------------------------------------------------------ */
typedef struct {
    const double *l_f, *cp_f, *rho, *phi, *qx, *qy, *qz, *BT, *WT, *e;
    const double *l_r, *rho_r, *cp_r;  /* frozen */
    const double *l_l, *l_t;           /* frozen lt_l, lt_t */
    int imblflo;                       /* frozen config.T_IMBLFLO */
} og_tfields;

static double solve_t(const og_grid *G, const og_tfields *F, double *T,
                      const double *Tn, double dt_T, double omega, double SOR,
                      int i, int j, int k)
{
    const int nx = G->nx, ny = G->ny, nz = G->nz;
    const double *dx = G->dx, *dy = G->dy, *dz = G->dz;
    const double *phi = F->phi;
    const size_t c = IX(i, j, k);
    double A_ = 0, B_ = 0, C_ = 0, D_ = 0, E_ = 0, F_ = 0, G_ = 0, H_ = 0,
           I_ = 0, J_ = 0, K_ = 0, L_ = 0, S_ = 0, M_ = 0, N_ = 0, O_ = 0,
           P_ = 0, Q_ = 0, R_ = 0, ET = 0;
    double Mnew = 0, Nnew = 0, Onew = 0, Pnew = 0, Qnew = 0, Rnew = 0;
    double Mold = 0, Nold = 0, Oold = 0, Pold = 0, Qold = 0, Rold = 0;
    double Dd[6] = {0, 0, 0, 0, 0, 0};
    double dd, dd2, por, lf, lr, cpf, rhocpf;
    (void)S_;
    if (F->l_l[c] != 0 || F->l_t[c] != 0)
        dispersivity_(G, F->qx, F->qy, F->qz, F->l_l, F->l_t, F->BT, i, j, k, Dd);
#define TFACE(o, d1, d2)                                                   \
    por = amean2(phi[c], phi[o], d1, d2);                                  \
    lf = harm2(F->l_f[c], F->l_f[o], d1, d2);                              \
    lr = harm2(F->l_r[c], F->l_r[o], d1, d2);                              \
    cpf = harm2(F->cp_f[c], F->cp_f[o], d1, d2);                           \
    rhocpf = harm2(F->rho[c], F->rho[o], d1, d2) * cpf;
    if (i != nx - 1) {
        size_t o = IX(i + 1, j, k);
        dd = dx[i];
        dd2 = (0.5 * (dx[i + 1] + dx[i])) * dd;
        TFACE(o, dx[i], dx[i + 1]);
        A_ = ((1 - por) * lr + por * lf + Dd[3] * rhocpf) / dd2;
        S_ = rhocpf / dd;
        N_ = min0(F->qx[c]) * S_;
        H_ = max0(F->qx[c]) * S_;
        Mnew = (A_ - N_) * T[o];
        Mold = (A_ - N_) * Tn[o];
    }
    if (i != 0) {
        size_t o = IX(i - 1, j, k);
        dd = dx[i];
        dd2 = (0.5 * (dx[i - 1] + dx[i])) * dd;
        TFACE(o, dx[i], dx[i - 1]);
        B_ = ((1 - por) * lr + por * lf + Dd[0] * rhocpf) / dd2;
        S_ = rhocpf / dd;
        M_ = max0(F->qx[o]) * S_;
        G_ = min0(F->qx[o]) * S_;
        Nnew = (B_ + M_) * T[o];
        Nold = (B_ + M_) * Tn[o];
    }
    if (j != ny - 1) {
        size_t o = IX(i, j + 1, k);
        dd = dy[j];
        dd2 = (0.5 * (dy[j + 1] + dy[j])) * dd;
        TFACE(o, dy[j], dy[j + 1]);
        C_ = ((1 - por) * lr + por * lf + Dd[4] * rhocpf) / dd2;
        S_ = rhocpf / dd;
        P_ = min0(F->qy[c]) * S_;
        J_ = max0(F->qy[c]) * S_;
        Onew = (C_ - P_) * T[o];
        Oold = (C_ - P_) * Tn[o];
    }
    if (j != 0) {
        size_t o = IX(i, j - 1, k);
        dd = dy[j];
        dd2 = (0.5 * (dy[j - 1] + dy[j])) * dd;
        TFACE(o, dy[j], dy[j - 1]);
        D_ = ((1 - por) * lr + por * lf + Dd[1] * rhocpf) / dd2;
        S_ = rhocpf / dd;
        O_ = max0(F->qy[o]) * S_;
        I_ = min0(F->qy[o]) * S_;
        Pnew = (D_ + O_) * T[o];
        Pold = (D_ + O_) * Tn[o];
    }
    if (k != nz - 1) {
        size_t o = IX(i, j, k + 1);
        dd = dz[k];
        dd2 = (0.5 * (dz[k + 1] + dz[k])) * dd;
        TFACE(o, dz[k], dz[k + 1]);
        E_ = ((1 - por) * lr + por * lf + Dd[5] * rhocpf) / dd2;
        S_ = rhocpf / dd;
        R_ = min0(F->qz[c]) * S_;
        L_ = max0(F->qz[c]) * S_;
        Qnew = (E_ - R_) * T[o];
        Qold = (E_ - R_) * Tn[o];
    }
    if (k != 0) {
        size_t o = IX(i, j, k - 1);
        dd = dz[k];
        dd2 = (0.5 * (dz[k - 1] + dz[k])) * dd;
        TFACE(o, dz[k], dz[k - 1]);
        F_ = ((1 - por) * lr + por * lf + Dd[2] * rhocpf) / dd2;
        S_ = rhocpf / dd;
        Q_ = max0(F->qz[o]) * S_;
        K_ = min0(F->qz[o]) * S_;
        Rnew = (F_ + Q_) * T[o];
        Rold = (F_ + Q_) * Tn[o];
    }
#undef TFACE
    double por_ = phi[c];
    double R = (por_ * F->rho[c] * F->cp_f[c] + (1 - por_) * F->rho_r[c] * F->cp_r[c]) / dt_T;
    double M = -A_ - B_ - C_ - D_ - E_ - F_ + G_ - H_ + I_ - J_ + K_ - L_;
    if (F->imblflo)
        ET = F->cp_f[c] * Tn[c] * F->e[c];
    return ((1 - SOR) * T[c] + SOR * (omega * (Mnew + Nnew + Onew + Pnew + Qnew + Rnew)
                                      + (1 - omega) * (Tn[c] * M + Mold + Nold + Oold + Pold + Qold + Rold)
                                      + R * Tn[c] + F->WT[c] - ET)
                                   / (R - omega * M));
}

static double solve_t_thunk(const og_grid *G, const void *F, double *X,
                            const double *Xn, double dt, double omega,
                            double SOR, int i, int j, int k)
{
    return solve_t(G, (const og_tfields *)F, X, Xn, dt, omega, SOR, i, j, k);
}

int og_compute_T(const og_grid *G, const og_tfields *F, double *T, double dt_T,
                 double omega, double SOR, int max_it, double inc_it,
                 double max_dt, double min_dt, double T_conv, double *out)
{
    return transport_loop(G, F, F->BT, solve_t_thunk, T, dt_T, omega, SOR,
                          max_it, inc_it, max_dt, min_dt, T_conv, out);
}

/* ------------------------------------------------------------------------ */
/* smolarkiewicz, tse.py:1083-1116                                          */
/* ------------------------------------------------------------------------ */
void og_smolarkiewicz(const og_grid *G, const double *C, const double *qx,
                      const double *qy, const double *qz, double *vx, double *vy,
                      double *vz, double dt, double eps, double Sc)
{
    const int nx = G->nx, ny = G->ny, nz = G->nz;
    const double *dx = G->dx, *dy = G->dy, *dz = G->dz;
#pragma omp parallel for schedule(static)
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny; ++j)
            for (int k = 0; k < nz; ++k) {
                size_t c = IX(i, j, k);
                if (C[c] > 0) {
                    double dd;
                    if (i < nx - 1) {
                        size_t o = IX(i + 1, j, k);
                        dd = 0.5 * (dx[i + 1] + dx[i]);
                        vx[c] = (Sc * (fabs(qx[c]) * dd - dt * (qx[c] * qx[c])) * (C[o] - C[c])
                                 / ((C[c] + C[o] + eps) * dd));
                    }
                    if (j < ny - 1) {
                        size_t o = IX(i, j + 1, k);
                        dd = 0.5 * (dy[j + 1] + dy[j]);
                        vy[c] = (Sc * (fabs(qy[c]) * dd - dt * (qy[c] * qy[c])) * (C[o] - C[c])
                                 / ((C[c] + C[o] + eps) * dd));
                    }
                    if (k < nz - 1) {
                        size_t o = IX(i, j, k + 1);
                        dd = 0.5 * (dz[k + 1] + dz[k]);
                        vz[c] = (Sc * (fabs(qz[c]) * dd - dt * (qz[c] * qz[c])) * (C[o] - C[c])
                                 / ((C[c] + C[o] + eps) * dd));
                    }
                } else {
                    vx[c] = 0;
                    vy[c] = 0;
                    vz[c] = 0;
                }
            }
}

/* ------------------------------------------------------------------------ */
/* explicit_C, tse.py:385-396 (D_max = per-cell max over species, computed   */
/* by the caller).                                                          */
/* ------------------------------------------------------------------------ */
double og_explicit_C(const og_grid *G, const double *Dmax, const double *phi)
{
    const int nx = G->nx, ny = G->ny, nz = G->nz;
    const double *dx = G->dx, *dy = G->dy, *dz = G->dz;
    double dt_NeC = 1e100;
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny; ++j)
            for (int k = 0; k < nz; ++k) {
                size_t c = IX(i, j, k);
                double v = 0.45 * Dmax[c] / phi[c]
                           / (1 / (dx[i] * dx[i]) + 1 / (dy[j] * dy[j]) + 1 / (dz[k] * dz[k]));
                dt_NeC = pymin(dt_NeC, v);
            }
    return dt_NeC;
}
