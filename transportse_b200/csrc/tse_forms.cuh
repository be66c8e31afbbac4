// Per-cell solver forms of the red-black solves: the coefficient arrays an
// assembly pass stores per colour, and the update of one cell in the
// reference's operation order (compute_P tse.py:658-697, compute_C
// tse.py:795-875, compute_T tse.py:930-1043).  `sum` is the numerator of the
// update, `den` its denominator and `k(q)` the weight of neighbour q in
// `sum`, which the defect-correction form uses for its correction equation.
#pragma once

#include "tse_common.cuh"

namespace tse {

// offset of neighbour q (x+, x-, y+, y-, z+, z-) of a compact cell in the
// other colour's array; zo = 1 for cells with odd k
__device__ __forceinline__ long long nb_offset(int q, long long SX, long long H, long long zo) {
    return q == 0 ? SX : q == 1 ? -SX : q == 2 ? H : q == 3 ? -H : q == 4 ? zo : zo - 1;
}

enum PArr {
    PA_A = 0, PA_C, PA_E, PA_G, PA_I, PA_K,   // transmissibilities x+ x- y+ y- z+ z-
    PA_AB, PA_CD, PA_IJ, PA_KL,               // buoyancy products
    PA_RPN, PA_WP, PA_DEN,                    // R*Pn, WP, R+M
    PA_S, PA_M, PA_PN,                        // storage numerator, M, Pn (reset)
    PA_P,                                     // solution
    PA_COUNT
};

struct PressureForm {
    double* arr[2];   // per colour: PA_COUNT arrays of Ncal doubles
    long long Ncal, SX;
    int H;
    int xgrav, zgrav;
    double SOR;

    __device__ __forceinline__ const double* a(int col, int k) const { return arr[col] + (long long)k * Ncal; }

    // numerator of the update (tse.py:691-694), in the reference's order;
    // a(k) is coefficient array k of the cell, x(q) its neighbour q (x+, x-,
    // y+, y-, z+, z-), read only where the flag says the neighbour exists
    template <class A, class X>
    __device__ __forceinline__ double sum_with(A a, X x, uint8_t f) const {
        double s = (f & F_XP) ? a(PA_A) * x(0) : 0.0;
        s = s + (xgrav ? a(PA_AB) : 0.0);
        s = s + ((f & F_XM) ? a(PA_C) * x(1) : 0.0);
        s = s - (xgrav ? a(PA_CD) : 0.0);
        s = s + ((f & F_YP) ? a(PA_E) * x(2) : 0.0);
        s = s + ((f & F_YM) ? a(PA_G) * x(3) : 0.0);
        s = s + ((f & F_ZP) ? a(PA_I) * x(4) : 0.0);
        s = s + (zgrav ? a(PA_IJ) : 0.0);
        s = s + ((f & F_ZM) ? a(PA_K) * x(5) : 0.0);
        s = s - (zgrav ? a(PA_KL) : 0.0);
        s = s + a(PA_RPN);
        s = s + a(PA_WP);
        return s;
    }
    __device__ __forceinline__ double sum(int col, long long m, uint8_t f, const double* Xo) const {
        const double* b = arr[col];
        const long long N = Ncal, sx = SX, h = H, zo = (long long)(f >> 7);
        return sum_with([&](int k) { return b[k * N + m]; },
                        [&](int q) { return __ldcg(Xo + m + nb_offset(q, sx, h, zo)); }, f);
    }
    // the arrays sum_with reads, in a fixed order (host side)
    int staged_arrays(int* idx) const {
        int n = 0;
        const int base[6] = {PA_A, PA_C, PA_E, PA_G, PA_I, PA_K};
        for (int q = 0; q < 6; ++q) idx[n++] = base[q];
        if (xgrav) { idx[n++] = PA_AB; idx[n++] = PA_CD; }
        if (zgrav) { idx[n++] = PA_IJ; idx[n++] = PA_KL; }
        idx[n++] = PA_RPN;
        idx[n++] = PA_WP;
        idx[n++] = PA_DEN;
        return n;
    }
    static constexpr int kSolution = PA_P;
    static constexpr int kArrays = PA_COUNT;
    __device__ __forceinline__ double den(int col, long long m) const {
        return arr[col][PA_DEN * Ncal + m];
    }
    // coefficient of neighbour q (x+, x-, y+, y-, z+, z-) in sum()
    __device__ __forceinline__ double k(int col, long long m, int q) const {
        return arr[col][(PA_A + q) * Ncal + m];
    }
    __device__ __forceinline__ double update(int col, long long m, uint8_t f, double xold,
                                             const double* Xo) const {
        const double s = sum(col, m, f, Xo);
        return (1.0 - SOR) * xold + (SOR * s) / den(col, m);
    }
    template <class A, class X>
    __device__ __forceinline__ double update_with(A a, X x, uint8_t f, double xold) const {
        const double s = sum_with(a, x, f);
        return (1.0 - SOR) * xold + (SOR * s) / a(PA_DEN);
    }

    // dt halving: P = Pn (tse.py:738) and the dt-dependent R terms
    __device__ __forceinline__ void reassemble(int col, long long m, double dt) const {
        double* b = arr[col];
        const double pn = b[PA_PN * Ncal + m];
        const double R = b[PA_S * Ncal + m] / dt;
        b[PA_RPN * Ncal + m] = R * pn;
        b[PA_DEN * Ncal + m] = R + b[PA_M * Ncal + m];
        b[PA_P * Ncal + m] = pn;
    }
};

enum TArr {
    TA_A = 0, TA_B, TA_C, TA_D, TA_E, TA_F,   // neighbour coefficients x+ x- y+ y- z+ z-
    TA_Y,                                     // (1-omega) * (Xn M + old neighbour sum)
    TA_RXN, TA_W, TA_EX, TA_DEN,              // R Xn, source, IMBLFLO term, R - omega M
    TA_RNUM, TA_M, TA_XN,                     // R numerator, M, Xn (reset)
    TA_X,                                     // solution
    TA_COUNT
};

struct TransportForm {
    double* arr[2];
    long long Ncal, SX;
    int H;
    int useY, useEX;
    double omega, SOR;

    // numerator of the update (tse.py:870-874), in the reference's order;
    // a(k) and x(q) as in PressureForm::sum_with
    template <class A, class X>
    __device__ __forceinline__ double sum_with(A a, X x, uint8_t f) const {
        double s = (f & F_XP) ? a(TA_A) * x(0) : 0.0;
        s = s + ((f & F_XM) ? a(TA_B) * x(1) : 0.0);
        s = s + ((f & F_YP) ? a(TA_C) * x(2) : 0.0);
        s = s + ((f & F_YM) ? a(TA_D) * x(3) : 0.0);
        s = s + ((f & F_ZP) ? a(TA_E) * x(4) : 0.0);
        s = s + ((f & F_ZM) ? a(TA_F) * x(5) : 0.0);
        double num = omega * s;
        if (useY) num = num + a(TA_Y);
        num = num + a(TA_RXN);
        num = num + a(TA_W);
        num = num - (useEX ? a(TA_EX) : 0.0);
        return num;
    }
    __device__ __forceinline__ double sum(int col, long long m, uint8_t f, const double* Xo) const {
        const double* b = arr[col];
        const long long N = Ncal, sx = SX, h = H, zo = (long long)(f >> 7);
        return sum_with([&](int k) { return b[k * N + m]; },
                        [&](int q) { return __ldcg(Xo + m + nb_offset(q, sx, h, zo)); }, f);
    }
    int staged_arrays(int* idx) const {
        int n = 0;
        for (int q = 0; q < 6; ++q) idx[n++] = TA_A + q;
        if (useY) idx[n++] = TA_Y;
        idx[n++] = TA_RXN;
        idx[n++] = TA_W;
        if (useEX) idx[n++] = TA_EX;
        idx[n++] = TA_DEN;
        return n;
    }
    static constexpr int kSolution = TA_X;
    static constexpr int kArrays = TA_COUNT;
    __device__ __forceinline__ double den(int col, long long m) const {
        return arr[col][TA_DEN * Ncal + m];
    }
    // coefficient of neighbour q in sum(): omega * (upwinded coefficient)
    __device__ __forceinline__ double k(int col, long long m, int q) const {
        return omega * arr[col][(TA_A + q) * Ncal + m];
    }
    __device__ __forceinline__ double update(int col, long long m, uint8_t f, double xold,
                                             const double* Xo) const {
        const double num = sum(col, m, f, Xo);
        return (1.0 - SOR) * xold + (SOR * num) / den(col, m);
    }
    template <class A, class X>
    __device__ __forceinline__ double update_with(A a, X x, uint8_t f, double xold) const {
        const double num = sum_with(a, x, f);
        return (1.0 - SOR) * xold + (SOR * num) / a(TA_DEN);
    }

    // dt halving: X = Xn (tse.py:911, 1077) and the dt-dependent R terms
    __device__ __forceinline__ void reassemble(int col, long long m, double dt) const {
        double* b = arr[col];
        const double xn = b[TA_XN * Ncal + m];
        const double R = b[TA_RNUM * Ncal + m] / dt;
        b[TA_RXN * Ncal + m] = R * xn;
        b[TA_DEN * Ncal + m] = R - omega * b[TA_M * Ncal + m];
        b[TA_X * Ncal + m] = xn;
    }
};

struct GridBarrier;

// Workspace carved for one solve, with the assembly already launched.
template <class Form>
struct SolveSetup {
    Layout L;
    long long Ncal;
    GridBarrier* bar;
    double* partials;
    uint8_t* mask[2];
    Form F;
    char* tail;          // workspace bytes after the exact form's arrays
    size_t tail_bytes;
    double* faces = nullptr;   // transport: the face pass's values
};
using PressureSetup = SolveSetup<PressureForm>;
using TransportSetup = SolveSetup<TransportForm>;

size_t pressure_ws_bytes(const Layout& L, long long* Ncal_out);
size_t transport_ws_bytes(const Layout& L, long long* Ncal_out);
int setup_pressure(const TseGrid* grid, const TsePressureArgs* args, void* d_ws, size_t ws_bytes,
                   cudaStream_t stream, PressureSetup& S);
int setup_species(const TseGrid* grid, const TseSpeciesArgs* args, void* d_ws, size_t ws_bytes,
                  cudaStream_t stream, TransportSetup& S);
int setup_heat(const TseGrid* grid, const TseHeatArgs* args, void* d_ws, size_t ws_bytes,
               cudaStream_t stream, TransportSetup& S);
int launch_unpack(double* out, const double* X0, const double* X1, const Layout& L,
                  cudaStream_t stream);

}  // namespace tse
