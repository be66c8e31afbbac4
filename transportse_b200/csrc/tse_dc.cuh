// Shared pieces of the mixed-precision (FP32 sweeps + FP64 defect
// correction) solves: the solver state, the control record, the per-cell
// FP32 relaxation and the workspace layout.  Used by the whole-GPU form
// (tse_dc.cu) and the batched one-block-per-model form (tse_batch.cu).
#pragma once

#include "tse_forms.cuh"
#include "tse_rbsolve.cuh"

namespace tse {

constexpr double kRefresh = 1e-4;

// events that end a run of correction sweeps
enum DcEvent { EV_NONE = 0, EV_CONVERGED, EV_CYCLE_END, EV_REFRESH, EV_HALVE, EV_STOP,
               EV_STOP_HALVED, EV_ERROR };

// Solver state carried across the kernels of one solve (device memory).
struct DcState {
    double t, dt, diff, x2;
    int num_it, num_sub_it, halvings, converged;
    int event, nev, cycles, checkno;
    int ev_it[8];
    double ev_dt[8];
    double ev_diff[8];
};

struct DcCtl {
    Layout L;
    long long Ncal;
    double inc_it, max_dt, min_dt, conv;
    int max_it;
    int pressure_schedule;
    int stop_on_first;
    int cycle;           // inner iterations between residual updates
    float sor;
    double* X[2];        // FP64 iterate per colour
    const uint8_t* mask[2];
    float* K[2];         // per colour: Ncal 24-byte coefficient records, then Ncal r'
    float* D[2];         // per colour: correction, valid on [-G, Nc + G); the
                         // margins stay 0 so neighbour loads need no guard
    double* partials;    // sweep kernel: 4 per block; residual kernel: 1 per block
    GridBarrier* bar;
    DcState* st;
    long long chunk;     // chunked sweep: compact cells per block
    int R;               // chunked sweep: PhaseSync neighbour radius
    unsigned* prog;      // chunked sweep: PhaseSync counters
};

// K'_q = k_q / Den of one cell (6 FP32 values, one 24-byte record)
template <class Form>
__device__ __forceinline__ void scale_cell(const Form& F, const DcCtl& c, int col, long long m) {
    float2* rec = reinterpret_cast<float2*>(c.K[col] + 6 * m);
    if (c.mask[col][m] & F_ACTIVE) {
        const double den = F.den(col, m);
#pragma unroll
        for (int q = 0; q < 3; ++q)
            rec[q] = make_float2((float)(F.k(col, m, 2 * q) / den), (float)(F.k(col, m, 2 * q + 1) / den));
    } else {
#pragma unroll
        for (int q = 0; q < 3; ++q) rec[q] = make_float2(0.0f, 0.0f);
    }
}

// The coefficients of a cell are one 24-byte record (three 8-byte loads
// from one address); the z-neighbours dq[m-1], dq[m+1] are the dq[m] values
// the adjacent lanes load (consecutive lanes hold consecutive m), fetched
// from memory only at a warp's edge or the end of the range.  All lanes of a
// warp call relax() together.
struct Cell {
    float2 k01, k23, k45;
    float r, old, xp, xm, yp, ym, z1;
    bool odd;
};

__device__ __forceinline__ void load_cell(Cell& a, const float* __restrict__ Kc, const float* dw,
                                          const float* dq, const uint8_t* __restrict__ msk,
                                          long long m, long long N, long long SX, int H) {
    const float2* rec = reinterpret_cast<const float2*>(Kc + 6 * m);
    a.k01 = rec[0];
    a.k23 = rec[1];
    a.k45 = rec[2];
    a.r = Kc[6 * N + m];
    a.odd = (msk[m] & F_KODD) != 0;
    a.old = dw[m];
    a.xp = __ldcg(dq + m + SX);
    a.xm = __ldcg(dq + m - SX);
    a.yp = __ldcg(dq + m + H);
    a.ym = __ldcg(dq + m - H);
    a.z1 = __ldcg(dq + m);
}

__device__ __forceinline__ float relax(const Cell& a, const float* dq, long long m, long long end,
                                       float sor) {
    const int lane = threadIdx.x & 31;
    float z0 = __shfl_up_sync(0xffffffffu, a.z1, 1);
    float z2 = __shfl_down_sync(0xffffffffu, a.z1, 1);
    if (lane == 0) z0 = __ldcg(dq + m - 1);
    if (lane == 31 || m + 1 >= end) z2 = __ldcg(dq + m + 1);
    float acc = a.r;
    acc = fmaf(a.k01.x, a.xp, acc);
    acc = fmaf(a.k01.y, a.xm, acc);
    acc = fmaf(a.k23.x, a.yp, acc);
    acc = fmaf(a.k23.y, a.ym, acc);
    acc = fmaf(a.k45.x, a.odd ? z2 : a.z1, acc);
    acc = fmaf(a.k45.y, a.odd ? a.z1 : z0, acc);
    return fmaf(sor, acc - a.old, a.old);
}

// FP32 arrays: per colour 7 * Ncal floats (records + r'), then the
// correction with margins of G >= SX + 1, then the state record and the
// PhaseSync counters.  The margins also hold the neighbour windows that the
// staged sweep copies for a chunk of up to kDcMaxChunk cells at either end
// (window starts rounded down to 16 bytes, lengths up to 8 floats longer).
constexpr int kDcMaxChunk = 1024;
__host__ __device__ inline long long dc_margin(const Layout& L) {
    return ((L.SX + kDcMaxChunk + 16 + 63) / 64) * 64;
}
__host__ __device__ inline long long dc_delta_len(const Layout& L, long long Ncal) {
    return Ncal + 2 * dc_margin(L);
}
size_t dc_extra_bytes(const Layout& L);

// Fill a control record for a solve whose exact-form setup is S (the FP32
// arrays live in S.tail); returns the first byte after the FP32 arrays.
template <class Form>
inline void dc_carve(SolveSetup<Form>& S, DcCtl& c, int x_index) {
    c.L = S.L;
    c.Ncal = S.Ncal;
    c.X[0] = S.F.arr[0] + (size_t)x_index * S.Ncal;
    c.X[1] = S.F.arr[1] + (size_t)x_index * S.Ncal;
    c.mask[0] = S.mask[0];
    c.mask[1] = S.mask[1];
    float* base = (float*)(((uintptr_t)S.tail + 255) & ~(uintptr_t)255);
    const long long G = dc_margin(S.L), dlen = dc_delta_len(S.L, S.Ncal);
    c.K[0] = base;
    c.K[1] = base + (size_t)7 * S.Ncal;
    float* dbase = base + (size_t)14 * S.Ncal;
    c.D[0] = dbase + G;
    c.D[1] = dbase + dlen + G;
    c.st = (DcState*)(dbase + 2 * dlen);
    c.prog = (unsigned*)((char*)c.st + align256(sizeof(DcState)));
    c.partials = S.partials;
    c.bar = S.bar;
}

}  // namespace tse
