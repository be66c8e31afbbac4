// Shared pieces of the mixed-precision (FP32 sweeps + FP64 defect
// correction) solves: the solver state, the control record, the per-cell
// FP32 relaxation and the workspace layout.  Used by the whole-GPU form
// (tse_dc.cu) and the batched one-block-per-model form (tse_batch.cu).
#pragma once

#include "tse_forms.cuh"
#include "tse_rbsolve.cuh"
#include "tse_tma.cuh"

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
    unsigned* prog;      // staged sweep: its barrier counter
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

// FP64 residual of the correction equation: fixed grid of the residual
// kernel (deterministic sums); one block's share of a model's cells
constexpr int kResBlocks = 2048;

__host__ __device__ inline int res_blocks(long long Nc) {
    const long long rb = (2 * Nc + kBlock - 1) / kBlock;
    return (int)(rb < kResBlocks ? rb : kResBlocks);
}

// r' = (sum(x) - Den x) / Den, d = 0 for the cells t = b*kBlock + tid +
// s*nblocks*kBlock of both colours (t < 2 Nc) as residual block b of nblocks;
// returns this thread's sum of x^2 (all cells, active or not)
template <class Form>
__device__ __forceinline__ double residual_block_cells(const Form& F, const DcCtl& c, long long b,
                                                       long long nblocks) {
    const long long Nc = c.L.Nc;
    double o2 = 0.0;
    for (long long t = b * kBlock + threadIdx.x; t < 2 * Nc; t += nblocks * kBlock) {
        const int col = t >= Nc;
        const long long m = t - col * Nc;
        const uint8_t f = c.mask[col][m];
        const double x = c.X[col][m];
        o2 = o2 + x * x;
        float rp = 0.0f;
        if (f & F_ACTIVE) {
            const double den = F.den(col, m);
            const double r = F.sum(col, m, f, c.X[1 - col]) - den * x;
            rp = (float)(r / den);
        }
        c.K[col][6 * c.Ncal + m] = rp;
        c.D[col][m] = 0.0f;
    }
    return o2;
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
// staged sweep's barrier counter.  The margins also hold the neighbour windows that the
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

// one model's solve steps (tse_dc.cu), for drivers that interleave models
template <class Form>
int dc_begin(const Form& F, const DcCtl& c, double dt, cudaStream_t stream);
template <class Form>
int dc_residual(const Form& F, const DcCtl& c, cudaStream_t stream);
template <class Form>
int dc_halve(const Form& F, const DcCtl& c, cudaStream_t stream);
int dc_apply(const DcCtl& c, cudaStream_t stream);
int dc_finish(const DcCtl& c, TseSolveStatus* d_status, double* X_out, cudaStream_t stream);
// the start of a solve whose setup was fused (setup_*_dc): state record,
// zeroed corrections, the x^2 total of the setup's nparts partials
int dc_begin_fused(const DcCtl& c, double dt, int nparts, cudaStream_t stream);

// The mixed-precision form's first correction cycle, written by the
// assembly pass of a solve: per colour the FP32 record K'_q = k_q / Den and
// r' = (sum(x) - Den x) / Den of the initial iterate (sum() in the form's
// order), and per block the sum of x^2.  No bit-exactness is claimed for
// this form: 1/Den is formed once.
struct DcFuse {
    float* K[2];
    long long Ncal;
    double* partials;
    int per_thread;   // cells a thread assembles (blocks of kBlock consecutive cells)
};

// Assembly grid of a fused setup: a function of the grid alone (at most
// kMaxBlocks blocks), so the x^2 sums are grouped the same way on every device.
inline void dc_fuse_grid(const Layout& L, long long& per, long long& nb) {
    const long long total = (long long)L.nx * L.ny * L.nzp;
    const long long groups = (total + kBlock - 1) / kBlock;
    per = (groups + kMaxBlocks - 1) / kMaxBlocks;
    nb = (groups + per - 1) / per;
}

// Pressure setup for the mixed-precision form (tse_pressure.cu): the exact
// form's arrays plus the first cycle's records, r' and *nparts x^2 partials.
int setup_pressure_dc(const TseGrid* grid, const TsePressureArgs* args, void* d_ws, size_t ws_bytes,
                      cudaStream_t stream, PressureSetup& S, int* nparts);

// Transport setups for the mixed-precision form (tse_transport.cu): the
// exact form's arrays plus, from the same pass, the FP32 records, r' of the
// initial iterate and *nparts per-block x^2 partials (S.partials) -- the
// first correction cycle's scale and residual.
int setup_species_dc(const TseGrid* grid, const TseSpeciesArgs* a, void* d_ws, size_t ws_bytes,
                     cudaStream_t stream, TransportSetup& S, int* nparts);
int setup_heat_dc(const TseGrid* grid, const TseHeatArgs* a, void* d_ws, size_t ws_bytes,
                  cudaStream_t stream, TransportSetup& S, int* nparts);

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

// ------------------------------------------------ FP32 sweeps, bulk-copy staged
// The same iterations as dc_sweep_kernel, with the memory side rebuilt for
// bytes in flight: the cells of a colour are cut into chunks of kTmaChunk,
// block b takes chunks b, b + G, ...; for each chunk one thread issues bulk
// asynchronous copies (cp.async.bulk, completion counted on an mbarrier) of
// everything the chunk's relaxations read -- the 24-byte coefficient records,
// r', the flag bytes, the old correction and three windows of the other
// colour's correction (x+, x-, and one covering y+-, z+-) -- into one of
// kTmaStages shared-memory stages; the block computes from filled stages
// while later chunks are in flight, so each SM keeps up to ~190 KB of reads
// outstanding with no registers held for them.  The per-cell arithmetic is
// relax()'s, operation for operation, so the corrections are identical to
// dc_sweep_kernel's; only the grouping of the check sums differs.
#ifndef TSE_TMA_CHUNK
#define TSE_TMA_CHUNK 512
#endif
#ifndef TSE_TMA_STAGES
#define TSE_TMA_STAGES 4   // two stages in computation, the rest in flight
#endif
#ifndef TSE_TMA_MINB
#define TSE_TMA_MINB 2
#endif
constexpr int kTmaChunk = TSE_TMA_CHUNK;
constexpr int kTmaStages = TSE_TMA_STAGES;
static_assert(kTmaChunk % 32 == 0, "chunk: 16-byte copies of every array");
static_assert(kTmaChunk <= kDcMaxChunk, "windows must stay inside the correction margins");

// byte offsets of one stage's arrays (all multiples of 16)
struct TmaStage {
    int rec, rp, msk, dw, wz, wxp, wxm, bytes;
    int lz, lx;   // window lengths in floats
    int stages;   // stages of the launch, over all its pipelines (set by the launcher)
    int chunk;    // cells a chunk (256, 512 or 1024)
};

__host__ __device__ inline TmaStage tma_stage(int H, int C = kTmaChunk) {
    TmaStage t;
    t.chunk = C;
    t.rec = 0;
    t.rp = 24 * C;
    t.msk = t.rp + 4 * C;
    t.dw = t.msk + C;
    t.wz = t.dw + 4 * C;
    // [m0 - H - 1, m0 + C + H] from a start rounded down by up to 3 floats
    t.lz = (C + 2 * H + 5 + 3) & ~3;
    // [m0 +- SX, m0 +- SX + C) from a start rounded down by up to 3 floats
    t.lx = C + 4;
    t.wxp = t.wz + 4 * t.lz;
    t.wxm = t.wxp + 4 * t.lx;
    t.bytes = (t.wxm + 4 * t.lx + 127) & ~127;
    t.stages = kTmaStages;
    return t;
}

// Chunk q of the colour being swept, in two parts.  The first part (records,
// r', flags, the chunk's own old correction) depends on nothing another block
// writes during the launch -- the old correction of a chunk is written only
// by the block that owns the chunk -- so it may be issued before the grid
// barrier that ends the previous phase; it adds its bytes to the stage's
// transaction count without arriving.  The second part (the three windows of
// the other colour, which other blocks have just written) is issued after the
// barrier and carries the stage's single arrival.
__device__ __forceinline__ void tma_issue_own_n(long long N, const TmaStage& T, unsigned char* stage,
                                                uint64_t* bar, const float* Kc, const float* dw,
                                                const uint8_t* msk, long long m0, long long cnt) {
    const unsigned b_rec = (unsigned)(24 * cnt), b_rp = (unsigned)(4 * cnt), b_msk = (unsigned)cnt,
                   b_dw = (unsigned)(4 * cnt);
    const uint64_t first = l2_evict_first(), last = l2_evict_last();
    mbar_add_tx(bar, b_rec + b_rp + b_msk + b_dw);
    bulk_g2s_hint(stage + T.rec, Kc + 6 * m0, b_rec, bar, first);
    bulk_g2s_hint(stage + T.rp, Kc + 6 * N + m0, b_rp, bar, first);
    bulk_g2s_hint(stage + T.msk, msk + m0, b_msk, bar, first);
    bulk_g2s_hint(stage + T.dw, dw + m0, b_dw, bar, last);
}

__device__ __forceinline__ void tma_issue_own(const DcCtl& c, const TmaStage& T, unsigned char* stage,
                                              uint64_t* bar, const float* Kc, const float* dw,
                                              const uint8_t* msk, long long m0, long long cnt) {
    tma_issue_own_n(c.Ncal, T, stage, bar, Kc, dw, msk, m0, cnt);
}

__device__ __forceinline__ void tma_issue_windows_n(long long SX, int H, const TmaStage& T,
                                                    unsigned char* stage, uint64_t* bar, const float* dq,
                                                    long long m0) {
    const long long zs = (m0 - H - 1) & ~3LL;
    const long long xps = (m0 + SX) & ~3LL;
    const long long xms = (m0 - SX) & ~3LL;
    // this model's own window length (a batch's stage slot is sized for its
    // largest H; a longer copy could leave this model's margins)
    const unsigned b_z = (unsigned)(4 * tma_stage(H, T.chunk).lz), b_x = (unsigned)(4 * T.lx);
    const uint64_t last = l2_evict_last();
    mbar_expect_tx(bar, b_z + 2 * b_x);
    bulk_g2s_hint(stage + T.wz, dq + zs, b_z, bar, last);
    bulk_g2s_hint(stage + T.wxp, dq + xps, b_x, bar, last);
    bulk_g2s_hint(stage + T.wxm, dq + xms, b_x, bar, last);
}

__device__ __forceinline__ void tma_issue_windows(const DcCtl& c, const TmaStage& T, unsigned char* stage,
                                                  uint64_t* bar, const float* dq, long long m0) {
    tma_issue_windows_n(c.L.SX, c.L.H, T, stage, bar, dq, m0);
}

// Roles: warps 0-7 consume, in two groups of four warps; group g computes the
// block's chunks i = g, g + 2, ..., so two chunks are in computation at once
// and neither waits for the other.  Warp 8 produces: its lane 0 issues the
// copies of chunk i into stage i % kTmaStages as soon as the consumers of
// chunk i - kTmaStages have released that stage (`empty` barrier, one arrival
// per consumer warp).  Consumers wait on the stage's `full` barrier (the
// copies' byte count).  Only the colour phases end in block- and grid-wide
// barriers.  Every wait is bounded; a wait that runs out raises a block flag
// that ends every other wait of the block, and the kernel leaves with
// EV_ERROR after the copies still in flight have landed (again bounded).
constexpr int kTmaConsumers = 256;                    // 8 warps, two groups of 4
constexpr int kTmaGroup = kTmaConsumers / 2;
constexpr int kTmaThreads = kTmaConsumers + 32;       // + one producer warp
constexpr int kTmaCellsPerThread = kTmaChunk / kTmaGroup;
static_assert(kTmaChunk % kTmaGroup == 0, "whole cells per consumer thread");

}  // namespace tse
