// Staged form of the FP64 persistent solve: the loop of rb_solve_kernel (the
// reference's `while not converged` of compute_P tse.py:699-740, compute_C
// 877-914 and compute_T 1045-1079) -- same checks, dt growth and halving,
// same per-cell arithmetic operation for operation (the forms' update_with)
// -- with the memory side of each half-sweep rebuilt for bytes in flight.
//
// The cells of a colour are cut into chunks of kXChunk; block b takes chunks
// b, b + G, ...  A producer warp issues, for each chunk, bulk asynchronous
// copies (cp.async.bulk, completion counted on an mbarrier; one copy a lane)
// of everything the chunk's updates read: the form's coefficient arrays, the
// old solution, the flag bytes and three windows of the other colour's
// solution (x+, x-, and one covering y+-, z+-), into a shared-memory stage
// of its ring as soon as the consumers have released the stage.  Consumer
// warps (groups of kXGroup threads) compute from filled stages and store the
// new values straight to global memory.  Only the colour phases end in
// block- and grid-wide barriers.  Every wait is bounded; a wait that runs out
// raises a block flag that ends the block's other waits, and the kernel
// reports TSE_STATUS_BARRIER_TIMEOUT after its in-flight copies have landed
// (again bounded).
//
// The per-cell values are identical to rb_solve_kernel's; only the grouping
// of the L2 sums of the convergence check differs (as between any two block
// counts of either kernel).
#pragma once

#include "tse_rbsolve.cuh"
#include "tse_tma.cuh"

namespace tse {

#ifndef TSE_X_CHUNK
#define TSE_X_CHUNK 256
#endif
#ifndef TSE_X_MINB
#define TSE_X_MINB 1          // blocks per SM the shared-memory plan is sized for
#endif
#ifndef TSE_X_STAGES
#define TSE_X_STAGES 8        // at most, over all pipelines
#endif
#ifndef TSE_X_GROUPS
#define TSE_X_GROUPS 2        // consumer groups, each computing its own chunks
#endif
#ifndef TSE_X_PIPES
#define TSE_X_PIPES 2         // independent pipelines (producer warp + stage ring)
#endif
constexpr int kXChunk = TSE_X_CHUNK;                  // cells per chunk
#ifndef TSE_X_CONSUMERS
#define TSE_X_CONSUMERS 256   // consumer threads
#endif
constexpr int kXConsumers = TSE_X_CONSUMERS;
constexpr int kXGroups = TSE_X_GROUPS;
constexpr int kXGroup = kXConsumers / kXGroups;
// Pipeline r: producer warp r, the consumer groups g with g % kXPipes == r,
// its own ring of stages and the chunks i = r, r + kXPipes, ... of each
// phase.  Each ring has one issuer that issues in order, which the parity
// waits on its mbarriers rely on: a stage is refilled only after its
// previous use was consumed, and that use only after the one before.
constexpr int kXPipes = TSE_X_PIPES;
constexpr int kXThreads = kXConsumers + 32 * kXPipes;
static_assert(kXGroups % kXPipes == 0, "every pipeline has its own consumer groups");
constexpr int kXCellsPerThread = kXChunk / kXGroup;
constexpr int kXMaxArrays = 16;   // + 5 more copies: one lane each
constexpr int kXMaxStages = TSE_X_STAGES;
static_assert(kXChunk % kXGroup == 0 && kXChunk >= kXGroup, "whole cells per consumer thread");
static_assert(kXChunk % 32 == 0, "flag-byte copies stay multiples of 16 bytes");

// Shared-memory plan of one staged solve (byte offsets are multiples of 16).
struct XPlan {
    int nst;                    // coefficient arrays staged per chunk
    int idx[kXMaxArrays];       // their indices in the form's array set
    signed char slot[24];       // form array index -> place among the staged ones
    int xo, msk, wz, wxp, wxm;  // old solution, flags, windows
    int lz, lx;                 // window lengths in doubles
    int bytes;                  // one stage, a multiple of 128
    int stages;
};

// Fill `P` for form F on layout L; false when no stage layout fits (very
// long columns), in which case the plain kernel runs.
template <class Form>
inline bool x_plan(const Form& F, const Layout& L, int smem_per_block, XPlan& P) {
    static_assert(Form::kArrays <= 24, "slot table");
    P.nst = F.staged_arrays(P.idx);
    // arrays a form reads only under a switch that is off map to slot 0:
    // never used, but any load of them stays inside the stage
    for (int k = 0; k < 24; ++k) P.slot[k] = 0;
    for (int q = 0; q < P.nst; ++q) P.slot[P.idx[q]] = (signed char)q;
    const long long C = kXChunk, H = L.H;
    P.xo = (int)(P.nst * C * 8);
    P.msk = P.xo + (int)(C * 8);
    P.wz = P.msk + (int)C;
    // [m0 - H, m0 + C + H) from a start rounded down to an even cell
    const long long lz = C + 2 * H + 2;
    const long long lx = C + 2;    // [m0 +- SX, m0 +- SX + C) likewise
    const long long bytes = ((long long)P.wz + 8 * lz + 16 * lx + 127) & ~127LL;
    P.lz = (int)lz;
    P.lx = (int)lx;
    P.wxp = P.wz + (int)(8 * lz);
    P.wxm = P.wxp + (int)(8 * lx);
    P.bytes = (int)bytes;
    P.stages = (int)(smem_per_block / bytes);
    if (P.stages > kXMaxStages) P.stages = kXMaxStages;
    P.stages -= P.stages % kXPipes;                 // an equal ring per pipeline
    return P.stages >= 2 * kXPipes;
}

// copy [s, s + len) of a solution array of n entries into dst, clamped to
// the array (the cells outside it are never read: their flags are unset);
// s and n are even, so every copy is 16-byte aligned and sized
__device__ __forceinline__ unsigned x_window_bytes(long long s, long long len, long long n) {
    const long long a = s > 0 ? s : 0, e = (s + len) < n ? (s + len) : n;
    return e > a ? (unsigned)(8 * (e - a)) : 0u;
}
__device__ __forceinline__ void x_window(unsigned char* dst, const double* X, long long s, long long len,
                                         long long n, uint64_t* bar, uint64_t policy) {
    const long long a = s > 0 ? s : 0;
    const unsigned bytes = x_window_bytes(s, len, n);
    if (bytes) bulk_g2s_hint(dst + 8 * (a - s), X + a, bytes, bar, policy);
}

template <class Form, int RING>
__global__ void __launch_bounds__(kXThreads, TSE_X_MINB) rb_solve_tma_kernel(Form F, SolveCtl c, XPlan P) {
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ __align__(8) uint64_t full[kXMaxStages];
    __shared__ __align__(8) uint64_t empty[kXMaxStages];
    __shared__ double sh[kXThreads / 32];
    __shared__ double s_diff;
    __shared__ int s_err;
    __shared__ int s_idx[kXMaxArrays];   // the producer's indexed table (no local copy)
    const unsigned nb = gridDim.x, b = blockIdx.x;
    const int tid = threadIdx.x;
    const int warp = tid >> 5, lane = tid & 31;
    const bool producer = warp >= kXConsumers / 32;
    const int group = tid / kXGroup;                    // consumers: 0 .. kXGroups-1
    const int gt = tid & (kXGroup - 1);
    // this thread's pipeline, and a consumer group's rank within it
    const int pipe = producer ? warp - kXConsumers / 32 : group % kXPipes;
    const int grank = group / kXPipes;
    constexpr int kGroupsPerPipe = kXGroups / kXPipes;
    const long long Nc = c.L.Nc, N = c.Ncal, SX = c.L.SX, C = kXChunk;
    const int H = c.L.H;
    constexpr unsigned S = RING * kXPipes;              // P.stages
    constexpr unsigned Sp = RING;                       // stages of a ring
    const unsigned ring0 = (unsigned)pipe * Sp;         // this pipeline's first stage
    const long long nch = (Nc + C - 1) / C;
    const long long mine = nch > (long long)b ? (nch - 1 - b) / nb + 1 : 0;
    // this pipeline's chunks of a phase: i = pipe, pipe + kXPipes, ...
    const long long pmine = mine > pipe ? (mine - 1 - pipe) / kXPipes + 1 : 0;
    const bool leader = (b == 0 && tid == 0);
    const uint64_t keep = l2_evict_last();
    volatile int* err = &s_err;

    if (tid == 0) {
        for (unsigned s = 0; s < S; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], kXGroup / 32);   // one arrival per warp of a group
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        s_err = 0;
    }
#pragma unroll
    for (int q = 0; q < kXMaxArrays; ++q)
        if (tid == q) s_idx[q] = P.idx[q];
    __syncthreads();
    unsigned uses = 0;         // chunks of this pipeline consumed, over all phases
    unsigned phase_base = 0;   // `uses` when the current phase began
    long long pstop = 0;       // producer: first of its chunks of the phase not issued

    double t = 0.0, dt = c.dt, diff = 1e100;
    int converged = 0, num_it = 0, num_sub_it = 0, halvings = 0, fail = 0, nev = 0;

    while (!converged) {
        num_it += 1;
        num_sub_it += 1;
        double d2 = 0.0, o2 = 0.0;
        const bool check = c.pressure_schedule ? (num_it < 50 || num_it % 10 == 0) : true;
        for (int col = 0; col < 2; ++col) {
            // selects, not indexed loads: kernel parameters indexed by a
            // runtime value would be copied to local memory
            double* Xw = col ? c.X[1] : c.X[0];
            const double* Xo = col ? c.X[0] : c.X[1];
            phase_base = uses;
            if (producer) {
                // the other colour (and, after a halving, the reset arrays)
                // were written by generic stores before the grid barrier; the
                // copies read them through the async proxy
                fence_proxy_async();
                const double* arr = col ? F.arr[1] : F.arr[0];
                const uint8_t* msk = col ? c.mask[1] : c.mask[0];
                const uint64_t first = l2_evict_first();
                for (pstop = 0; pstop < pmine; ++pstop) {
                    const long long i = pipe + pstop * kXPipes;
                    const unsigned u = uses + (unsigned)pstop;
                    const unsigned s = ring0 + u % Sp;
                    // lane 0 waits for the stage, the warp follows its outcome
                    int okw = 1;
                    if (lane == 0 && u >= Sp) okw = mbar_wait_flag(&empty[s], (u / Sp - 1) & 1u, err);
                    if (!__shfl_sync(0xffffffffu, okw, 0)) break;
                    const long long m0 = (b + i * nb) * C;
                    const long long cnt = (N - m0) < C ? (N - m0) : C;   // % 32 == 0
                    const long long zs = (m0 - H) & ~1LL;
                    const long long xps = (m0 + SX) & ~1LL, xms = (m0 - SX) & ~1LL;
                    unsigned char* stg = smem + (size_t)s * P.bytes;
                    uint64_t* bar = &full[s];
                    const unsigned b_arr = (unsigned)(8 * cnt);
                    if (lane == 0)
                        mbar_expect_tx(bar, (unsigned)(P.nst + 1) * b_arr + (unsigned)cnt +
                                                x_window_bytes(zs, P.lz, N) +
                                                x_window_bytes(xps, P.lx, N) +
                                                x_window_bytes(xms, P.lx, N));
                    __syncwarp();
                    // one copy a lane: a single thread issues bulk copies
                    // one after another, far slower than the copies stream
                    if (lane < P.nst)
                        bulk_g2s_hint(stg + (size_t)lane * C * 8, arr + (size_t)s_idx[lane] * N + m0,
                                      b_arr, bar, first);
                    else if (lane == P.nst)
                        bulk_g2s_hint(stg + P.xo, Xw + m0, b_arr, bar, keep);
                    else if (lane == P.nst + 1)
                        bulk_g2s_hint(stg + P.msk, msk + m0, (unsigned)cnt, bar, first);
                    else if (lane == P.nst + 2)
                        x_window(stg + P.wz, Xo, zs, P.lz, N, bar, keep);
                    else if (lane == P.nst + 3)
                        x_window(stg + P.wxp, Xo, xps, P.lx, N, bar, keep);
                    else if (lane == P.nst + 4)
                        x_window(stg + P.wxm, Xo, xms, P.lx, N, bar, keep);
                }
                __syncwarp();
            } else {
                for (long long j = grank; j < pmine; j += kGroupsPerPipe) {
                    const long long i = pipe + j * kXPipes;
                    const unsigned u = uses + (unsigned)j;
                    const unsigned s = ring0 + u % Sp;
                    // warp-uniform: lane 0 waits, the warp follows its outcome,
                    // then every lane observes the completed phase (acquire)
                    int okw = 1;
                    if (lane == 0) okw = mbar_wait_flag(&full[s], (u / Sp) & 1u, err);
                    if (!__shfl_sync(0xffffffffu, okw, 0)) break;
                    mbar_try_wait(&full[s], (u / Sp) & 1u);
                    const unsigned char* stg = smem + (size_t)s * P.bytes;
                    const long long m0 = (b + i * nb) * C;
                    const int nval = (int)((Nc - m0) < C ? (Nc - m0) : C);
                    const int oz = (int)(m0 - ((m0 - H) & ~1LL));
                    const int oxp = (int)(m0 + SX - ((m0 + SX) & ~1LL));
                    const int oxm = (int)(m0 - SX - ((m0 - SX) & ~1LL));
                    const double* sa = reinterpret_cast<const double*>(stg);
                    const double* xo = reinterpret_cast<const double*>(stg + P.xo);
                    const uint8_t* fl = stg + P.msk;
                    const double* wz = reinterpret_cast<const double*>(stg + P.wz);
                    const double* wxp = reinterpret_cast<const double*>(stg + P.wxp);
                    const double* wxm = reinterpret_cast<const double*>(stg + P.wxm);
                    double* out = Xw + m0;
#pragma unroll
                    for (int r = 0; r < kXCellsPerThread; ++r) {
                        const int l = gt + r * kXGroup;
                        if (l < nval) {
                            const uint8_t f = fl[l];
                            const double xold = xo[l];
                            o2 = o2 + xold * xold;
                            if (f & F_ACTIVE) {
                                const int iz = l + oz, zo = f >> 7;
                                const double xn = F.update_with(
                                    [&](int k) { return sa[P.slot[k] * kXChunk + l]; },
                                    [&](int q) {
                                        return q == 0 ? wxp[l + oxp]
                                             : q == 1 ? wxm[l + oxm]
                                             : q == 2 ? wz[iz + H]
                                             : q == 3 ? wz[iz - H]
                                             : q == 4 ? wz[iz + zo]
                                                      : wz[iz - 1 + zo];
                                    },
                                    f, xold);
                                st_hint(out + l, xn, keep);
                                const double d = xn - xold;
                                d2 = d2 + d * d;
                            }
                        }
                    }
                    // the warp's reads of the stage are done: release it
                    __syncwarp();
                    if (lane == 0) mbar_arrive(&empty[s]);
                }
            }
            uses += (unsigned)pmine;
            // this phase's stores are read by the next phase's copies
            fence_proxy_async();
            __syncthreads();
            if (*err) { fail = 1; break; }   // block-uniform after the barrier
            if (col == 1 && check) {
                // per-block partial sums, published by the barrier below
                const double b1 = block_sum<kXThreads>(d2, sh);
                const double b2 = block_sum<kXThreads>(o2, sh);
                if (tid == 0) {
                    c.partials[2 * b] = b1;
                    c.partials[2 * b + 1] = b2;
                }
            }
            if (!grid_sync(c.bar, nb)) { fail = 1; break; }
        }
        if (fail) break;
        diff = 1e100;
        if (check) {
            double s1 = 0.0, s2 = 0.0;
            for (unsigned q = tid; q < nb; q += blockDim.x) {
                s1 = s1 + __ldcg(c.partials + 2 * q);
                s2 = s2 + __ldcg(c.partials + 2 * q + 1);
            }
            s1 = block_sum<kXThreads>(s1, sh);
            s2 = block_sum<kXThreads>(s2, sh);
            if (tid == 0) {
                const double l2 = sqrt(s1) / sqrt(s2 + 1e-200);
                s_diff = (l2 != l2) ? 1.0 : l2;
            }
            __syncthreads();
            diff = s_diff;
            // the next partial writes come after the next half-sweep barrier,
            // which every block reaches only after this read
        }
        if (diff < c.conv || c.stop_on_first) {
            converged = 1;
            t += dt;
            if (num_sub_it < c.max_it / 2.0) dt = pymin(dt * c.inc_it, c.max_dt);
        } else {
            if (num_sub_it >= c.max_it) {
                if (leader && nev < 8) {
                    c.status->ev_it[nev] = num_it;
                    c.status->ev_dt[nev] = dt;
                    c.status->ev_diff[nev] = diff;
                }
                nev += 1;
                dt = dt / 2;
                num_sub_it = 0;
                halvings += 1;
                const long long stride = (long long)nb * blockDim.x;
                for (int col = 0; col < 2; ++col)
                    for (long long m = (long long)b * blockDim.x + tid; m < Nc; m += stride)
                        F.reassemble(col, m, dt);
                // the reset arrays are read next by the copies
                fence_proxy_async();
                if (!grid_sync(c.bar, nb)) { fail = 1; break; }
            }
            if (dt <= c.min_dt) break;
        }
    }
    if (fail && producer && lane == 0) {
        // every copy this block issued lands before its shared memory is
        // released (bounded waits).  Earlier phases were consumed in full;
        // of this phase's chunks, a warp's own issued ones (the waits return
        // at once for those already complete)
        atomicExch(&c.bar->error, 1);
        for (long long j = 0; j < pstop && j < pmine; ++j) {
            const unsigned v = phase_base + (unsigned)j;
            mbar_wait_bounded(&full[ring0 + v % Sp], (v / Sp) & 1u);
        }
    }
    if (leader) {
        TseSolveStatus* s = c.status;
        s->t = t;
        s->dt = dt;
        s->diff = diff;
        s->converged = converged;
        s->num_it = num_it;
        s->num_sub_it = num_sub_it;
        s->halvings = halvings;
        s->error = fail ? TSE_STATUS_BARRIER_TIMEOUT : TSE_STATUS_OK;
        s->n_events = nev < 8 ? nev : 8;
        s->cycles = 0;
    }
}

// Launch the staged loop when selected and its stages fit, TSE_X_MINB blocks
// per SM (fewer for small grids: at least four chunks a block per half-sweep).
// Returns TSE_OK, TSE_ERR_LAUNCH, or 1 when the plain kernel should run.
template <class Form>
inline int launch_rb_solve_tma(const Form& F, SolveCtl& ctl, cudaStream_t stream) {
    if (ctl.plain_sweep) return 1;
    int dev = 0, sms = 0, optin = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess)
        return 1;
    int per_sm_smem = 0;
    cudaDeviceGetAttribute(&per_sm_smem, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev);
    // TSE_X_MINB blocks per SM: their share of the SM's shared memory less
    // each block's reserved 1 KB and static arrays
    const int budget = per_sm_smem / TSE_X_MINB - 2048;
    XPlan P;
    if (budget <= 0 || !x_plan(F, ctl.L, budget < optin ? budget : optin, P)) return 1;
    // one instantiation per ring length (2, 3 or 4 stages): stage and parity
    // arithmetic by compile-time constants
    constexpr int kMaxRing = kXMaxStages / kXPipes;
    constexpr int kR3 = kMaxRing < 3 ? 2 : 3, kR4 = kMaxRing < 4 ? kR3 : 4;
    const int avail = P.stages / kXPipes;
    const int ring = avail >= kR4 ? kR4 : avail >= kR3 ? kR3 : 2;
    const void* kernel = ring == kR4   ? (const void*)rb_solve_tma_kernel<Form, kR4>
                         : ring == kR3 ? (const void*)rb_solve_tma_kernel<Form, kR3>
                                       : (const void*)rb_solve_tma_kernel<Form, 2>;
    P.stages = ring * kXPipes;
    // a fixed ceiling, set once per call (no per-size attribute changes that
    // concurrent host threads could interleave)
    if (cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             budget < optin ? budget : optin) != cudaSuccess) {
        cudaGetLastError();
        return 1;
    }
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kXThreads, P.stages * P.bytes) !=
            cudaSuccess ||
        per_sm < 1) {
        cudaGetLastError();
        return 1;
    }
    const long long nch = (ctl.L.Nc + kXChunk - 1) / kXChunk;
    long long nb = (nch + 3) / 4;
    const long long maxb = (long long)sms * per_sm;
    if (nb > maxb) nb = maxb;
    if (nb < 1) nb = 1;
    if (nb > kMaxBlocks) nb = kMaxBlocks;
    void* args[] = {(void*)&F, (void*)&ctl, (void*)&P};
    const cudaError_t e = cudaLaunchCooperativeKernel(kernel, dim3((unsigned)nb), dim3(kXThreads), args,
                                                      (size_t)P.stages * P.bytes, stream);
    return e == cudaSuccess ? TSE_OK : TSE_ERR_LAUNCH;
}

}  // namespace tse
