// FP32 red-black SOR with FP64 defect correction: the mixed-precision form of
// the pressure, species and heat solves.
//
// The FP64 solves (tse_pressure.cu, tse_transport.cu) stream 11-15 double
// words per cell-update.  Here the same SOR iteration runs on a correction:
// with the FP64 iterate x, the residual of the reference's per-cell equation
//   r = sum(x) - Den * x            (sum / Den as in compute_P/C/T.solve)
// is formed in FP64, and red-black SOR sweeps
//   d = (1 - SOR) d + SOR (sum_q K'_q d_q + r')  with K'_q = k_q / Den, r' = r / Den
// run in FP32 from d = 0.  In exact arithmetic x + d follows the FP64 SOR
// iteration step for step, so the reference's convergence test (relative L2
// change of one iteration, checked on its schedule) and its dt control are
// applied to the change of d unchanged.  x += d in FP64 and the residual is
// formed again (a correction cycle ends) at convergence, every `cycle`
// iterations, and at a check whose change has fallen below kRefresh * |d|:
// FP32 resolves d to ~6e-8 |d|, so the measured change stays ~1e3 times above
// d's rounding and the iteration counts track the FP64 form's.
//
// Kernels: the FP32 sweeps run in one cooperative kernel that iterates until
// an event (converged, cycle end, dt halving, stop): dc_sweep_tma_kernel,
// which stages each chunk's data in shared memory with bulk asynchronous
// copies, or, where its stages do not fit, dc_sweep_kernel (48 registers,
// 5 blocks per SM, plain loads).  The FP64 residual, the x += d update and the dt
// halving (reset + new R terms) are separate, ordinary kernels, so their
// register appetite does not limit the sweeps' occupancy; the first cycle's
// records, residual and x^2 come from the assembly pass itself (setup_*_dc),
// and the last x += d is fused with the unpack.  The host reads one small
// state record per correction cycle.
//
// An inner cell-update streams the six FP32 coefficients (one 24-byte record),
// r' and the flag byte from DRAM -- 29 bytes; d and the neighbours' d stay in
// L2 -- against 89 bytes of coefficients and flags for the FP64 form.
//
// Compiled with FMA contraction (no bit-exactness is claimed for this form).
#include "tse_dc.cuh"

namespace tse {

#ifndef TSE_SWEEP_MINB
#define TSE_SWEEP_MINB 5   // 48 registers, no spills (measured best of 4/5/6/8)
#endif
constexpr int kSweepMinBlocks = TSE_SWEEP_MINB;
#ifndef TSE_SWEEP_BLOCK
#define TSE_SWEEP_BLOCK 256
#endif
constexpr int kSweepBlock = TSE_SWEEP_BLOCK;
#ifndef TSE_TMA_PREFETCH
#define TSE_TMA_PREFETCH 1   // 1: a phase's own parts are copied before its grid barrier
#endif

// Pipelines of the staged sweep: each has its own producer warp, its own ring
// of stages and its own consumer group, and takes every PIPES-th chunk of the
// block.  A producer warp issues its copies one after another, at a rate that
// bounds a pipeline's throughput: two pipelines per block, one block per SM,
// up to 4 stages a ring.  (Measured against one pipeline -- two consumer
// groups sharing a ring -- and two blocks per SM: faster at every grid from
// 96^3 to 256 x 256 x 128.)
constexpr int kDcPipes = 2;
constexpr int kDcMaxRing = 4;
template <int PIPES>
struct DcLayout {
    static constexpr int kThreads = kTmaConsumers + 32 * PIPES;
    static constexpr int kMinBlocks = PIPES == 1 ? 2 : 1;
    static constexpr int kGroupsPerPipe = (kTmaConsumers / kTmaGroup) / PIPES;
    static_assert((kTmaConsumers / kTmaGroup) % PIPES == 0, "every pipeline has its own consumer groups");
};

// ------------------------------------------------------------ FP64 kernels
// a solve's state record at its start: all zero but dt and diff (written on
// the device, so starting a solve queues no host-memory copy)
__global__ void dc_init_state_kernel(DcState* st, double dt) {
    DcState s;
    memset(&s, 0, sizeof(s));
    s.dt = dt;
    s.diff = 1e100;
    *st = s;
}

// K'_q = k_q / Den for every cell (at the start and after dt halving)
template <class Form>
__global__ void dc_scale_kernel(Form F, DcCtl c) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= 2 * c.L.Nc) return;
    const int col = t >= c.L.Nc;
    scale_cell(F, c, col, t - col * c.L.Nc);
}

// dt halving: x = Xn, new R terms (tse.py:733-738), rescaled coefficients
template <class Form>
__global__ void dc_halve_kernel(Form F, DcCtl c) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= 2 * c.L.Nc) return;
    const int col = t >= c.L.Nc;
    const long long m = t - col * c.L.Nc;
    F.reassemble(col, m, c.st->dt);
    scale_cell(F, c, col, m);
}

// r' = (sum(x) - Den x) / Den in FP64, d = 0, per-block sums of x^2
template <class Form>
__global__ void __launch_bounds__(kBlock) dc_residual_kernel(Form F, DcCtl c) {
    __shared__ double sh[kBlock / 32];
    const double o2 = residual_block_cells(F, c, blockIdx.x, gridDim.x);
    const double b = block_sum<kBlock>(o2, sh);
    if (threadIdx.x == 0) c.partials[blockIdx.x] = b;
}

// x^2 total into the state; counts the cycle
__global__ void dc_x2_kernel(DcCtl c, int nparts) {
    __shared__ double sh[kBlock / 32];
    double s = 0.0;
    int b = threadIdx.x;
    // eight loads in flight, summed in the order of the plain loop
    for (; b + 7 * kBlock < nparts; b += 8 * kBlock) {
        double v[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) v[u] = c.partials[b + u * kBlock];
#pragma unroll
        for (int u = 0; u < 8; ++u) s = s + v[u];
    }
    for (; b < nparts; b += kBlock) s = s + c.partials[b];
    s = block_sum<kBlock>(s, sh);
    if (threadIdx.x == 0) {
        c.st->x2 = s;
        c.st->cycles += 1;
    }
}

// x += d for active cells
__global__ void dc_apply_kernel(DcCtl c) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= 2 * c.L.Nc) return;
    const int col = t >= c.L.Nc;
    const long long m = t - col * c.L.Nc;
    if (c.mask[col][m] & F_ACTIVE) c.X[col][m] = c.X[col][m] + (double)c.D[col][m];
}

// x += d and the natural-layout result in one pass: the last cycle of a
// solve (dc_apply_kernel then unpack_kernel, without storing x)
__global__ void dc_apply_unpack_kernel(double* out, DcCtl c) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long total = (long long)c.L.nx * c.L.ny * c.L.nz;
    if (t >= total) return;
    int i, j, k;
    long long row;
    grid_coords(t, c.L.ny, c.L.nz, i, j, k, row);
    const long long m = (row * c.L.nzp + k) >> 1;
    const int col = (i + j + k) & 1;
    double x = c.X[col][m];
    if (c.mask[col][m] & F_ACTIVE) x = x + (double)c.D[col][m];
    out[t] = x;
}

// ------------------------------------------------------------ FP32 sweeps
__device__ __forceinline__ double reduce_slot(const double* parts, int slot, unsigned nb, double* sh,
                                              double* s_val) {
    double s = 0.0;
    for (unsigned b = threadIdx.x; b < nb; b += blockDim.x) s = s + __ldcg(parts + 4 * b + slot);
    s = block_sum<kSweepBlock>(s, sh);
    if (threadIdx.x == 0) *s_val = s;
    __syncthreads();
    const double r = *s_val;
    __syncthreads();
    return r;
}

// Inner iterations of one correction cycle.  Cells are interleaved over the
// grid (block b, thread t: m = b*256 + t + s*gridDim*256), which keeps all
// blocks streaming one narrow window of memory; colour phases are separated
// by the grid barrier.  Per-block partial sums alternate between two slot
// pairs by check parity, so a slot is rewritten only after a further barrier.
__global__ void __launch_bounds__(kSweepBlock, kSweepMinBlocks) dc_sweep_kernel(DcCtl c) {
    __shared__ double sh[kSweepBlock / 32];
    __shared__ double s_val;
    const unsigned nb = gridDim.x;
    const long long Nc = c.L.Nc, N = c.Ncal, SX = c.L.SX;
    const int H = c.L.H;
    const int lane = threadIdx.x & 31;
    const long long end = Nc;
    const long long step = (long long)nb * blockDim.x;
    const long long w0 = (long long)blockIdx.x * blockDim.x + threadIdx.x - lane;
    const bool leader = (blockIdx.x == 0 && threadIdx.x == 0);
    const float sor = c.sor;
    DcState* st = c.st;
    double t = st->t, dt = st->dt, diff = 1e100;
    const double x2 = st->x2;
    int num_it = st->num_it, num_sub_it = st->num_sub_it, checkno = st->checkno;
    int event = EV_CYCLE_END;
    bool halved = false;

    for (int inner = 0; inner < c.cycle; ++inner) {
        num_it += 1;
        num_sub_it += 1;
        const bool check = c.pressure_schedule ? (num_it < 50 || num_it % 10 == 0) : true;
        if (check) checkno += 1;
        float d2 = 0.0f, dd = 0.0f;
        bool ok = true;
        for (int col = 0; col < 2 && ok; ++col) {
            const float* __restrict__ Kc = c.K[col];
            float* dw = c.D[col];
            const float* dq = c.D[1 - col];
            const uint8_t* __restrict__ msk = c.mask[col];
            // all loads of a cell are independent: coefficients of absent
            // neighbours are 0 and dq's margins are 0; inactive cells have
            // all-zero coefficients and r' = 0 and stay at d = 0.  Trips are
            // counted per warp so every lane joins the shuffles; lanes past
            // the end load a valid cell and store nothing.
            for (long long w = w0; w < end; w += step) {
                const long long ma = w + lane;
                const bool va = ma < end;
                const long long la = va ? ma : end - 1;
                Cell a;
                load_cell(a, Kc, dw, dq, msk, la, N, SX, H);
                const float na = relax(a, dq, la, end, sor);
                if (va) {
                    dw[ma] = na;
                    const float ch = na - a.old;
                    d2 = fmaf(ch, ch, d2);
                    dd = fmaf(na, na, dd);
                }
            }
            if (col == 1 && check) {
                const double b1 = block_sum<kSweepBlock>((double)d2, sh);
                const double b3 = block_sum<kSweepBlock>((double)dd, sh);
                if (threadIdx.x == 0) {
                    c.partials[4 * blockIdx.x + 2 * (checkno & 1)] = b1;
                    c.partials[4 * blockIdx.x + 2 * (checkno & 1) + 1] = b3;
                }
            }
            ok = grid_sync(c.bar, nb);
        }
        if (!ok) { event = EV_ERROR; break; }
        diff = 1e100;
        bool refresh = false;
        if (check) {
            const double s1 = reduce_slot(c.partials, 2 * (checkno & 1), nb, sh, &s_val);
            const double s3 = reduce_slot(c.partials, 2 * (checkno & 1) + 1, nb, sh, &s_val);
            const double l2 = sqrt(s1) / sqrt(x2 + 1e-200);
            diff = (l2 != l2) ? 1.0 : l2;
            refresh = sqrt(s1) < kRefresh * sqrt(s3);
        }
        if (diff < c.conv || c.stop_on_first) {
            t += dt;
            if (num_sub_it < c.max_it / 2.0) dt = pymin(dt * c.inc_it, c.max_dt);
            event = EV_CONVERGED;
            break;
        }
        if (num_sub_it >= c.max_it) {
            if (leader && st->nev < 8) {
                st->ev_it[st->nev] = num_it;
                st->ev_dt[st->nev] = dt;
                st->ev_diff[st->nev] = diff;
            }
            if (leader) st->nev += 1;
            dt = dt / 2;
            num_sub_it = 0;
            halved = true;
        }
        if (dt <= c.min_dt) { event = halved ? EV_STOP_HALVED : EV_STOP; break; }
        if (halved) { event = EV_HALVE; break; }
        if (refresh) { event = EV_REFRESH; break; }
    }
    if (leader) {
        st->t = t;
        st->dt = dt;
        st->diff = diff;
        st->num_it = num_it;
        st->num_sub_it = num_sub_it;
        st->checkno = checkno;
        st->event = event;
        if (halved) st->halvings += 1;
        if (event == EV_CONVERGED) st->converged = 1;
    }
}

// ------------------------------------------------ FP32 sweeps, bulk-copy staged
// (the staging pieces are in tse_dc.cuh)
template <int RING, int PIPES, int CHUNK>
__global__ void __launch_bounds__(DcLayout<PIPES>::kThreads, DcLayout<PIPES>::kMinBlocks)
    dc_sweep_tma_kernel(DcCtl c, TmaStage T) {
    static_assert(CHUNK % kTmaGroup == 0 && CHUNK <= kDcMaxChunk, "whole cells per thread, in the margins");
    constexpr int kCellsPerThread = CHUNK / kTmaGroup;
    constexpr int kPipes = PIPES;
    constexpr int kThreads = DcLayout<PIPES>::kThreads;
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ __align__(8) uint64_t full[RING * PIPES];
    __shared__ __align__(8) uint64_t empty[RING * PIPES];
    __shared__ double sh[kThreads / 32];
    __shared__ int s_err;
    const unsigned nb = gridDim.x, b = blockIdx.x;
    const int tid = threadIdx.x;
    const int warp = tid >> 5, lane = tid & 31;
    const bool producer = warp >= kTmaConsumers / 32;
    const int group = tid / kTmaGroup;                  // consumers: 0 or 1
    const int gt = tid & (kTmaGroup - 1);               // thread within its group
    // this thread's pipeline (producer warp + its ring of stages +
    // its consumer groups), and a consumer group's rank within it
    const int pipe = producer ? warp - kTmaConsumers / 32 : group % kPipes;
    const int grank = group / kPipes;
    constexpr int kGroupsPerPipe = DcLayout<PIPES>::kGroupsPerPipe;
    constexpr unsigned ring = RING;                     // stages of a ring (T.stages / PIPES)
    const unsigned ring0 = (unsigned)pipe * ring;    // the pipeline's first stage
    const long long Nc = c.L.Nc, N = c.Ncal, SX = c.L.SX, C = CHUNK;
    const int H = c.L.H;
    const long long nch = (Nc + C - 1) / C;
    const long long mine = nch > (long long)b ? (nch - 1 - b) / nb + 1 : 0;   // chunks of this block
    // this pipeline's chunks of a phase: i = pipe, pipe + kPipes, ...
    const long long pmine = mine > pipe ? (mine - 1 - pipe) / kPipes + 1 : 0;
    unsigned* bar_count = c.prog;   // count_sync's counter, zeroed before the launch
    unsigned bars = 0;              // device-wide barriers passed in this launch
    const bool leader = (b == 0 && tid == 0);
    const float sor = c.sor;
    const uint64_t keep = l2_evict_last();
    DcState* st = c.st;
    double t = st->t, dt = st->dt, diff = 1e100;
    const double x2 = st->x2;
    int num_it = st->num_it, num_sub_it = st->num_sub_it, checkno = st->checkno;
    int event = EV_CYCLE_END;
    bool halved = false;
    volatile int* err = &s_err;

    if (tid == 0) {
        for (int s = 0; s < RING * kPipes; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], kTmaGroup / 32);   // one arrival per warp of a group
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        s_err = 0;
    }
    __syncthreads();
    unsigned uses = 0;      // this pipeline's chunks consumed, over all colour phases
    unsigned issued = 0;    // producer: this pipeline's chunks issued, over all phases
    // producer: chunks of the coming phase whose own parts are already in flight
    long long primed = 0;
    const long long pro = pmine < (long long)ring ? pmine : (long long)ring;
#if TSE_TMA_PREFETCH
    if (producer && lane == 0) {
        for (long long j = 0; j < pro; ++j) {
            const long long m0 = (b + (pipe + j * kPipes) * nb) * C;
            const long long cnt = (N - m0) < C ? (N - m0) : C;
            tma_issue_own(c, T, smem + (size_t)(ring0 + j) * T.bytes, &full[ring0 + j], c.K[0], c.D[0],
                          c.mask[0], m0, cnt);
        }
        primed = pro;
    }
#endif

    for (int inner = 0; inner < c.cycle; ++inner) {
        num_it += 1;
        num_sub_it += 1;
        const bool check = c.pressure_schedule ? (num_it < 50 || num_it % 10 == 0) : true;
        if (check) checkno += 1;
        float d2 = 0.0f, dd = 0.0f;
        bool ok = true;
        for (int col = 0; col < 2 && ok; ++col) {
            const float* Kc = c.K[col];
            float* dw = c.D[col];
            const float* dq = c.D[1 - col];
            const uint8_t* msk = c.mask[col];
            if (producer) {
                if (lane == 0) {
                    // the other colour was written (generic stores) before
                    // the grid barrier; the copies read it through the async proxy
                    fence_proxy_async();
                    bool pok = true;
                    for (long long j = 0; j < pmine; ++j, ++issued) {
                        const unsigned s = ring0 + issued % ring;
                        const long long m0 = (b + (pipe + j * kPipes) * nb) * C;
                        unsigned char* stg = smem + (size_t)s * T.bytes;
                        if (j >= primed) {
                            if (issued >= (unsigned)ring &&
                                !mbar_wait_flag(&empty[s], (issued / ring - 1) & 1u, err)) {
                                pok = false;
                                break;
                            }
                            const long long cnt = (N - m0) < C ? (N - m0) : C;   // % 32 == 0
                            tma_issue_own(c, T, stg, &full[s], Kc, dw, msk, m0, cnt);
                        }
                        tma_issue_windows(c, T, stg, &full[s], dq, m0);
                    }
                    primed = 0;
#if TSE_TMA_PREFETCH
                    // the next phase's own parts (records, r', flags, own
                    // correction: nothing another block writes) go out as the
                    // consumers free the stages, before the grid barrier
                    const int nc = 1 - col;
                    for (long long j = 0; pok && j < pro; ++j) {
                        const unsigned v = issued + (unsigned)j;
                        const unsigned s = ring0 + v % ring;
                        if (v >= (unsigned)ring &&
                            !mbar_wait_flag(&empty[s], (v / ring - 1) & 1u, err))
                            break;
                        const long long m0 = (b + (pipe + j * kPipes) * nb) * C;
                        const long long cnt = (N - m0) < C ? (N - m0) : C;
                        tma_issue_own(c, T, smem + (size_t)s * T.bytes, &full[s], c.K[nc], c.D[nc],
                                      c.mask[nc], m0, cnt);
                        primed = j + 1;
                    }
#endif
                }
                __syncwarp();
            } else {
                for (long long j = grank; j < pmine; j += kGroupsPerPipe) {
                    const unsigned u = uses + (unsigned)j;
                    const unsigned s = ring0 + u % ring;
                    // warp-uniform: lane 0 waits, the warp follows its outcome,
                    // then every lane observes the completed phase (acquire)
                    int okw = 1;
                    if (lane == 0) okw = mbar_wait_flag(&full[s], (u / ring) & 1u, err);
                    if (!__shfl_sync(0xffffffffu, okw, 0)) break;
                    mbar_try_wait(&full[s], (u / ring) & 1u);
                    const unsigned char* stg = smem + (size_t)s * T.bytes;
                    const long long m0 = (b + (pipe + j * kPipes) * nb) * C;
                    const int nval = (int)((Nc - m0) < C ? (Nc - m0) : C);
                    // window offsets of cell l of the chunk (32-bit from here on)
                    const int oz = (int)(m0 - ((m0 - H - 1) & ~3LL));
                    const int oxp = (int)(m0 + SX - ((m0 + SX) & ~3LL));
                    const int oxm = (int)(m0 - SX - ((m0 - SX) & ~3LL));
                    const float2* rec = reinterpret_cast<const float2*>(stg + T.rec);
                    const float* rp = reinterpret_cast<const float*>(stg + T.rp);
                    const uint8_t* fl = stg + T.msk;
                    const float* dwo = reinterpret_cast<const float*>(stg + T.dw);
                    const float* wz = reinterpret_cast<const float*>(stg + T.wz);
                    const float* wxp = reinterpret_cast<const float*>(stg + T.wxp);
                    const float* wxm = reinterpret_cast<const float*>(stg + T.wxm);
                    float* out = dw + m0;
#pragma unroll
                    for (int r = 0; r < kCellsPerThread; ++r) {
                        const int l = gt + r * kTmaGroup;
                        if (l < nval) {
                            const float2 k01 = rec[3 * l], k23 = rec[3 * l + 1], k45 = rec[3 * l + 2];
                            const bool odd = (fl[l] & F_KODD) != 0;
                            const float old = dwo[l];
                            const int iz = l + oz;
                            const float z0 = wz[iz - 1], z1 = wz[iz], z2 = wz[iz + 1];
                            float acc = rp[l];
                            acc = fmaf(k01.x, wxp[l + oxp], acc);
                            acc = fmaf(k01.y, wxm[l + oxm], acc);
                            acc = fmaf(k23.x, wz[iz + H], acc);
                            acc = fmaf(k23.y, wz[iz - H], acc);
                            acc = fmaf(k45.x, odd ? z2 : z1, acc);
                            acc = fmaf(k45.y, odd ? z1 : z0, acc);
                            const float na = fmaf(sor, acc - old, old);
                            st_hint(out + l, na, keep);
                            const float ch = na - old;
                            d2 = fmaf(ch, ch, d2);
                            dd = fmaf(na, na, dd);
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
            if (*err) { ok = false; break; }   // block-uniform after the barrier
            if (col == 1 && check) {
                const double b1 = block_sum<kThreads>((double)d2, sh);
                const double b3 = block_sum<kThreads>((double)dd, sh);
                if (tid == 0) {
                    c.partials[4 * b + 2 * (checkno & 1)] = b1;
                    c.partials[4 * b + 2 * (checkno & 1) + 1] = b3;
                }
            }
            ok = count_sync(bar_count, ++bars * nb, c.bar);
        }
        if (!ok) { event = EV_ERROR; break; }
        diff = 1e100;
        bool refresh = false;
        if (check) {
            double s1 = 0.0, s3 = 0.0;
            for (unsigned q = tid; q < nb; q += blockDim.x) {
                s1 = s1 + __ldcg(c.partials + 4 * q + 2 * (checkno & 1));
                s3 = s3 + __ldcg(c.partials + 4 * q + 2 * (checkno & 1) + 1);
            }
            s1 = block_sum<kThreads>(s1, sh);
            s3 = block_sum<kThreads>(s3, sh);
            if (tid == 0) {
                sh[0] = s1;
                sh[1] = s3;
            }
            __syncthreads();
            s1 = sh[0];
            s3 = sh[1];
            __syncthreads();
            const double l2 = sqrt(s1) / sqrt(x2 + 1e-200);
            diff = (l2 != l2) ? 1.0 : l2;
            refresh = sqrt(s1) < kRefresh * sqrt(s3);
        }
        if (diff < c.conv || c.stop_on_first) {
            t += dt;
            if (num_sub_it < c.max_it / 2.0) dt = pymin(dt * c.inc_it, c.max_dt);
            event = EV_CONVERGED;
            break;
        }
        if (num_sub_it >= c.max_it) {
            if (leader && st->nev < 8) {
                st->ev_it[st->nev] = num_it;
                st->ev_dt[st->nev] = dt;
                st->ev_diff[st->nev] = diff;
            }
            if (leader) st->nev += 1;
            dt = dt / 2;
            num_sub_it = 0;
            halved = true;
        }
        if (dt <= c.min_dt) { event = halved ? EV_STOP_HALVED : EV_STOP; break; }
        if (halved) { event = EV_HALVE; break; }
        if (refresh) { event = EV_REFRESH; break; }
    }
    if (producer && lane == 0) {
        // every copy this block issued lands before its shared memory is
        // released (bounded waits, flag ignored): after an error the last
        // issued use of each stage; primed stages get their missing arrival
        if (event == EV_ERROR) {
            atomicExch(&c.bar->error, 1);
            const unsigned first = issued > (unsigned)ring ? issued - ring : 0u;
            for (unsigned v = first; v < issued; ++v)
                mbar_wait_bounded(&full[ring0 + v % ring], (v / ring) & 1u);
        }
        for (long long j = 0; j < primed; ++j) {
            const unsigned v = issued + (unsigned)j;
            mbar_arrive(&full[ring0 + v % ring]);
            mbar_wait_bounded(&full[ring0 + v % ring], (v / ring) & 1u);
        }
    }
    if (leader) {
        st->t = t;
        st->dt = dt;
        st->diff = diff;
        st->num_it = num_it;
        st->num_sub_it = num_sub_it;
        st->checkno = checkno;
        st->event = event;
        if (halved) st->halvings += 1;
        if (event == EV_CONVERGED) st->converged = 1;
    }
}

// copy the final state into the caller's status record
__global__ void dc_status_kernel(const DcState* st, TseSolveStatus* s) {
    s->t = st->t;
    s->dt = st->dt;
    s->diff = st->diff;
    s->converged = st->converged;
    s->num_it = st->num_it;
    s->num_sub_it = st->num_sub_it;
    s->halvings = st->halvings;
    s->error = st->event == EV_ERROR ? TSE_STATUS_BARRIER_TIMEOUT : TSE_STATUS_OK;
    s->n_events = st->nev < 8 ? st->nev : 8;
    for (int q = 0; q < 8; ++q) {
        s->ev_it[q] = st->ev_it[q];
        s->ev_dt[q] = st->ev_dt[q];
        s->ev_diff[q] = st->ev_diff[q];
    }
    s->cycles = st->cycles;
}

// ------------------------------------------------------------------ host
size_t dc_extra_bytes(const Layout& L) {
    long long Ncal = (L.Nc + 31) & ~31LL;
    return 2 * ((size_t)7 * Ncal + (size_t)dc_delta_len(L, Ncal)) * sizeof(float) +
           align256(sizeof(DcState)) + 256 + 512;
}

static int sweep_blocks(long long Nc, int cap) {
    static int cached_dev = -1, cached_per_sm = 0, cached_sms = 0;
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev != cached_dev) {
        cudaDeviceGetAttribute(&cached_sms, cudaDevAttrMultiProcessorCount, dev);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&cached_per_sm, dc_sweep_kernel, kSweepBlock, 0);
        cached_dev = dev;
    }
    long long maxb = (long long)cached_sms * (cached_per_sm > 0 ? cached_per_sm : 1);
    long long want = (Nc + (long long)kSweepBlock * 4 - 1) / ((long long)kSweepBlock * 4);
    if (want < 1) want = 1;
    long long nb = want < maxb ? want : maxb;
    // the setup's partials region holds 2 * kMaxBlocks doubles
    if (nb > kMaxBlocks / 2) nb = kMaxBlocks / 2;
    if (cap > 0 && nb > cap) nb = cap;
    return (int)nb;
}

#ifndef TSE_SWEEP_TMA
#define TSE_SWEEP_TMA 1   // 1: bulk-copy staged sweeps where the stages fit in shared memory
#endif
// dynamic shared memory ceiling of the staged sweep: the device's per-block
// opt-in limit less the kernel's static arrays and a margin
static size_t tma_max_smem() {
    int dev = 0, optin = 0;
    cudaGetDevice(&dev);
    if (cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return optin > 2048 ? (size_t)optin - 2048 : 0;
}

// blocks of the staged sweep: as many as fit (dynamic shared memory
// included), at most one per chunk of a colour; 0 when the stages for this
// grid's windows do not fit (the plain sweep kernel runs instead)
// the instantiation for rings of `ring` stages (2 .. 4), `pipes` pipelines
// per block (1: two blocks per SM) and chunks of `chunk` cells
template <int PIPES, int CHUNK>
static const void* tma_kernel_r(int ring) {
    return ring <= 2 ? (const void*)dc_sweep_tma_kernel<2, PIPES, CHUNK>
         : ring == 3 ? (const void*)dc_sweep_tma_kernel<3, PIPES, CHUNK>
                     : (const void*)dc_sweep_tma_kernel<4, PIPES, CHUNK>;
}
static const void* tma_kernel(int ring, int pipes, int chunk) {
    if (pipes == 1)
        return chunk == 256 ? tma_kernel_r<1, 256>(ring) : chunk == 1024 ? tma_kernel_r<1, 1024>(ring)
                                                                         : tma_kernel_r<1, 512>(ring);
    return chunk == 256 ? tma_kernel_r<2, 256>(ring) : chunk == 1024 ? tma_kernel_r<2, 1024>(ring)
                                                                     : tma_kernel_r<2, 512>(ring);
}

static int tma_blocks(long long Nc, int cap, size_t smem, const void* kernel, int threads, int chunk) {
    const size_t ceil_smem = tma_max_smem();
    if (!TSE_SWEEP_TMA || smem == 0 || smem > ceil_smem) return 0;
    int dev = 0, sms = 0, per_sm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    // the same ceiling for every grid, so concurrent callers never lower it
    // below another's launch
    if (cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ceil_smem) !=
            cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, smem) !=
            cudaSuccess ||
        per_sm < 1) {
        cudaGetLastError();
        return 0;
    }
    long long nb = (long long)sms * per_sm;
    const long long nch = (Nc + chunk - 1) / chunk;
    if (nb > nch) nb = nch;
    if (nb > kMaxBlocks / 2) nb = kMaxBlocks / 2;
    if (cap > 0 && nb > cap) nb = cap;
    return nb < 1 ? 1 : (int)nb;
}

template <class Form>
static int run_dc(SolveSetup<Form>& S, double dt, double inc_it, double max_dt, double min_dt,
                  double conv, int max_it, int pressure_schedule, int stop_on_first,
                  TseDcOptions* opts, double sor, int x_index, double* X_out,
                  TseSolveStatus* d_status, cudaStream_t stream, int first_parts = 0) {
    const int cycle = opts ? opts->cycle : 0;
    const int cap = opts ? opts->max_blocks : 0;
    if (S.tail_bytes < dc_extra_bytes(S.L)) return TSE_ERR_WORKSPACE;
    DcCtl c;
    dc_carve(S, c, x_index);
    c.inc_it = inc_it;
    c.max_dt = max_dt;
    c.min_dt = min_dt;
    c.conv = conv;
    c.max_it = max_it;
    c.pressure_schedule = pressure_schedule;
    c.stop_on_first = stop_on_first;
    c.cycle = cycle > 0 ? cycle : 256;
    c.sor = (float)sor;
    const long long dlen = dc_delta_len(S.L, S.Ncal);
    float* dbase = c.D[0] - dc_margin(S.L);
    // the margins must read as 0 (kernels rewrite the interior only)
    if (cudaMemsetAsync(dbase, 0, (size_t)2 * dlen * sizeof(float), stream) != cudaSuccess)
        return TSE_ERR_LAUNCH;
    dc_init_state_kernel<<<1, 1, 0, stream>>>(c.st, dt);
    if (cudaGetLastError() != cudaSuccess) return TSE_ERR_LAUNCH;
    const long long cells2 = 2 * S.L.Nc;
    const unsigned gcells = (unsigned)((cells2 + kBlock - 1) / kBlock);
    // the staged sweep's variant: chunk size, pipelines per block and ring
    // length from the call's options (0: 512 cells, 2 pipelines, as many
    // stages as fit up to 4 a ring)
    const int chunk = (opts && (opts->chunk == 256 || opts->chunk == 1024)) ? opts->chunk : 512;
    const int pipes = (opts && opts->pipes == 1) ? 1 : kDcPipes;
    const int want_ring = (opts && opts->ring >= 2 && opts->ring <= kDcMaxRing) ? opts->ring : kDcMaxRing;
    TmaStage T = tma_stage(S.L.H, chunk);
    {
        // one pipeline per block runs two blocks per SM: each gets half
        const size_t room = tma_max_smem() / (pipes == 1 ? 2 : 1);
        int st = (int)std::min<size_t>((size_t)(want_ring * pipes), room / (size_t)T.bytes);
        st -= st % pipes;
        T.stages = st >= 2 * pipes ? st : 0;
    }
    const size_t tma_smem = (size_t)T.stages * T.bytes;
    const int tma_threads = kTmaConsumers + 32 * pipes;
    const void* tma_k = T.stages > 0 ? tma_kernel(T.stages / pipes, pipes, chunk) : nullptr;
    const int nb_tma = tma_k ? tma_blocks(S.L.Nc, cap, tma_smem, tma_k, tma_threads, chunk) : 0;
    if (opts) {
        // the variant that ran (0 when the plain-load sweep did)
        opts->chunk = nb_tma > 0 ? chunk : 0;
        opts->pipes = nb_tma > 0 ? pipes : 0;
        opts->ring = nb_tma > 0 ? T.stages / pipes : 0;
    }
    const int nb = nb_tma > 0 ? nb_tma : sweep_blocks(S.L.Nc, cap);
    // first_parts > 0: the setup has written the records, r' and that many
    // x^2 partials (the first cycle's scale and residual)
    if (first_parts == 0) {
        dc_scale_kernel<<<gcells, kBlock, 0, stream>>>(S.F, c);
        if (cudaGetLastError() != cudaSuccess) return TSE_ERR_LAUNCH;
    }
    const bool timing = opts && opts->timing;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    if (timing) {
        opts->sweep_launches = 0;
        opts->sweep_iterations = 0;
        opts->sweep_ms = 0.0;
        opts->loop_ms = 0.0;
        if (cudaEventCreate(&ev0) != cudaSuccess || cudaEventCreate(&ev1) != cudaSuccess)
            return TSE_ERR_LAUNCH;
    }
    int prev_it = 0;
    int rc = TSE_OK;
    bool final_apply = false;
    for (;;) {
        if (first_parts > 0) {
            dc_x2_kernel<<<1, kBlock, 0, stream>>>(c, first_parts);
            first_parts = 0;
        } else {
            const unsigned rb = (unsigned)res_blocks(S.L.Nc);
            dc_residual_kernel<<<rb, kBlock, 0, stream>>>(S.F, c);
            dc_x2_kernel<<<1, kBlock, 0, stream>>>(c, (int)rb);
        }
        void* args[] = {(void*)&c};
        void* targs[] = {(void*)&c, (void*)&T};
        // staged sweep: its barrier counter starts at 0
        if (nb_tma > 0 && cudaMemsetAsync(c.prog, 0, sizeof(unsigned), stream) != cudaSuccess) {
            rc = TSE_ERR_LAUNCH;
            break;
        }
        if (timing) cudaEventRecord(ev0, stream);
        if (cudaGetLastError() != cudaSuccess) {
            rc = TSE_ERR_LAUNCH;
            break;
        }
        const cudaError_t le =
            nb_tma > 0 ? cudaLaunchCooperativeKernel(tma_k, dim3(nb),
                                                     dim3(tma_threads), targs, tma_smem, stream)
                       : cudaLaunchCooperativeKernel((const void*)dc_sweep_kernel, dim3(nb),
                                                     dim3(kSweepBlock), args, 0, stream);
        if (le != cudaSuccess) {
            rc = TSE_ERR_LAUNCH;
            break;
        }
        if (timing) cudaEventRecord(ev1, stream);
        int head[2] = {EV_ERROR, 0};   // event, num_it
        if (cudaMemcpyAsync(&head[0], &c.st->event, sizeof(int), cudaMemcpyDeviceToHost, stream) !=
                cudaSuccess ||
            cudaMemcpyAsync(&head[1], &c.st->num_it, sizeof(int), cudaMemcpyDeviceToHost, stream) !=
                cudaSuccess ||
            cudaStreamSynchronize(stream) != cudaSuccess) {
            rc = TSE_ERR_LAUNCH;
            break;
        }
        const int event = head[0];
        if (timing) {
            float ms = 0.0f;
            cudaEventElapsedTime(&ms, ev0, ev1);
            opts->sweep_launches += 1;
            opts->sweep_iterations += head[1] - prev_it;
            opts->sweep_ms += ms;
        }
        prev_it = head[1];
        if (event == EV_HALVE || event == EV_STOP_HALVED) {
            dc_halve_kernel<<<gcells, kBlock, 0, stream>>>(S.F, c);
            if (cudaGetLastError() != cudaSuccess) { rc = TSE_ERR_LAUNCH; break; }
            if (event == EV_STOP_HALVED) break;
            continue;
        }
        if (event == EV_ERROR) break;
        if (event == EV_CONVERGED || event == EV_STOP) {
            final_apply = true;   // x += d fused with the unpack below
            break;
        }
        dc_apply_kernel<<<gcells, kBlock, 0, stream>>>(c);
        if (cudaGetLastError() != cudaSuccess) { rc = TSE_ERR_LAUNCH; break; }
    }
    if (timing) {
        cudaEventDestroy(ev0);
        cudaEventDestroy(ev1);
    }
    if (rc != TSE_OK) return rc;
    dc_status_kernel<<<1, 1, 0, stream>>>(c.st, d_status);
    if (cudaGetLastError() != cudaSuccess) return TSE_ERR_LAUNCH;
    if (final_apply) {
        const long long nat = (long long)S.L.nx * S.L.ny * S.L.nz;
        dc_apply_unpack_kernel<<<(unsigned)((nat + kBlock - 1) / kBlock), kBlock, 0, stream>>>(X_out, c);
        return cudaGetLastError() == cudaSuccess ? TSE_OK : TSE_ERR_LAUNCH;
    }
    return launch_unpack(X_out, c.X[0], c.X[1], S.L, stream);
}

// ------------------------------------------- per-model steps, for batches
// The steps run_dc takes for one model, for drivers that interleave many
// models (tse_batch.cu): start (state record, zero margins, scaled records),
// residual (r', d = 0, x^2), halving (reset + new R terms + rescale), x += d,
// and finish (status record + natural-layout result).
template <class Form>
int dc_begin(const Form& F, const DcCtl& c, double dt, cudaStream_t stream) {
    float* dbase = c.D[0] - dc_margin(c.L);
    const long long dlen = dc_delta_len(c.L, c.Ncal);
    if (cudaMemsetAsync(dbase, 0, (size_t)2 * dlen * sizeof(float), stream) != cudaSuccess)
        return TSE_ERR_LAUNCH;
    dc_init_state_kernel<<<1, 1, 0, stream>>>(c.st, dt);
    if (cudaGetLastError() != cudaSuccess) return TSE_ERR_LAUNCH;
    const unsigned g = (unsigned)((2 * c.L.Nc + kBlock - 1) / kBlock);
    dc_scale_kernel<<<g, kBlock, 0, stream>>>(F, c);
    return cudaGetLastError() == cudaSuccess ? TSE_OK : TSE_ERR_LAUNCH;
}

template <class Form>
int dc_residual(const Form& F, const DcCtl& c, cudaStream_t stream) {
    const unsigned rb = (unsigned)res_blocks(c.L.Nc);
    dc_residual_kernel<<<rb, kBlock, 0, stream>>>(F, c);
    dc_x2_kernel<<<1, kBlock, 0, stream>>>(c, (int)rb);
    return cudaGetLastError() == cudaSuccess ? TSE_OK : TSE_ERR_LAUNCH;
}

template <class Form>
int dc_halve(const Form& F, const DcCtl& c, cudaStream_t stream) {
    const unsigned g = (unsigned)((2 * c.L.Nc + kBlock - 1) / kBlock);
    dc_halve_kernel<<<g, kBlock, 0, stream>>>(F, c);
    return cudaGetLastError() == cudaSuccess ? TSE_OK : TSE_ERR_LAUNCH;
}

int dc_apply(const DcCtl& c, cudaStream_t stream) {
    const unsigned g = (unsigned)((2 * c.L.Nc + kBlock - 1) / kBlock);
    dc_apply_kernel<<<g, kBlock, 0, stream>>>(c);
    return cudaGetLastError() == cudaSuccess ? TSE_OK : TSE_ERR_LAUNCH;
}

int dc_begin_fused(const DcCtl& c, double dt, int nparts, cudaStream_t stream) {
    float* dbase = c.D[0] - dc_margin(c.L);
    const long long dlen = dc_delta_len(c.L, c.Ncal);
    if (cudaMemsetAsync(dbase, 0, (size_t)2 * dlen * sizeof(float), stream) != cudaSuccess)
        return TSE_ERR_LAUNCH;
    dc_init_state_kernel<<<1, 1, 0, stream>>>(c.st, dt);
    dc_x2_kernel<<<1, kBlock, 0, stream>>>(c, nparts);
    return cudaGetLastError() == cudaSuccess ? TSE_OK : TSE_ERR_LAUNCH;
}

int dc_finish(const DcCtl& c, TseSolveStatus* d_status, double* X_out, cudaStream_t stream) {
    dc_status_kernel<<<1, 1, 0, stream>>>(c.st, d_status);
    if (cudaGetLastError() != cudaSuccess) return TSE_ERR_LAUNCH;
    return launch_unpack(X_out, c.X[0], c.X[1], c.L, stream);
}

template int dc_begin<PressureForm>(const PressureForm&, const DcCtl&, double, cudaStream_t);
template int dc_begin<TransportForm>(const TransportForm&, const DcCtl&, double, cudaStream_t);
template int dc_residual<PressureForm>(const PressureForm&, const DcCtl&, cudaStream_t);
template int dc_residual<TransportForm>(const TransportForm&, const DcCtl&, cudaStream_t);
template int dc_halve<PressureForm>(const PressureForm&, const DcCtl&, cudaStream_t);
template int dc_halve<TransportForm>(const TransportForm&, const DcCtl&, cudaStream_t);

}  // namespace tse

using namespace tse;

extern "C" int32_t tse_compute_P_dc(const TseGrid* grid, const TsePressureArgs* args,
                                    TseDcOptions* opts,
                                    TseSolveStatus* d_status, void* d_ws, size_t ws_bytes,
                                    void* stream_) {
    if (!grid || !args || !d_status || !d_ws) return TSE_ERR_ARG;
    if (grid->nx < 1 || grid->ny < 1 || grid->nz < 1 || args->max_it < 1) return TSE_ERR_ARG;
    if (!args->P || !args->Pn || !args->c_f || !args->nue || !args->rho_f || !args->phi ||
        !args->Kx || !args->Ky || !args->Kz || !args->c_r || !args->BP || !args->WP)
        return TSE_ERR_ARG;
    cudaStream_t stream = (cudaStream_t)stream_;
    PressureSetup S;
    int nparts = 0;
    int rc = setup_pressure_dc(grid, args, d_ws, ws_bytes, stream, S, &nparts);
    if (rc != TSE_OK) return rc;
    return run_dc(S, args->dt_P, args->inc_it, args->max_dt, args->min_dt, args->P_conv,
                  args->max_it, 1, 0, opts, args->SOR, PA_P, args->P, d_status, stream, nparts);
}

extern "C" int32_t tse_compute_C_dc(const TseGrid* grid, const TseSpeciesArgs* a,
                                    TseDcOptions* opts,
                                    TseSolveStatus* d_status, void* d_ws, size_t ws_bytes,
                                    void* stream_) {
    if (!grid || !a || !d_status || !d_ws) return TSE_ERR_ARG;
    if (grid->nx < 1 || grid->ny < 1 || grid->nz < 1 || a->max_it < 1) return TSE_ERR_ARG;
    if (!a->C || !a->D_fx || !a->D_fy || !a->D_fz || !a->phi || !a->rho_f || !a->qx || !a->qy ||
        !a->qz || !a->BC || !a->WC || !a->RC || !a->e || !a->l_l || !a->l_t)
        return TSE_ERR_ARG;
    cudaStream_t stream = (cudaStream_t)stream_;
    TransportSetup S;
    int nparts = 0;
    int rc = setup_species_dc(grid, a, d_ws, ws_bytes, stream, S, &nparts);
    if (rc != TSE_OK) return rc;
    return run_dc(S, a->dt, a->inc_it, a->max_dt, a->min_dt, a->conv, a->max_it, 0,
                  a->omega == 0.0, opts, a->SOR, TA_X, a->C, d_status, stream, nparts);
}

extern "C" int32_t tse_compute_T_dc(const TseGrid* grid, const TseHeatArgs* a,
                                    TseDcOptions* opts,
                                    TseSolveStatus* d_status, void* d_ws, size_t ws_bytes,
                                    void* stream_) {
    if (!grid || !a || !d_status || !d_ws) return TSE_ERR_ARG;
    if (grid->nx < 1 || grid->ny < 1 || grid->nz < 1 || a->max_it < 1) return TSE_ERR_ARG;
    if (!a->T || !a->l_f || !a->cp_f || !a->rho_f || !a->phi || !a->qx || !a->qy || !a->qz ||
        !a->BT || !a->WT || !a->e || !a->l_r || !a->rho_r || !a->cp_r || !a->l_l || !a->l_t)
        return TSE_ERR_ARG;
    cudaStream_t stream = (cudaStream_t)stream_;
    TransportSetup S;
    int nparts = 0;
    int rc = setup_heat_dc(grid, a, d_ws, ws_bytes, stream, S, &nparts);
    if (rc != TSE_OK) return rc;
    return run_dc(S, a->dt, a->inc_it, a->max_dt, a->min_dt, a->conv, a->max_it, 0,
                  a->omega == 0.0, opts, a->SOR, TA_X, a->T, d_status, stream, nparts);
}
