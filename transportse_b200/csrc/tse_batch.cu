// Batched mixed-precision solves of many independent models, in two forms.
//
// The fused form (the default; further down): every model's cells in one
// cooperative sweep sharing the colour-phase barriers, the loop around the
// sweeps (plan, events, residuals) run on the device as one CUDA graph.
//
// The cluster form (opts->max_blocks > 0): one thread-block cluster per model.
//
// For a small model the whole-GPU solve (tse_dc.cu) is bound by its two
// device-wide barriers per red+black iteration, not by memory: a 124K-cell
// model spends ~11 us per iteration.  Here a cluster of CTAs runs one model's
// entire solve -- coefficient scaling, FP64 residual, FP32 red-black sweeps
// with the reference's convergence test and dt control (tse.py:699-740 /
// 877-914 / 1045-1079), x += d, dt halving, and the unpack to the natural
// layout -- separating its phases with the hardware cluster barrier and
// reducing through distributed shared memory, then takes the next model from
// a device work queue.  Many clusters stream their models at once, so the
// batch together runs at memory rate.  Nothing waits on anything outside its
// own cluster (whose CTAs the hardware co-schedules), so the kernel has no
// spin-wait.
//
// The arithmetic is the whole-GPU form's (same per-cell relaxation, same
// correction-cycle and restart rules); only the grouping of the L2 partial
// sums differs.  Control flow depends only on values every CTA of a cluster
// computes identically (each CTA sums the same partials in the same order), so
// all CTAs take the same branches and pass the same barriers.
#include <cmath>
#include <vector>
#include <algorithm>
#include <atomic>
#include <chrono>
#include <mutex>
#include <type_traits>
#include <cooperative_groups.h>

#include "tse_dc.cuh"

namespace cg = cooperative_groups;

namespace tse {

constexpr int kBatchBlock = 256;
constexpr int kBatchMaxCluster = 16;

template <class Form>
struct BatchItem {
    Form F;
    DcCtl c;
    double dt;
    TseSolveStatus* status;
    double* X_out;
    long long cells;
    int nparts;   // > 0: the setup wrote the first cycle (records, r', x^2 partials)
};

struct BatchShared {
    double sh[kBatchBlock / 32];
    double slots[2 * kBatchMaxCluster];
    double bc[2];
    int model;
};

// Sums of NV values per thread over the cluster, identical in every CTA:
// block sums go to slot[rank] of CTA 0's array; after the barrier each CTA
// adds the slots in rank order.  The slots are rewritten only after a later
// cluster barrier, and bc after a later block barrier.
template <int NV>
__device__ __forceinline__ void cluster_sums(cg::cluster_group& cl, const double (&v)[NV],
                                             BatchShared& S, double (&out)[NV]) {
    const unsigned rank = cl.block_rank(), ncta = cl.num_blocks();
    double b[NV];
#pragma unroll
    for (int q = 0; q < NV; ++q) b[q] = block_sum<kBatchBlock>(v[q], S.sh);
    if (threadIdx.x == 0) {
        double* s0 = cl.map_shared_rank(S.slots, 0);
#pragma unroll
        for (int q = 0; q < NV; ++q) s0[NV * rank + q] = b[q];
    }
    cl.sync();
    if (threadIdx.x == 0) {
        const double* s0 = cl.map_shared_rank(S.slots, 0);
#pragma unroll
        for (int q = 0; q < NV; ++q) {
            double s = 0.0;
            for (unsigned r = 0; r < ncta; ++r) s = s + s0[NV * r + q];
            S.bc[q] = s;
        }
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < NV; ++q) out[q] = S.bc[q];
}

template <class Form>
__device__ void cluster_dc_solve(cg::cluster_group& cl, const BatchItem<Form>& it, BatchShared& S) {
    const Form& F = it.F;
    const DcCtl& c = it.c;
    const long long Nc = c.L.Nc, N = c.Ncal, SX = c.L.SX;
    const int H = c.L.H;
    const int lane = threadIdx.x & 31;
    const long long g = (long long)cl.block_rank() * kBatchBlock + threadIdx.x;
    const long long step = (long long)cl.num_blocks() * kBatchBlock;
    const bool leader = cl.block_rank() == 0 && threadIdx.x == 0;
    const float sor = c.sor;
    const long long G = dc_margin(c.L), dlen = dc_delta_len(c.L, N);
    TseSolveStatus* st = it.status;

    // every per-cell pass below maps cell m to the same thread, so a thread
    // rereads only its own writes of r', the records and d[m]; neighbour
    // values (d, x of the other colour) are read from L2 after a barrier
    for (int col = 0; col < 2; ++col) {
        float* d = c.D[col] - G;
        for (long long m = g; m < dlen; m += step) d[m] = 0.0f;
        for (long long m = g; m < Nc; m += step) scale_cell(F, c, col, m);
    }
    cl.sync();

    double t = 0.0, dt = it.dt, diff = 1e100;
    int num_it = 0, num_sub_it = 0, halvings = 0, converged = 0, nev = 0, cycles = 0;
    bool done = false;
    while (!done) {
        cycles += 1;
        // FP64 residual of the current iterate, d = 0
        double o2 = 0.0;
        for (int col = 0; col < 2; ++col) {
            const double* Xw = c.X[col];
            const double* Xo = c.X[1 - col];
            const uint8_t* msk = c.mask[col];
            float* Kc = c.K[col];
            float* Dc = c.D[col];
            for (long long m = g; m < Nc; m += step) {
                const uint8_t f = msk[m];
                const double x = Xw[m];
                o2 = o2 + x * x;
                float rp = 0.0f;
                if (f & F_ACTIVE) {
                    const double den = F.den(col, m);
                    const double r = F.sum(col, m, f, Xo) - den * x;
                    rp = (float)(r / den);
                }
                Kc[6 * N + m] = rp;
                Dc[m] = 0.0f;
            }
        }
        double x2;
        {
            const double v[1] = {o2};
            double out[1];
            cluster_sums<1>(cl, v, S, out);
            x2 = out[0];
        }

        int event = EV_CYCLE_END;
        bool halved = false;
        for (int inner = 0; inner < c.cycle; ++inner) {
            num_it += 1;
            num_sub_it += 1;
            const bool check = c.pressure_schedule ? (num_it < 50 || num_it % 10 == 0) : true;
            float d2 = 0.0f, dd = 0.0f;
            for (int col = 0; col < 2; ++col) {
                const float* __restrict__ Kc = c.K[col];
                float* dw = c.D[col];
                const float* dq = c.D[1 - col];
                const uint8_t* __restrict__ msk = c.mask[col];
                // trips counted per warp so every lane joins the shuffles
                for (long long w = g - lane; w < Nc; w += step) {
                    const long long ma = w + lane;
                    const bool va = ma < Nc;
                    const long long la = va ? ma : Nc - 1;
                    Cell a;
                    load_cell(a, Kc, dw, dq, msk, la, N, SX, H);
                    const float na = relax(a, dq, la, Nc, sor);
                    if (va) {
                        dw[ma] = na;
                        const float ch = na - a.old;
                        d2 = fmaf(ch, ch, d2);
                        dd = fmaf(na, na, dd);
                    }
                }
                // at a check, the reduction's barrier ends the black phase
                if (col == 0 || !check) cl.sync();
            }
            diff = 1e100;
            bool refresh = false;
            if (check) {
                const double v[2] = {(double)d2, (double)dd};
                double out[2];
                cluster_sums<2>(cl, v, S, out);
                const double l2 = sqrt(out[0]) / sqrt(x2 + 1e-200);
                diff = (l2 != l2) ? 1.0 : l2;
                refresh = sqrt(out[0]) < kRefresh * sqrt(out[1]);
            }
            if (diff < c.conv || c.stop_on_first) {
                t += dt;
                if (num_sub_it < c.max_it / 2.0) dt = pymin(dt * c.inc_it, c.max_dt);
                event = EV_CONVERGED;
                break;
            }
            if (num_sub_it >= c.max_it) {
                if (leader && nev < 8) {
                    st->ev_it[nev] = num_it;
                    st->ev_dt[nev] = dt;
                    st->ev_diff[nev] = diff;
                }
                nev += 1;
                dt = dt / 2;
                num_sub_it = 0;
                halvings += 1;
                halved = true;
            }
            if (dt <= c.min_dt) { event = halved ? EV_STOP_HALVED : EV_STOP; break; }
            if (halved) { event = EV_HALVE; break; }
            if (refresh) { event = EV_REFRESH; break; }
        }
        if (event == EV_HALVE || event == EV_STOP_HALVED) {
            // x = Xn, new R terms, rescaled coefficients (tse.py:733-738)
            for (int col = 0; col < 2; ++col)
                for (long long m = g; m < Nc; m += step) {
                    F.reassemble(col, m, dt);
                    scale_cell(F, c, col, m);
                }
            cl.sync();
            if (event == EV_STOP_HALVED) done = true;
            continue;
        }
        for (int col = 0; col < 2; ++col) {
            double* Xw = c.X[col];
            const float* dw = c.D[col];
            const uint8_t* msk = c.mask[col];
            for (long long m = g; m < Nc; m += step)
                if (msk[m] & F_ACTIVE) Xw[m] = Xw[m] + (double)dw[m];
        }
        cl.sync();
        if (event == EV_CONVERGED) converged = 1;
        if (event == EV_CONVERGED || event == EV_STOP) done = true;
    }
    if (leader) {
        st->t = t;
        st->dt = dt;
        st->diff = diff;
        st->converged = converged;
        st->num_it = num_it;
        st->num_sub_it = num_sub_it;
        st->halvings = halvings;
        st->error = TSE_STATUS_OK;
        st->n_events = nev < 8 ? nev : 8;
        st->cycles = cycles;
    }
    // compact colour arrays -> natural (nx, ny, nz); the last barrier above
    // made every x visible
    const Layout& L = c.L;
    const long long nat = (long long)L.nx * L.ny * L.nz;
    for (long long q = g; q < nat; q += step) {
        int i, j, k;
        long long row;
        grid_coords(q, L.ny, L.nz, i, j, k, row);
        const long long m = (row * L.nzp + k) >> 1;
        it.X_out[q] = ((i + j + k) & 1) ? __ldcg(c.X[1] + m) : __ldcg(c.X[0] + m);
    }
}

template <class Form>
__global__ void __launch_bounds__(kBatchBlock, 4) batch_dc_kernel(const BatchItem<Form>* items, int n,
                                                                  int* queue) {
    __shared__ BatchShared S;
    cg::cluster_group cl = cg::this_cluster();
    for (;;) {
        if (cl.block_rank() == 0 && threadIdx.x == 0) S.model = atomicAdd(queue, 1);
        cl.sync();
        const int q = *cl.map_shared_rank(&S.model, 0);
        // no CTA leaves, or lets CTA 0 rewrite the index, while another may
        // still read it
        cl.sync();
        if (q >= n) return;
        cluster_dc_solve(cl, items[q], S);
    }
}

template <class Form>
static int launch_batch(std::vector<BatchItem<Form>>& items, const TseDcOptions* opts, void* d_ws,
                        size_t ws_bytes, cudaStream_t stream) {
    const int n = (int)items.size();
    const size_t item_bytes = align256(sizeof(BatchItem<Form>) * n);
    if (item_bytes + 256 > ws_bytes) return TSE_ERR_WORKSPACE;
    // largest models first, so the longest solves start at once
    std::stable_sort(items.begin(), items.end(),
                     [](const BatchItem<Form>& a, const BatchItem<Form>& b) { return a.cells > b.cells; });
    BatchItem<Form>* d_items = (BatchItem<Form>*)d_ws;
    int* queue = (int*)((char*)d_ws + item_bytes);
    // pageable source: the copy is staged before this call returns
    if (cudaMemcpyAsync(d_items, items.data(), sizeof(BatchItem<Form>) * n, cudaMemcpyHostToDevice,
                        stream) != cudaSuccess ||
        cudaMemsetAsync(queue, 0, sizeof(int), stream) != cudaSuccess)
        return TSE_ERR_LAUNCH;
    int cs = (opts && opts->max_blocks > 0) ? opts->max_blocks : 8;
    if (cs > kBatchMaxCluster) cs = kBatchMaxCluster;
    if (cs > 8 && cudaFuncSetAttribute(batch_dc_kernel<Form>,
                                       cudaFuncAttributeNonPortableClusterSizeAllowed, 1) != cudaSuccess)
        return TSE_ERR_LAUNCH;
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = (unsigned)cs;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.blockDim = dim3(kBatchBlock);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = stream;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    cfg.gridDim = dim3((unsigned)cs);
    int resident = 0;
    if (cudaOccupancyMaxActiveClusters(&resident, batch_dc_kernel<Form>, &cfg) != cudaSuccess ||
        resident < 1)
        return TSE_ERR_LAUNCH;
    const int clusters = n < resident ? n : resident;
    cfg.gridDim = dim3((unsigned)(clusters * cs));
    if (cudaLaunchKernelEx(&cfg, batch_dc_kernel<Form>, (const BatchItem<Form>*)d_items, n, queue) !=
        cudaSuccess)
        return TSE_ERR_LAUNCH;
    return cudaGetLastError() == cudaSuccess ? TSE_OK : TSE_ERR_LAUNCH;
}

static void fill_ctl(DcCtl& c, double inc_it, double max_dt, double min_dt, double conv, int max_it,
                     int pressure_schedule, int stop_on_first, const TseDcOptions* opts, double sor) {
    c.inc_it = inc_it;
    c.max_dt = max_dt;
    c.min_dt = min_dt;
    c.conv = conv;
    c.max_it = max_it;
    c.pressure_schedule = pressure_schedule;
    c.stop_on_first = stop_on_first;
    c.cycle = (opts && opts->cycle > 0) ? opts->cycle : 256;
    c.sor = (float)sor;
}

// NaN in dt or min_dt would keep a non-converging solve halving forever
static bool finite_dt(double dt, double min_dt) { return std::isfinite(dt) && std::isfinite(min_dt); }

// ====================================================== fused batched sweeps
// Pipelines of the fused sweep, as in the single-model staged sweep: two per
// block, one block per SM, up to 4 stages a ring.  (Measured against one
// pipeline and two blocks per SM: 24.9 against 23.9 G cell-updates/s on the
// serving workload, 99 against 102 on the 48-model ensemble -- within the
// runs' spread.)
constexpr int kFusedPipes = 2;
constexpr int kFusedMaxRing = 4;

// All models of a batch in one cooperative sweep: the chunks (kTmaChunk
// cells) of every active model form one table, interleaved over the blocks,
// and every block runs the staged producer/consumer pipeline of
// dc_sweep_tma_kernel over it, each chunk copied from its own model's arrays.
// The models share the colour-phase barriers, so a small model costs its
// bytes, not two device-wide barriers per iteration; a model that finishes
// drops out of the table at the next launch and the rest keep the GPU.
//
// All active models advance one iteration per global iteration, so they
// share the iteration count and the check schedule (pressure: every
// iteration below 50, then every 10th; transport: every iteration).  At a
// check each chunk stores its two colours' sums; after the barrier one block
// per model adds its chunks in order and takes that model's decision
// (converged, dt halving, stop, refresh, cycle end: the order of
// dc_sweep_kernel); any event ends the launch after one more barrier.  A
// model's cycle end and dt halving fall on iterations known in advance, so
// the host bounds each launch by the nearest one and the decisions run there
// too.  Between launches the host finishes each model's event with the
// per-model steps of tse_dc.cu (x += d, residual, halving).
struct FusedItem {
    DcCtl c;
    long long cfirst, nchunks;   // this model's chunks in the table
    int inner;                   // iterations since its last residual, at launch
    int age0;                    // its own iteration count at launch (models
                                 // admitted later count from their admission)
};

struct FusedChunk {
    long long m0;
    int item;
    int pad;
};

struct FusedArgs {
    const FusedItem* items;
    int nitems;
    const FusedChunk* chunks;
    long long nchunks;
    double2* cpart;      // per chunk, colour and consumer warp: (sum of change^2, sum of d^2)
    int* any_event;
    GridBarrier* bar;
    int g_max;           // iterations this launch runs at most
    int num_it0;         // the models' iteration count at launch
    int pressure_schedule;
    // the pressure check schedule (every iteration below 50, then every 10th)
    // of the youngest model and of every model's phase: at launch iteration
    // g some model checks if young + g < 50 or bit g % 10 of mask10 is set
    int young;
    int mask10;
};

// the check schedule of a model of age a (its own iterations) under the
// pressure schedule (tse.py:719-723) or the transport one (every iteration)
__device__ __forceinline__ bool model_checks(int pressure_schedule, int a) {
    return pressure_schedule ? (a < 50 || a % 10 == 0) : true;
}

// one model's decision after global iteration g (thread 0 of its block)
__device__ void fused_decide(const FusedItem& I, int g, int num_it, bool check, double s1, double s3,
                             int* any_event) {
    const DcCtl& c = I.c;
    DcState* st = c.st;
    double t = st->t, dt = st->dt;
    int sub = st->num_sub_it + (num_it - st->num_it);
    const int inner = I.inner + g;
    double diff = 1e100;
    bool refresh = false;
    if (check) {
        const double l2 = sqrt(s1) / sqrt(st->x2 + 1e-200);
        diff = (l2 != l2) ? 1.0 : l2;
        refresh = sqrt(s1) < kRefresh * sqrt(s3);
    }
    int ev = EV_NONE;
    if (diff < c.conv || c.stop_on_first) {
        t += dt;
        if (sub < c.max_it / 2.0) dt = pymin(dt * c.inc_it, c.max_dt);
        ev = EV_CONVERGED;
        st->converged = 1;
    } else {
        bool halved = false;
        if (sub >= c.max_it) {
            if (st->nev < 8) {
                st->ev_it[st->nev] = num_it;
                st->ev_dt[st->nev] = dt;
                st->ev_diff[st->nev] = diff;
            }
            st->nev += 1;
            dt = dt / 2;
            sub = 0;
            st->halvings += 1;
            halved = true;
        }
        if (dt <= c.min_dt) ev = halved ? EV_STOP_HALVED : EV_STOP;
        else if (halved) ev = EV_HALVE;
        else if (refresh) ev = EV_REFRESH;
        else if (inner >= c.cycle) ev = EV_CYCLE_END;
    }
    st->t = t;
    st->dt = dt;
    st->diff = diff;
    st->num_it = num_it;
    st->num_sub_it = sub;
    st->event = ev;
    if (ev != EV_NONE) atomicExch(any_event, 1);
}

// What a consumer group needs of a staged chunk besides its copied arrays,
// written by the producer into the stage's header before the copies are
// issued (the stage's full barrier publishes it with them), so consumers
// read no table or model record from global memory
struct ChunkHdr {
    long long m0, SX, Nc;
    float* out;
    int H;
    float sor;
};

template <int RING, int PIPES>
__device__ __forceinline__ void fused_sweep_body(const FusedArgs& A, const TmaStage& T) {
    constexpr int kPipes = PIPES;
    constexpr int kFusedThreads = kTmaConsumers + 32 * PIPES;
    static_assert((kTmaConsumers / kTmaGroup) % PIPES == 0, "every pipeline has its own consumer groups");
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ __align__(8) uint64_t full[RING * PIPES];
    __shared__ __align__(8) uint64_t empty[RING * PIPES];
    __shared__ ChunkHdr hdr[RING * PIPES];
    __shared__ double sh[kFusedThreads / 32];
    __shared__ int s_err;
    const unsigned nb = gridDim.x, b = blockIdx.x;
    const int tid = threadIdx.x;
    const int warp = tid >> 5, lane = tid & 31;
    const bool producer = warp >= kTmaConsumers / 32;
    const int group = tid / kTmaGroup;                  // consumers: 0 or 1
    const int gt = tid & (kTmaGroup - 1);
    // pipelines as in dc_sweep_tma_kernel: producer warp + ring + groups
    const int pipe = producer ? warp - kTmaConsumers / 32 : group % kPipes;
    const int grank = group / kPipes;
    constexpr int kGroupsPerPipe = (kTmaConsumers / kTmaGroup) / kPipes;
    const unsigned ring0 = (unsigned)pipe * RING;
    const long long C = kTmaChunk;
    const long long mine = A.nchunks > (long long)b ? (A.nchunks - 1 - b) / nb + 1 : 0;
    const long long pmine = mine > pipe ? (mine - 1 - pipe) / kPipes + 1 : 0;
    const uint64_t keep = l2_evict_last();
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
    unsigned uses = 0, issued = 0;
    unsigned bars = 0;   // device-wide barriers passed (A.bar->count, zeroed per launch)
    bool ok = true;
    for (int g = 1; g <= A.g_max && ok; ++g) {
        // whether any model checks at this iteration (the chunks then store
        // their sums; each model's decision uses its own schedule)
        const bool check = !A.pressure_schedule || A.young + g < 50 || ((A.mask10 >> (g % 10)) & 1);
        const bool last = g == A.g_max;
        for (int col = 0; col < 2 && ok; ++col) {
            if (producer) {
                // the warp fetches the table entries of its next 32 chunks at
                // once (one memory round trip per 32 chunks, not per chunk);
                // lane 0 takes each from its lane, reads the chunk's model
                // record (cached after its first chunk), writes the consumers'
                // header and issues the copies
                if (lane == 0) fence_proxy_async();
                bool pok = true;
                for (long long j0 = 0; j0 < pmine && pok; j0 += 32) {
                    FusedChunk mine_ch = {0, 0, 0};
                    if (j0 + lane < pmine) mine_ch = A.chunks[b + (pipe + (j0 + lane) * kPipes) * nb];
                    const int nj = (int)((pmine - j0) < 32 ? (pmine - j0) : 32);
                    for (int t = 0; t < nj; ++t) {
                        const long long m0 = __shfl_sync(0xffffffffu, mine_ch.m0, t);
                        const int item = __shfl_sync(0xffffffffu, mine_ch.item, t);
                        int okw = 1;
                        if (lane == 0) {
                            const unsigned s = ring0 + issued % RING;
                            if (issued >= (unsigned)RING &&
                                !mbar_wait_flag(&empty[s], (issued / RING - 1) & 1u, err)) {
                                okw = 0;
                            } else {
                                const DcCtl& c = A.items[item].c;
                                const long long cnt = (c.Ncal - m0) < C ? (c.Ncal - m0) : C;
                                unsigned char* stg = smem + (size_t)s * T.bytes;
                                ChunkHdr h;
                                h.m0 = m0;
                                h.SX = c.L.SX;
                                h.Nc = c.L.Nc;
                                h.out = c.D[col] + m0;
                                h.H = c.L.H;
                                h.sor = c.sor;
                                hdr[s] = h;
                                tma_issue_own_n(c.Ncal, T, stg, &full[s], c.K[col], c.D[col], c.mask[col], m0,
                                                cnt);
                                tma_issue_windows_n(h.SX, h.H, T, stg, &full[s], c.D[1 - col], m0);
                                ++issued;
                            }
                        }
                        if (!__shfl_sync(0xffffffffu, okw, 0)) {
                            pok = false;
                            break;
                        }
                    }
                }
                // lane 0 counted the copies it issued; the other lanes follow
                issued = __shfl_sync(0xffffffffu, issued, 0);
            } else {
                for (long long j = grank; j < pmine; j += kGroupsPerPipe) {
                    const unsigned u = uses + (unsigned)j;
                    const unsigned s = ring0 + u % RING;
                    // warp-uniform: lane 0 waits, the warp follows its outcome,
                    // then every lane observes the completed phase (acquire)
                    int okw = 1;
                    if (lane == 0) okw = mbar_wait_flag(&full[s], (u / RING) & 1u, err);
                    if (!__shfl_sync(0xffffffffu, okw, 0)) break;
                    mbar_try_wait(&full[s], (u / RING) & 1u);
                    const unsigned char* stg = smem + (size_t)s * T.bytes;
                    const long long q = b + (pipe + j * kPipes) * nb;
                    const ChunkHdr h = hdr[s];
                    const long long m0 = h.m0, SX = h.SX;
                    const int H = h.H;
                    const float sor = h.sor;
                    const int nval = (int)((h.Nc - m0) < C ? (h.Nc - m0) : C);
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
                    float* out = h.out;
                    float d2 = 0.0f, dd = 0.0f;
#pragma unroll
                    for (int r = 0; r < kTmaCellsPerThread; ++r) {
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
                            const float ch2 = na - old;
                            d2 = fmaf(ch2, ch2, d2);
                            dd = fmaf(na, na, dd);
                        }
                    }
                    // the warp's reads of the stage are done: release it
                    __syncwarp();
                    if (lane == 0) mbar_arrive(&empty[s]);
                    if (check) {
                        // this warp's sums for the chunk (the model's
                        // decision adds them in a fixed order)
                        double a = d2, e = dd;
#pragma unroll
                        for (int o = 16; o > 0; o >>= 1) {
                            a = a + __shfl_down_sync(0xffffffffu, a, o);
                            e = e + __shfl_down_sync(0xffffffffu, e, o);
                        }
                        if (lane == 0) A.cpart[(2 * q + col) * 4 + (warp & 3)] = make_double2(a, e);
                    }
                }
            }
            uses += (unsigned)pmine;
            fence_proxy_async();
            __syncthreads();
            if (*err) { ok = false; break; }
            ok = count_sync(&A.bar->count, ++bars * nb, A.bar);
        }
        if (!ok) break;
        if (check || last) {
            for (int it = (int)b; it < A.nitems; it += (int)nb) {
                const FusedItem& I = A.items[it];
                const int age = I.age0 + g;
                const bool mcheck = check && model_checks(A.pressure_schedule, age);
                double s1 = 0.0, s3 = 0.0;
                if (mcheck)
                    for (long long k = tid; k < I.nchunks; k += blockDim.x) {
                        const double2* pk = A.cpart + 8 * (I.cfirst + k);   // 2 colours x 4 warps
#pragma unroll
                        for (int j = 0; j < 8; ++j) {
                            const double2 pj = __ldcg(pk + j);
                            s1 = s1 + pj.x;
                            s3 = s3 + pj.y;
                        }
                    }
                s1 = block_sum<kFusedThreads>(s1, sh);
                s3 = block_sum<kFusedThreads>(s3, sh);
                if (tid == 0) fused_decide(I, g, age, mcheck, s1, s3, A.any_event);
                __syncthreads();
            }
            ok = count_sync(&A.bar->count, ++bars * nb, A.bar);
            if (ok && *(volatile int*)A.any_event) break;
        }
    }
    if (!ok && producer && lane == 0) {
        // the last copies issued into each stage land before the block's
        // shared memory is released (bounded waits, flag ignored)
        atomicExch(&A.bar->error, 1);
        const unsigned first = issued > (unsigned)RING ? issued - RING : 0u;
        for (unsigned v = first; v < issued; ++v)
            mbar_wait_bounded(&full[ring0 + v % RING], (v / RING) & 1u);
    }
    if (!ok && b == 0 && tid == 0)
        for (int it = 0; it < A.nitems; ++it) A.items[it].c.st->event = EV_ERROR;
}

template <int RING, int PIPES>
__global__ void __launch_bounds__(kTmaConsumers + 32 * PIPES, PIPES == 1 ? 2 : 1)
    fused_sweep_kernel(FusedArgs A, TmaStage T) {
    fused_sweep_body<RING, PIPES>(A, T);
}

struct FusedCtl;
__device__ void fused_add_sweep_ns(FusedCtl* ctl, unsigned long long ns);

// the same with its arguments in device memory, written by the plan kernel
// of the device-driven loop; block 0 adds the launch's duration (global
// timer, from its start to after the launch's last device-wide barrier) to
// the loop's sweep time, the kernel's own time inside the graph, where no
// host event can bracket it
template <int RING, int PIPES>
__global__ void __launch_bounds__(kTmaConsumers + 32 * PIPES, PIPES == 1 ? 2 : 1)
    fused_sweep_dev_kernel(const FusedArgs* Ad, TmaStage T, FusedCtl* ctl) {
    const bool clock = blockIdx.x == 0 && threadIdx.x == 0;
    const uint64_t t0 = clock ? globaltimer() : 0;
    const FusedArgs A = *Ad;
    fused_sweep_body<RING, PIPES>(A, T);
    if (clock) fused_add_sweep_ns(ctl, globaltimer() - t0);
}

__global__ void fused_gather_kernel(const FusedItem* items, int n, DcState* out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = *items[i].c.st;
}

// dynamic shared memory ceiling: the device's per-block opt-in limit less the
// kernel's static arrays and a margin
static size_t fused_max_smem() {
    int dev = 0, optin = 0;
    cudaGetDevice(&dev);
    if (cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return optin > 2048 ? (size_t)optin - 2048 : 0;
}

// bytes the device-driven loop adds to the batch workspace (defined with it)
static size_t fused_loop_bytes(int n);

// bytes of the fused form's batch workspace for n models of `cells` cells in all
static size_t fused_ws_bytes(int n, long long cells) {
    const size_t nch = (size_t)(cells / kTmaChunk) + (size_t)n + 1;
    return align256(sizeof(FusedItem) * n) + align256(sizeof(FusedChunk) * nch) +
           align256(sizeof(double2) * 8 * nch) + align256(sizeof(DcState) * n) + 256 +
           align256(sizeof(GridBarrier)) + 256 + fused_loop_bytes(n);
}

template <class Form>
static int run_fused(std::vector<BatchItem<Form>>& v, TseDcOptions* opts, void* d_ws, size_t ws_bytes,
                     cudaStream_t stream) {
    const int n = (int)v.size();
    long long cells = 0;
    int Hmax = 0;
    for (auto& it : v) {
        cells += (long long)it.c.L.nx * it.c.L.ny * it.c.L.nz;
        Hmax = it.c.L.H > Hmax ? it.c.L.H : Hmax;
    }
    if (fused_ws_bytes(n, cells) > ws_bytes) return TSE_ERR_WORKSPACE;
    TmaStage T = tma_stage(Hmax);
    // as many stages as fit (up to 4 a ring, an equal ring per pipeline); one
    // instantiation per ring length
    int dev = 0, sms = 0, per_sm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int pipes = kFusedPipes;
    const int avail =
        (int)std::min<size_t>((size_t)(kFusedMaxRing * pipes), fused_max_smem() / (size_t)T.bytes);
    const int ring = avail / pipes;
    if (ring < 2) return TSE_ERR_ARG;
    const void* kernel = ring == 2   ? (const void*)fused_sweep_kernel<2, kFusedPipes>
                         : ring == 3 ? (const void*)fused_sweep_kernel<3, kFusedPipes>
                                     : (const void*)fused_sweep_kernel<4, kFusedPipes>;
    const int fused_threads = kTmaConsumers + 32 * pipes;
    T.stages = ring * pipes;
    const size_t smem = (size_t)T.stages * T.bytes;
    // carve the batch workspace
    const size_t nch_max = (size_t)(cells / kTmaChunk) + (size_t)n + 1;
    char* p = (char*)d_ws;
    FusedItem* d_items = (FusedItem*)p;
    p += align256(sizeof(FusedItem) * n);
    FusedChunk* d_chunks = (FusedChunk*)p;
    p += align256(sizeof(FusedChunk) * nch_max);
    double2* d_cpart = (double2*)p;
    p += align256(sizeof(double2) * 8 * nch_max);
    DcState* d_states = (DcState*)p;
    p += align256(sizeof(DcState) * n);
    int* d_any = (int*)p;
    p += 256;
    GridBarrier* d_bar = (GridBarrier*)p;

    if (cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)fused_max_smem()) !=
            cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, fused_threads, smem) != cudaSuccess ||
        per_sm < 1)
        return TSE_ERR_LAUNCH;

    // every model: state, scaled records, first residual (written by a fused
    // setup, which leaves the x^2 total)
    for (auto& it : v) {
        int rc = it.nparts > 0 ? dc_begin_fused(it.c, it.dt, it.nparts, stream)
                               : dc_begin(it.F, it.c, it.dt, stream);
        if (rc == TSE_OK && it.nparts == 0) rc = dc_residual(it.F, it.c, stream);
        if (rc != TSE_OK) return rc;
    }
    std::vector<int> active(n), inner(n, 0);
    for (int i = 0; i < n; ++i) active[i] = i;
    std::vector<DcState> st(n);
    for (int i = 0; i < n; ++i) {
        memset(&st[i], 0, sizeof(DcState));
        st[i].dt = v[i].dt;
    }
    int num_it = 0;
    int rc = TSE_OK;
    // optional: launches, global iterations and event time of the fused sweeps
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
    // the host loop synchronises every launch: its wall time is the loop's
    const auto loop_t0 = std::chrono::steady_clock::now();
    std::vector<FusedItem> hitems;
    std::vector<FusedChunk> hchunks;
    std::vector<DcState> got;
    while (!active.empty()) {
        // the nearest cycle end or dt halving among the active models
        int g_max = 1 << 30;
        for (int i : active) {
            const DcCtl& c = v[i].c;
            int lim = c.cycle - inner[i];
            const int h = c.max_it - st[i].num_sub_it;
            lim = h < lim ? h : lim;
            if (st[i].dt <= c.min_dt) lim = 1;
            g_max = lim < g_max ? lim : g_max;
        }
        if (g_max < 1) g_max = 1;
        hitems.clear();
        hchunks.clear();
        for (int k = 0; k < (int)active.size(); ++k) {
            const int i = active[k];
            FusedItem I;
            memset(&I, 0, sizeof(I));
            I.c = v[i].c;
            I.cfirst = (long long)hchunks.size();
            const long long nc = (v[i].c.L.Nc + kTmaChunk - 1) / kTmaChunk;
            I.nchunks = nc;
            I.inner = inner[i];
            I.age0 = st[i].num_it;
            for (long long q = 0; q < nc; ++q) hchunks.push_back(FusedChunk{q * kTmaChunk, k, 0});
            hitems.push_back(I);
        }
        const int na = (int)hitems.size();
        const long long nch = (long long)hchunks.size();
        FusedArgs A;
        A.items = d_items;
        A.nitems = na;
        A.chunks = d_chunks;
        A.nchunks = nch;
        A.cpart = d_cpart;
        A.any_event = d_any;
        A.bar = d_bar;
        A.g_max = g_max;
        A.num_it0 = num_it;
        A.pressure_schedule = v[0].c.pressure_schedule;
        // every model of the host loop starts together: one age, one phase
        A.young = num_it;
        A.mask10 = 1 << ((10 - num_it % 10) % 10);
        long long nb = (long long)sms * per_sm;
        if (nb > nch) nb = nch;
        if (nb > kMaxBlocks) nb = kMaxBlocks;
        // pageable sources: staged before the calls return
        if (cudaMemcpyAsync(d_items, hitems.data(), sizeof(FusedItem) * na, cudaMemcpyHostToDevice,
                            stream) != cudaSuccess ||
            cudaMemcpyAsync(d_chunks, hchunks.data(), sizeof(FusedChunk) * nch, cudaMemcpyHostToDevice,
                            stream) != cudaSuccess ||
            cudaMemsetAsync(d_any, 0, sizeof(int), stream) != cudaSuccess ||
            cudaMemsetAsync(d_bar, 0, sizeof(GridBarrier), stream) != cudaSuccess) {
            rc = TSE_ERR_LAUNCH;
            break;
        }
        void* args[] = {(void*)&A, (void*)&T};
        if (timing) cudaEventRecord(ev0, stream);
        if (cudaLaunchCooperativeKernel(kernel, dim3((unsigned)nb), dim3(fused_threads), args, smem,
                                        stream) != cudaSuccess) {
            rc = TSE_ERR_LAUNCH;
            break;
        }
        if (timing) cudaEventRecord(ev1, stream);
        fused_gather_kernel<<<(na + 127) / 128, 128, 0, stream>>>(d_items, na, d_states);
        got.resize(na);
        if (cudaGetLastError() != cudaSuccess ||
            cudaMemcpyAsync(got.data(), d_states, sizeof(DcState) * na, cudaMemcpyDeviceToHost,
                            stream) != cudaSuccess ||
            cudaStreamSynchronize(stream) != cudaSuccess) {
            rc = TSE_ERR_LAUNCH;
            break;
        }
        const int ran = got[0].num_it - num_it;
        num_it = got[0].num_it;
        if (timing) {
            float ms = 0.0f;
            cudaEventElapsedTime(&ms, ev0, ev1);
            opts->sweep_launches += 1;
            opts->sweep_iterations += ran;
            opts->sweep_ms += ms;
        }
        std::vector<int> next;
        bool failed = false;
        for (int k = 0; k < na; ++k) {
            const int i = active[k];
            st[i] = got[k];
            inner[i] += ran;
            const int ev = got[k].event;
            int r = TSE_OK;
            bool done = false;
            switch (ev) {
                case EV_NONE: break;
                case EV_CONVERGED:
                case EV_STOP: r = dc_apply(v[i].c, stream); done = true; break;
                case EV_REFRESH:
                case EV_CYCLE_END:
                    r = dc_apply(v[i].c, stream);
                    if (r == TSE_OK) r = dc_residual(v[i].F, v[i].c, stream);
                    inner[i] = 0;
                    break;
                case EV_HALVE:
                    r = dc_halve(v[i].F, v[i].c, stream);
                    if (r == TSE_OK) r = dc_residual(v[i].F, v[i].c, stream);
                    inner[i] = 0;
                    break;
                case EV_STOP_HALVED: r = dc_halve(v[i].F, v[i].c, stream); done = true; break;
                default: failed = true; done = true; break;   // EV_ERROR: reported per model
            }
            if (r != TSE_OK) rc = r;
            if (!done) next.push_back(i);
        }
        if (rc != TSE_OK) break;
        if (failed) {
            active.clear();
            break;
        }
        active.swap(next);
    }
    if (timing) {
        opts->loop_ms =
            std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - loop_t0).count();
        cudaEventDestroy(ev0);
        cudaEventDestroy(ev1);
    }
    // status records and results of every model (a failed launch leaves
    // the models' state records as they were)
    for (auto& it : v) {
        const int r = dc_finish(it.c, it.status, it.X_out, stream);
        if (rc == TSE_OK) rc = r;
    }
    return rc;
}

// ------------------------------------------------ device-driven fused solves
// run_fused's host loop reads every model's state after each sweep launch and
// queues the models' next steps.  Here the same loop runs on the device, as a
// CUDA graph holding one conditional WHILE node whose body is
//   plan -> chunk table -> fused sweep -> events -> x += d / dt halving
//        -> residual -> x^2
// so the host launches the graph once per batch solve and reads one small
// record when it ends.  Each step computes what run_fused's host code and
// its per-model kernels compute, in the same order and blocking -- a model's
// residual runs as the same res_blocks(Nc) blocks of residual_block_cells, its
// x^2 is summed as dc_x2_kernel sums it -- so the results are run_fused's bit
// for bit.  The body runs at most kGraphMaxRuns times per graph launch (the
// host relaunches the graph while models remain), so no launch can loop on
// the device without end.

struct FusedCtl {
    int n;                   // models of the batch
    int nactive;             // models solving or waiting, after the last events pass
    int num_it;              // the models' global iteration count
    int failed;              // a sweep reported EV_ERROR
    int runs;                // loop-body runs in the current graph launch
    int launches;            // sweep launches over the whole solve
    long long iterations;    // global iterations over the whole solve
    long long resid_total;   // residual blocks of the current body run, all models
    unsigned long long sweep_ns;   // summed duration of the sweep launches
    long long budget;        // cells (both colours) active at once; 0: every model
    int max_runs;            // loop-body runs per graph launch
    int pad;
};

__device__ void fused_add_sweep_ns(FusedCtl* ctl, unsigned long long ns) { ctl->sweep_ns += ns; }

// one model of the device-driven loop
struct FusedModel {
    DcCtl c;
    long long nchunks;       // ceil(Nc / kTmaChunk)
    int active;              // 1 while solving
    int inner;               // iterations since the model's last residual
    int waiting;             // 1 until admitted (a cell budget holds it back)
    int pad;
};

enum : int { ACT_APPLY = 1, ACT_HALVE = 2, ACT_RESID = 4 };
constexpr int kGraphMaxRuns = 4096;
constexpr int kPlanThreads = 1024;

// inclusive block-wide prefix sum; *total gets the block's sum
template <typename V>
__device__ V block_inclusive_scan(V v, V* sh, V* total) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const V u = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v += u;
    }
    if (lane == 31) sh[w] = v;
    __syncthreads();
    if (w == 0) {
        V x = lane < nw ? sh[lane] : V(0);
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const V u = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += u;
        }
        sh[lane] = x;
    }
    __syncthreads();
    if (w > 0) v += sh[w - 1];
    *total = sh[nw - 1];
    __syncthreads();
    return v;
}

// Admission, then the active models in index order, their iteration limit
// for the launch (run_fused's g_max), their chunk ranges and the sweep's
// arguments.  Admission (a cell budget): waiting models join in index order
// while the active cells stay within ctl->budget -- the first waiting model
// always, when none is active -- so models that converge early hand their
// share of the GPU to the next ones instead of leaving it idle until the
// slowest model of the batch is done.  An admitted model counts its own
// iterations from 0 (its state record is its solve's from the start), so
// its iterations, checks and decisions are those of its solve alone.  Under
// the pressure schedule (checks every 10th of a model's own iterations past
// its 50th) models join only on multiples of 10 of the loop's count -- a
// launch ends there while models wait and room is free -- so the running
// models share one check phase and most iterations need no check at all.
__global__ void __launch_bounds__(kPlanThreads) fused_plan_kernel(const FusedCtl* ctl, FusedModel* models,
                                                                  FusedItem* items, int* idx, FusedArgs* args,
                                                                  FusedChunk* chunks, double2* cpart,
                                                                  int* any_event, GridBarrier* bar) {
    __shared__ long long sh_ll[32];
    __shared__ int sh_i[32];
    __shared__ int s_gmax, s_base_k, s_young, s_mask, s_cap;
    __shared__ long long s_base_ch, s_active_cells, s_base_w, s_waiting_cells;
    const int n = ctl->n;
    if (threadIdx.x == 0) {
        s_gmax = 1 << 30;
        s_base_k = 0;
        s_base_ch = 0;
        s_active_cells = 0;
        s_base_w = 0;
        s_young = 1 << 30;
        s_mask = 0;
        s_cap = 1 << 30;
        s_waiting_cells = 0;
    }
    __syncthreads();
    if (ctl->budget > 0) {
        // cells of the active models and of the waiting ones
        for (int base = 0; base < n; base += kPlanThreads) {
            const int i = base + threadIdx.x;
            const long long cells = (i < n && models[i].active) ? 2 * models[i].c.L.Nc : 0;
            const long long wcells = (i < n && models[i].waiting) ? 2 * models[i].c.L.Nc : 0;
            long long tot, wtot;
            block_inclusive_scan<long long>(cells, sh_ll, &tot);
            block_inclusive_scan<long long>(wcells, sh_ll, &wtot);
            if (threadIdx.x == 0) {
                s_active_cells += tot;
                s_waiting_cells += wtot;
            }
            __syncthreads();
        }
        // waiting models in index order, while they fit -- under the pressure
        // schedule on multiples of 10 of the loop's count (any time when no
        // model runs); between them the launch ends at the next multiple
        const long long room = ctl->budget - s_active_cells;
        const bool none = s_active_cells == 0;
        const int phase = ctl->num_it % 10;
        const bool sched = models[0].c.pressure_schedule != 0;
        const bool admit_now = none || !sched || phase == 0;
        if (!admit_now && s_waiting_cells > 0 && room > 0 && threadIdx.x == 0) s_cap = 10 - phase;
        for (int base = 0; base < n && admit_now; base += kPlanThreads) {
            const int i = base + threadIdx.x;
            const bool w = i < n && models[i].waiting;
            const long long cells = w ? 2 * models[i].c.L.Nc : 0;
            long long tot;
            const long long p = block_inclusive_scan<long long>(cells, sh_ll, &tot);
            const long long incl = s_base_w + p;
            if (w && (incl <= room || (none && incl == cells))) {
                models[i].waiting = 0;
                models[i].active = 1;
                models[i].inner = 0;
            }
            __syncthreads();
            if (threadIdx.x == 0) s_base_w += tot;
            __syncthreads();
        }
    }
    for (int base = 0; base < n; base += kPlanThreads) {
        const int i = base + threadIdx.x;
        int a = 0;
        long long nc = 0;
        if (i < n && models[i].active) {
            const FusedModel& M = models[i];
            const DcState* st = M.c.st;
            a = 1;
            nc = M.nchunks;
            int lim = M.c.cycle - M.inner;
            const int h = M.c.max_it - st->num_sub_it;
            lim = h < lim ? h : lim;
            if (st->dt <= M.c.min_dt) lim = 1;
            atomicMin(&s_gmax, lim);
            atomicMin(&s_young, st->num_it);
            atomicOr(&s_mask, 1 << ((10 - st->num_it % 10) % 10));
        }
        int tot_a;
        long long tot_c;
        const int pa = block_inclusive_scan<int>(a, sh_i, &tot_a);
        const long long pc = block_inclusive_scan<long long>(nc, sh_ll, &tot_c);
        if (a) {
            const int k = s_base_k + pa - 1;
            FusedItem I;
            I.c = models[i].c;
            I.cfirst = s_base_ch + pc - nc;
            I.nchunks = nc;
            I.inner = models[i].inner;
            I.age0 = models[i].c.st->num_it;
            items[k] = I;
            idx[k] = i;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            s_base_k += tot_a;
            s_base_ch += tot_c;
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        FusedArgs A;
        A.items = items;
        A.nitems = s_base_k;
        A.chunks = chunks;
        A.nchunks = s_base_ch;
        A.cpart = cpart;
        A.any_event = any_event;
        A.bar = bar;
        const int gm = s_gmax < s_cap ? s_gmax : s_cap;
        A.g_max = gm < 1 ? 1 : gm;
        A.num_it0 = ctl->num_it;
        A.pressure_schedule = s_base_k > 0 ? items[0].c.pressure_schedule : 0;
        A.young = s_young;
        A.mask10 = s_mask;
        *args = A;
        *any_event = 0;
        bar->count = 0;
        bar->gen = 0;
        bar->error = 0;
    }
}

// the chunk table: chunk q of the launch is chunk q - cfirst of the last
// model whose range starts at or before q
__global__ void fused_fill_kernel(const FusedArgs* args, FusedChunk* chunks) {
    const FusedArgs A = *args;
    for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < A.nchunks;
         q += (long long)gridDim.x * blockDim.x) {
        int lo = 0, hi = A.nitems - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (A.items[mid].cfirst <= q) lo = mid;
            else hi = mid - 1;
        }
        FusedChunk ch;
        ch.m0 = (q - A.items[lo].cfirst) * kTmaChunk;
        ch.item = lo;
        ch.pad = 0;
        chunks[q] = ch;
    }
}

// run_fused's event handling: each model's next step from its event, its
// iterations since the last residual, whether it goes on; the residual
// blocks of the models that need one; the loop condition
__global__ void __launch_bounds__(kPlanThreads) fused_events_kernel(FusedCtl* ctl, FusedModel* models,
                                                                    const FusedArgs* args, const int* idx,
                                                                    int* act, long long* rstart,
                                                                    cudaGraphConditionalHandle cond) {
    __shared__ long long sh_ll[32];
    __shared__ int s_ran, s_failed, s_active;
    __shared__ long long s_base;
    const FusedArgs A = *args;
    const int na = A.nitems;
    if (threadIdx.x == 0) {
        // every model decides at the launch's last iteration: its own count
        // then tells how many iterations the launch ran
        s_ran = na > 0 ? A.items[0].c.st->num_it - A.items[0].age0 : 0;
        s_failed = 0;
        s_active = 0;
        s_base = 0;
    }
    __syncthreads();
    const int ran = s_ran;
    for (int base = 0; base < na; base += kPlanThreads) {
        const int k = base + threadIdx.x;
        long long rb = 0;
        if (k < na) {
            FusedModel& M = models[idx[k]];
            const int ev = A.items[k].c.st->event;
            int a = 0;
            M.inner += ran;
            switch (ev) {
                case EV_NONE: break;
                case EV_CONVERGED:
                case EV_STOP: a = ACT_APPLY; M.active = 0; break;
                case EV_REFRESH:
                case EV_CYCLE_END: a = ACT_APPLY | ACT_RESID; M.inner = 0; break;
                case EV_HALVE: a = ACT_HALVE | ACT_RESID; M.inner = 0; break;
                case EV_STOP_HALVED: a = ACT_HALVE; M.active = 0; break;
                default: atomicExch(&s_failed, 1); M.active = 0; break;   // EV_ERROR
            }
            act[k] = a;
            if (a & ACT_RESID) rb = res_blocks(A.items[k].c.L.Nc);
        }
        long long tot;
        const long long p = block_inclusive_scan<long long>(rb, sh_ll, &tot);
        if (k < na) rstart[k] = s_base + p - rb;
        __syncthreads();
        if (threadIdx.x == 0) s_base += tot;
        __syncthreads();
    }
    // a failure ends every model, after this pass's steps (as run_fused)
    const bool failed = s_failed != 0;
    for (int i = threadIdx.x; i < ctl->n; i += blockDim.x) {
        if (failed) {
            models[i].active = 0;
            models[i].waiting = 0;
        } else if (models[i].active || models[i].waiting) {
            atomicAdd(&s_active, 1);
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        ctl->num_it += ran;
        ctl->launches += 1;
        ctl->iterations += ran;
        ctl->runs += 1;
        ctl->resid_total = s_base;
        if (failed) ctl->failed = 1;
        ctl->nactive = s_active;
        cudaGraphSetConditional(cond, (s_active > 0 && !failed && ctl->runs < ctl->max_runs) ? 1u : 0u);
    }
}

// x += d (dc_apply_kernel) or the dt-halving reset (dc_halve_kernel) of the
// models whose event asks for it, chunk by chunk
template <class Form>
__global__ void fused_update_kernel(const FusedArgs* args, const Form* forms, const int* idx, const int* act) {
    const FusedArgs A = *args;
    for (long long q = blockIdx.x; q < A.nchunks; q += gridDim.x) {
        const FusedChunk ch = A.chunks[q];
        const int a = act[ch.item];
        if (!(a & (ACT_APPLY | ACT_HALVE))) continue;
        const DcCtl& c = A.items[ch.item].c;
        const Form F = forms[idx[ch.item]];
        const long long Nc = c.L.Nc;
        for (int t = threadIdx.x; t < 2 * kTmaChunk; t += blockDim.x) {
            const int col = t >= kTmaChunk;
            const long long m = ch.m0 + (t - col * kTmaChunk);
            if (m >= Nc) continue;
            if (a & ACT_APPLY) {
                if (c.mask[col][m] & F_ACTIVE) c.X[col][m] = c.X[col][m] + (double)c.D[col][m];
            } else {
                F.reassemble(col, m, c.st->dt);
                scale_cell(F, c, col, m);
            }
        }
    }
}

// the residual of the models that need one: block vb of the launch is
// residual block vb - rstart[k] of the last model k starting at or before vb
template <class Form>
__global__ void __launch_bounds__(kBlock) fused_residual_kernel(const FusedArgs* args, const Form* forms,
                                                                const int* idx, const long long* rstart,
                                                                const FusedCtl* ctl) {
    __shared__ double sh[kBlock / 32];
    const FusedArgs A = *args;
    const long long total = ctl->resid_total;
    for (long long vb = blockIdx.x; vb < total; vb += gridDim.x) {
        int lo = 0, hi = A.nitems - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (rstart[mid] <= vb) lo = mid;
            else hi = mid - 1;
        }
        const DcCtl& c = A.items[lo].c;
        const Form F = forms[idx[lo]];
        const long long b = vb - rstart[lo];
        const double o2 = residual_block_cells(F, c, b, res_blocks(c.L.Nc));
        const double s = block_sum<kBlock>(o2, sh);
        if (threadIdx.x == 0) c.partials[b] = s;
    }
}

// x^2 totals of the models whose residual was formed (dc_x2_kernel)
__global__ void __launch_bounds__(kBlock) fused_x2_kernel(const FusedArgs* args, const int* act) {
    __shared__ double sh[kBlock / 32];
    const FusedArgs A = *args;
    for (int k = blockIdx.x; k < A.nitems; k += gridDim.x) {
        if (!(act[k] & ACT_RESID)) continue;
        const DcCtl& c = A.items[k].c;
        const int nparts = res_blocks(c.L.Nc);
        double s = 0.0;
        for (int b = threadIdx.x; b < nparts; b += blockDim.x) s = s + c.partials[b];
        s = block_sum<kBlock>(s, sh);
        if (threadIdx.x == 0) {
            c.st->x2 = s;
            c.st->cycles += 1;
        }
    }
}

static size_t fused_loop_bytes(int n) {
    const size_t form = sizeof(PressureForm) > sizeof(TransportForm) ? sizeof(PressureForm) : sizeof(TransportForm);
    return align256(sizeof(FusedModel) * n) + 2 * align256(sizeof(int) * n) + align256(sizeof(long long) * n) +
           align256(sizeof(FusedArgs)) + align256(sizeof(FusedCtl)) + align256(form * n);
}

// Instantiated device-loop graphs, kept across calls.  A graph's nodes hold
// the addresses it carves from the batch workspace, the launch shapes and
// the stage layout, which the key fixes (device, form, workspace address,
// model count, total cells, tallest column, ring length); everything that
// varies between calls -- the models, their state, their arguments -- goes in
// through the workspace before the launch.  Slots are handed out one call at
// a time (a slot in use is neither shared nor evicted); a call that finds
// every slot busy builds its own graph and destroys it at the end.  The cache
// is kept until the process exits (a device reset is not supported).
struct GraphKey {
    int dev, form;
    const void* ws;
    int n;
    long long cells;
    int Hmax, ring;
    bool operator==(const GraphKey& o) const {
        return dev == o.dev && form == o.form && ws == o.ws && n == o.n && cells == o.cells &&
               Hmax == o.Hmax && ring == o.ring;
    }
};
struct GraphSlot {
    GraphKey key;
    cudaGraph_t graph;
    cudaGraphExec_t exec;
    bool busy;
    unsigned long long used;   // last use, for eviction
};
constexpr int kGraphSlots = 32;
static std::mutex g_graph_mu;
static GraphSlot g_graph_slots[kGraphSlots];
static unsigned long long g_graph_clock = 0;

// the cached graph of `key` (slot->exec set), or a slot reserved for it
// (exec null: the caller builds and hands the graph over at release), or
// null when every slot is busy
static GraphSlot* graph_cache_acquire(const GraphKey& key) {
    std::lock_guard<std::mutex> lk(g_graph_mu);
    GraphSlot* victim = nullptr;
    for (auto& s : g_graph_slots) {
        if (s.exec && s.key == key && !s.busy) {
            s.busy = true;
            s.used = ++g_graph_clock;
            return &s;
        }
    }
    for (auto& s : g_graph_slots) {
        if (s.busy) continue;
        if (!s.exec) { victim = &s; break; }
        if (!victim || s.used < victim->used) victim = &s;
    }
    if (!victim) return nullptr;
    if (victim->exec) {
        cudaGraphExecDestroy(victim->exec);
        cudaGraphDestroy(victim->graph);
        victim->exec = nullptr;
        victim->graph = nullptr;
    }
    victim->key = key;
    victim->busy = true;
    victim->used = ++g_graph_clock;
    return victim;
}

// end of a call: a graph built for a reserved slot goes into it; without a
// slot the graph is destroyed
static void graph_cache_release(GraphSlot* slot, cudaGraph_t graph, cudaGraphExec_t exec) {
    std::lock_guard<std::mutex> lk(g_graph_mu);
    if (!slot) {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        return;
    }
    if (!slot->exec && exec) {
        slot->exec = exec;
        slot->graph = graph;
    }
    slot->busy = false;
}

// batch solves run by each loop since the library was loaded
std::atomic<long long> g_graph_solves{0}, g_host_solves{0};

// The fused form with the device-driven loop.  Returns 1 without doing
// anything when the graph cannot be built (mode 0, the legacy stream, a
// runtime without conditional nodes), so the caller runs run_fused.
template <class Form>
static int run_fused_graph(std::vector<BatchItem<Form>>& v, TseDcOptions* opts, void* d_ws, size_t ws_bytes,
                           cudaStream_t stream) {
    if ((opts && opts->host_loop == 1) || stream == nullptr) return 1;
    const int n = (int)v.size();
    // cells (both colours) active at once; below the batch's total, waiting
    // models are admitted as others finish
    long long budget = (opts && opts->active_cells > 0) ? opts->active_cells : 0;
    long long cells = 0;
    int Hmax = 0;
    for (auto& it : v) {
        cells += (long long)it.c.L.nx * it.c.L.ny * it.c.L.nz;
        Hmax = it.c.L.H > Hmax ? it.c.L.H : Hmax;
    }
    if (fused_ws_bytes(n, cells) > ws_bytes) return TSE_ERR_WORKSPACE;
    TmaStage T = tma_stage(Hmax);
    int dev = 0, sms = 0, per_sm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int pipes = kFusedPipes;
    const int avail =
        (int)std::min<size_t>((size_t)(kFusedMaxRing * pipes), fused_max_smem() / (size_t)T.bytes);
    const int ring = avail / pipes;
    if (ring < 2) return TSE_ERR_ARG;
    const void* kernel = ring == 2   ? (const void*)fused_sweep_dev_kernel<2, kFusedPipes>
                         : ring == 3 ? (const void*)fused_sweep_dev_kernel<3, kFusedPipes>
                                     : (const void*)fused_sweep_dev_kernel<4, kFusedPipes>;
    const int fused_threads = kTmaConsumers + 32 * pipes;
    T.stages = ring * pipes;
    const size_t smem = (size_t)T.stages * T.bytes;
    if (cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)fused_max_smem()) !=
            cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, fused_threads, smem) != cudaSuccess ||
        per_sm < 1) {
        cudaGetLastError();
        return 1;
    }
    // the batch workspace: run_fused's areas, then the loop's own
    const size_t nch_max = (size_t)(cells / kTmaChunk) + (size_t)n + 1;
    char* p = (char*)d_ws;
    FusedItem* d_items = (FusedItem*)p;
    p += align256(sizeof(FusedItem) * n);
    FusedChunk* d_chunks = (FusedChunk*)p;
    p += align256(sizeof(FusedChunk) * nch_max);
    double2* d_cpart = (double2*)p;
    p += align256(sizeof(double2) * 8 * nch_max);
    p += align256(sizeof(DcState) * n);
    int* d_any = (int*)p;
    p += 256;
    GridBarrier* d_bar = (GridBarrier*)p;
    p += align256(sizeof(GridBarrier)) + 256;
    FusedModel* d_models = (FusedModel*)p;
    p += align256(sizeof(FusedModel) * n);
    int* d_idx = (int*)p;
    p += align256(sizeof(int) * n);
    int* d_act = (int*)p;
    p += align256(sizeof(int) * n);
    long long* d_rstart = (long long*)p;
    p += align256(sizeof(long long) * n);
    FusedArgs* d_args = (FusedArgs*)p;
    p += align256(sizeof(FusedArgs));
    FusedCtl* d_ctl = (FusedCtl*)p;
    p += align256(sizeof(FusedCtl));
    Form* d_forms = (Form*)p;

    long long nb = (long long)sms * per_sm;
    if (nb > (long long)nch_max) nb = (long long)nch_max;
    const unsigned grid_small = (unsigned)(4 * sms), grid_big = (unsigned)(8 * sms);

    // the graph: one WHILE node, its body built node by node.  Its
    // nodes hold only workspace addresses, launch shapes and the stage
    // layout, all fixed by the key, so a later call with the same key reuses
    // the instantiated graph (the models' data go in through the workspace)
    const GraphKey key{dev, std::is_same<Form, PressureForm>::value ? 0 : 1, d_ws, n, cells, Hmax, ring};
    GraphSlot* slot = graph_cache_acquire(key);
    cudaGraph_t graph = nullptr, body = nullptr;
    cudaGraphExec_t exec = slot ? slot->exec : nullptr;
    cudaGraphConditionalHandle cond;
    bool built = exec != nullptr;
    if (!built) {
        built = cudaGraphCreate(&graph, 0) == cudaSuccess &&
                cudaGraphConditionalHandleCreate(&cond, graph, 1, cudaGraphCondAssignDefault) == cudaSuccess;
        if (built) {
            cudaGraphNodeParams cp = {};
            cp.type = cudaGraphNodeTypeConditional;
            cp.conditional.handle = cond;
            cp.conditional.type = cudaGraphCondTypeWhile;
            cp.conditional.size = 1;
            cudaGraphNode_t node;
            built = cudaGraphAddNode(&node, graph, nullptr, 0, &cp) == cudaSuccess;
            if (built) body = cp.conditional.phGraph_out[0];
        }
        // The body, node by node (no stream capture: a capture in progress
        // would stand in the way of other threads' work on their own
        // streams, e.g. a model's state going up from pageable memory): the
        // loop's kernels in order, the sweep a cooperative launch.
        cudaGraphNode_t prev = nullptr;
        auto add = [&](const void* func, unsigned grid, unsigned block, size_t shmem, void** kargs,
                       bool coop) {
            if (!built) return;
            cudaKernelNodeParams kp = {};
            kp.func = const_cast<void*>(func);
            kp.gridDim = dim3(grid);
            kp.blockDim = dim3(block);
            kp.sharedMemBytes = (unsigned)shmem;
            kp.kernelParams = kargs;
            kp.extra = nullptr;
            cudaGraphNode_t node;
            built = cudaGraphAddKernelNode(&node, body, prev ? &prev : nullptr, prev ? 1 : 0, &kp) ==
                    cudaSuccess;
            if (built && coop) {
                cudaKernelNodeAttrValue v = {};
                v.cooperative = 1;
                built = cudaGraphKernelNodeSetAttribute(node, cudaKernelNodeAttributeCooperative, &v) ==
                        cudaSuccess;
            }
            prev = node;
        };
        const FusedCtl* c_ctl = d_ctl;
        const FusedArgs* c_args = d_args;
        const int* c_idx = d_idx;
        const int* c_act = d_act;
        const long long* c_rstart = d_rstart;
        const Form* c_forms = d_forms;
        FusedCtl* m_ctl = d_ctl;
        void* a_plan[] = {(void*)&c_ctl, (void*)&d_models, (void*)&d_items, (void*)&d_idx, (void*)&d_args,
                          (void*)&d_chunks, (void*)&d_cpart, (void*)&d_any, (void*)&d_bar};
        void* a_fill[] = {(void*)&c_args, (void*)&d_chunks};
        void* a_sweep[] = {(void*)&c_args, (void*)&T, (void*)&m_ctl};
        void* a_events[] = {(void*)&m_ctl, (void*)&d_models, (void*)&c_args, (void*)&c_idx, (void*)&d_act,
                            (void*)&d_rstart, (void*)&cond};
        void* a_update[] = {(void*)&c_args, (void*)&c_forms, (void*)&c_idx, (void*)&c_act};
        void* a_resid[] = {(void*)&c_args, (void*)&c_forms, (void*)&c_idx, (void*)&c_rstart, (void*)&c_ctl};
        void* a_x2[] = {(void*)&c_args, (void*)&c_act};
        add((const void*)fused_plan_kernel, 1, kPlanThreads, 0, a_plan, false);
        add((const void*)fused_fill_kernel, grid_small, kBlock, 0, a_fill, false);
        add(kernel, (unsigned)nb, (unsigned)fused_threads, smem, a_sweep, true);
        add((const void*)fused_events_kernel, 1, kPlanThreads, 0, a_events, false);
        add((const void*)fused_update_kernel<Form>, grid_big, kBlock, 0, a_update, false);
        add((const void*)fused_residual_kernel<Form>, grid_big, kBlock, 0, a_resid, false);
        add((const void*)fused_x2_kernel, grid_small, kBlock, 0, a_x2, false);
        if (!built) cudaGetLastError();
        if (built) built = cudaGraphInstantiate(&exec, graph, 0) == cudaSuccess;
        if (!built) {
            cudaGetLastError();
            if (exec) cudaGraphExecDestroy(exec);
            if (graph) cudaGraphDestroy(graph);
            graph_cache_release(slot, nullptr, nullptr);
            return 1;
        }
    }
    // the graph goes back to the cache (or is destroyed) when the call ends
    struct Release {
        GraphSlot* slot;
        cudaGraph_t graph;
        cudaGraphExec_t exec;
        ~Release() { graph_cache_release(slot, graph, exec); }
    } release{slot, graph, exec};

    // every model: state, scaled records, first residual (as run_fused)
    int rc = TSE_OK;
    for (auto& it : v) {
        rc = it.nparts > 0 ? dc_begin_fused(it.c, it.dt, it.nparts, stream)
                           : dc_begin(it.F, it.c, it.dt, stream);
        if (rc == TSE_OK && it.nparts == 0) rc = dc_residual(it.F, it.c, stream);
        if (rc != TSE_OK) break;
    }
    std::vector<FusedModel> hm(n);
    std::vector<Form> hf(n);
    for (int i = 0; i < n && rc == TSE_OK; ++i) {
        memset(&hm[i], 0, sizeof(FusedModel));
        hm[i].c = v[i].c;
        hm[i].nchunks = (v[i].c.L.Nc + kTmaChunk - 1) / kTmaChunk;
        // with a cell budget every model waits for the first plan to admit it
        hm[i].active = budget > 0 ? 0 : 1;
        hm[i].waiting = budget > 0 ? 1 : 0;
        hm[i].inner = 0;
        hf[i] = v[i].F;
    }
    FusedCtl hc;
    memset(&hc, 0, sizeof(hc));
    hc.n = n;
    hc.nactive = n;
    hc.budget = budget;
    hc.max_runs = (opts && opts->graph_runs > 0) ? opts->graph_runs : kGraphMaxRuns;
    // pageable sources: staged before the calls return
    if (rc == TSE_OK &&
        (cudaMemcpyAsync(d_models, hm.data(), sizeof(FusedModel) * n, cudaMemcpyHostToDevice, stream) !=
             cudaSuccess ||
         cudaMemcpyAsync(d_forms, hf.data(), sizeof(Form) * n, cudaMemcpyHostToDevice, stream) != cudaSuccess ||
         cudaMemcpyAsync(d_ctl, &hc, sizeof(FusedCtl), cudaMemcpyHostToDevice, stream) != cudaSuccess))
        rc = TSE_ERR_LAUNCH;
    const bool timing = opts && opts->timing;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    if (rc == TSE_OK && timing &&
        (cudaEventCreate(&ev0) != cudaSuccess || cudaEventCreate(&ev1) != cudaSuccess))
        rc = TSE_ERR_LAUNCH;
    if (rc == TSE_OK && timing) cudaEventRecord(ev0, stream);
    // graph launches until every model has finished: one, unless a solve needs
    // more than max_runs sweep launches
    int launches = 0;
    for (int launch = 0; rc == TSE_OK; ++launch) {
        ++launches;
        if (cudaGraphLaunch(exec, stream) != cudaSuccess ||
            cudaMemcpyAsync(&hc, d_ctl, sizeof(FusedCtl), cudaMemcpyDeviceToHost, stream) != cudaSuccess ||
            cudaStreamSynchronize(stream) != cudaSuccess) {
            rc = TSE_ERR_LAUNCH;
            break;
        }
        if (hc.failed || hc.nactive == 0) break;
        if (launch >= 100000) {
            rc = TSE_ERR_LAUNCH;
            break;
        }
        hc.runs = 0;
        if (cudaMemcpyAsync(&d_ctl->runs, &hc.runs, sizeof(int), cudaMemcpyHostToDevice, stream) != cudaSuccess)
            rc = TSE_ERR_LAUNCH;
    }
    if (timing && ev0) {
        cudaEventRecord(ev1, stream);
        cudaEventSynchronize(ev1);
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, ev0, ev1);
        opts->sweep_launches = hc.launches;
        opts->sweep_iterations = hc.iterations;
        opts->sweep_ms = (double)hc.sweep_ns * 1e-6;
        opts->loop_ms = ms;
        cudaEventDestroy(ev0);
        cudaEventDestroy(ev1);
    }
    if (opts) opts->graph_runs = launches;
    g_graph_solves.fetch_add(1);
    // status records and results of every model
    for (auto& it : v) {
        const int r = dc_finish(it.c, it.status, it.X_out, stream);
        if (rc == TSE_OK) rc = r;
    }
    return rc;
}

}  // namespace tse

using namespace tse;

extern "C" int32_t tse_batch_loop_stats(int64_t* graph_solves, int64_t* host_solves) {
    if (!graph_solves || !host_solves) return TSE_ERR_ARG;
    *graph_solves = g_graph_solves.load();
    *host_solves = g_host_solves.load();
    return TSE_OK;
}

extern "C" size_t tse_batch_workspace_bytes(int32_t n, int64_t total_cells) {
    if (n < 1) n = 1;
    if (total_cells < 0) total_cells = 0;
    const size_t a = sizeof(BatchItem<PressureForm>), b = sizeof(BatchItem<TransportForm>);
    const size_t cluster = align256((a > b ? a : b) * (size_t)n) + 256;
    const size_t fused = fused_ws_bytes(n, total_cells);
    return cluster > fused ? cluster : fused;
}

extern "C" int32_t tse_compute_P_dc_batch(const TseBatchPressure* items, int32_t n,
                                          TseDcOptions* opts, void* d_batch_ws,
                                          size_t batch_ws_bytes, void* stream_) {
    if (!items || n < 1 || !d_batch_ws) return TSE_ERR_ARG;
    cudaStream_t stream = (cudaStream_t)stream_;
    std::vector<BatchItem<PressureForm>> v(n);
    // the cluster form scales and forms the first residual in its own kernel
    const bool fused = !(opts && opts->max_blocks > 0);
    for (int i = 0; i < n; ++i) {
        const TseBatchPressure& b = items[i];
        const TsePressureArgs* a = b.args;
        if (!b.grid || !a || !b.d_status || !b.d_workspace || a->max_it < 1 ||
            !finite_dt(a->dt_P, a->min_dt) || !a->P)
            return TSE_ERR_ARG;
        PressureSetup S;
        int np = 0;
        int rc = fused ? setup_pressure_dc(b.grid, a, b.d_workspace, b.workspace_bytes, stream, S, &np)
                         : setup_pressure(b.grid, a, b.d_workspace, b.workspace_bytes, stream, S);
        if (rc != TSE_OK) return rc;
        if (S.tail_bytes < dc_extra_bytes(S.L)) return TSE_ERR_WORKSPACE;
        v[i].F = S.F;
        dc_carve(S, v[i].c, PA_P);
        fill_ctl(v[i].c, a->inc_it, a->max_dt, a->min_dt, a->P_conv, a->max_it, 1, 0, opts, a->SOR);
        v[i].dt = a->dt_P;
        v[i].status = b.d_status;
        v[i].X_out = a->P;
        v[i].cells = 2 * S.L.Nc;
        v[i].nparts = np;
    }
    if (opts && opts->max_blocks > 0) return launch_batch(v, opts, d_batch_ws, batch_ws_bytes, stream);
    const int g = run_fused_graph(v, opts, d_batch_ws, batch_ws_bytes, stream);
    if (g != 1) return g;
    g_host_solves.fetch_add(1);
    return run_fused(v, opts, d_batch_ws, batch_ws_bytes, stream);
}

extern "C" int32_t tse_compute_C_dc_batch(const TseBatchSpecies* items, int32_t n,
                                          TseDcOptions* opts, void* d_batch_ws,
                                          size_t batch_ws_bytes, void* stream_) {
    if (!items || n < 1 || !d_batch_ws) return TSE_ERR_ARG;
    cudaStream_t stream = (cudaStream_t)stream_;
    std::vector<BatchItem<TransportForm>> v(n);
    const bool fused = !(opts && opts->max_blocks > 0);
    for (int i = 0; i < n; ++i) {
        const TseBatchSpecies& b = items[i];
        const TseSpeciesArgs* a = b.args;
        if (!b.grid || !a || !b.d_status || !b.d_workspace || a->max_it < 1 ||
            !finite_dt(a->dt, a->min_dt) || !a->C)
            return TSE_ERR_ARG;
        TransportSetup S;
        int np = 0;
        int rc = fused ? setup_species_dc(b.grid, a, b.d_workspace, b.workspace_bytes, stream, S, &np)
                         : setup_species(b.grid, a, b.d_workspace, b.workspace_bytes, stream, S);
        if (rc != TSE_OK) return rc;
        if (S.tail_bytes < dc_extra_bytes(S.L)) return TSE_ERR_WORKSPACE;
        v[i].F = S.F;
        dc_carve(S, v[i].c, TA_X);
        fill_ctl(v[i].c, a->inc_it, a->max_dt, a->min_dt, a->conv, a->max_it, 0, a->omega == 0.0,
                 opts, a->SOR);
        v[i].dt = a->dt;
        v[i].status = b.d_status;
        v[i].X_out = a->C;
        v[i].cells = 2 * S.L.Nc;
        v[i].nparts = np;
    }
    if (opts && opts->max_blocks > 0) return launch_batch(v, opts, d_batch_ws, batch_ws_bytes, stream);
    const int g = run_fused_graph(v, opts, d_batch_ws, batch_ws_bytes, stream);
    if (g != 1) return g;
    g_host_solves.fetch_add(1);
    return run_fused(v, opts, d_batch_ws, batch_ws_bytes, stream);
}

extern "C" int32_t tse_compute_T_dc_batch(const TseBatchHeat* items, int32_t n,
                                          TseDcOptions* opts, void* d_batch_ws,
                                          size_t batch_ws_bytes, void* stream_) {
    if (!items || n < 1 || !d_batch_ws) return TSE_ERR_ARG;
    cudaStream_t stream = (cudaStream_t)stream_;
    std::vector<BatchItem<TransportForm>> v(n);
    const bool fused = !(opts && opts->max_blocks > 0);
    for (int i = 0; i < n; ++i) {
        const TseBatchHeat& b = items[i];
        const TseHeatArgs* a = b.args;
        if (!b.grid || !a || !b.d_status || !b.d_workspace || a->max_it < 1 ||
            !finite_dt(a->dt, a->min_dt) || !a->T)
            return TSE_ERR_ARG;
        TransportSetup S;
        int np = 0;
        int rc = fused ? setup_heat_dc(b.grid, a, b.d_workspace, b.workspace_bytes, stream, S, &np)
                         : setup_heat(b.grid, a, b.d_workspace, b.workspace_bytes, stream, S);
        if (rc != TSE_OK) return rc;
        if (S.tail_bytes < dc_extra_bytes(S.L)) return TSE_ERR_WORKSPACE;
        v[i].F = S.F;
        dc_carve(S, v[i].c, TA_X);
        fill_ctl(v[i].c, a->inc_it, a->max_dt, a->min_dt, a->conv, a->max_it, 0, a->omega == 0.0,
                 opts, a->SOR);
        v[i].dt = a->dt;
        v[i].status = b.d_status;
        v[i].X_out = a->T;
        v[i].cells = 2 * S.L.Nc;
        v[i].nparts = np;
    }
    if (opts && opts->max_blocks > 0) return launch_batch(v, opts, d_batch_ws, batch_ws_bytes, stream);
    const int g = run_fused_graph(v, opts, d_batch_ws, batch_ws_bytes, stream);
    if (g != 1) return g;
    g_host_solves.fetch_add(1);
    return run_fused(v, opts, d_batch_ws, batch_ws_bytes, stream);
}
