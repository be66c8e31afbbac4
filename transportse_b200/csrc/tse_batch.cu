// Batched mixed-precision solves: many independent models in one persistent
// launch, one thread-block cluster per model.
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
        const int k = (int)(q % L.nz);
        const long long row = q / L.nz;
        const int j = (int)(row % L.ny);
        const int i = (int)(row / L.ny);
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
    c.cycle = (opts && opts->cycle > 0) ? opts->cycle : 128;
    c.sor = (float)sor;
}

// NaN in dt or min_dt would keep a non-converging solve halving forever
static bool finite_dt(double dt, double min_dt) { return std::isfinite(dt) && std::isfinite(min_dt); }

}  // namespace tse

using namespace tse;

extern "C" size_t tse_batch_workspace_bytes(int32_t n) {
    const size_t a = sizeof(BatchItem<PressureForm>), b = sizeof(BatchItem<TransportForm>);
    return align256((a > b ? a : b) * (size_t)(n > 0 ? n : 1)) + 256;
}

extern "C" int32_t tse_compute_P_dc_batch(const TseBatchPressure* items, int32_t n,
                                          const TseDcOptions* opts, void* d_batch_ws,
                                          size_t batch_ws_bytes, void* stream_) {
    if (!items || n < 1 || !d_batch_ws) return TSE_ERR_ARG;
    cudaStream_t stream = (cudaStream_t)stream_;
    std::vector<BatchItem<PressureForm>> v(n);
    for (int i = 0; i < n; ++i) {
        const TseBatchPressure& b = items[i];
        const TsePressureArgs* a = b.args;
        if (!b.grid || !a || !b.d_status || !b.d_workspace || a->max_it < 1 ||
            !finite_dt(a->dt_P, a->min_dt) || !a->P)
            return TSE_ERR_ARG;
        PressureSetup S;
        int rc = setup_pressure(b.grid, a, b.d_workspace, b.workspace_bytes, stream, S);
        if (rc != TSE_OK) return rc;
        if (S.tail_bytes < dc_extra_bytes(S.L)) return TSE_ERR_WORKSPACE;
        v[i].F = S.F;
        dc_carve(S, v[i].c, PA_P);
        fill_ctl(v[i].c, a->inc_it, a->max_dt, a->min_dt, a->P_conv, a->max_it, 1, 0, opts, a->SOR);
        v[i].dt = a->dt_P;
        v[i].status = b.d_status;
        v[i].X_out = a->P;
        v[i].cells = 2 * S.L.Nc;
    }
    return launch_batch(v, opts, d_batch_ws, batch_ws_bytes, stream);
}

extern "C" int32_t tse_compute_C_dc_batch(const TseBatchSpecies* items, int32_t n,
                                          const TseDcOptions* opts, void* d_batch_ws,
                                          size_t batch_ws_bytes, void* stream_) {
    if (!items || n < 1 || !d_batch_ws) return TSE_ERR_ARG;
    cudaStream_t stream = (cudaStream_t)stream_;
    std::vector<BatchItem<TransportForm>> v(n);
    for (int i = 0; i < n; ++i) {
        const TseBatchSpecies& b = items[i];
        const TseSpeciesArgs* a = b.args;
        if (!b.grid || !a || !b.d_status || !b.d_workspace || a->max_it < 1 ||
            !finite_dt(a->dt, a->min_dt) || !a->C)
            return TSE_ERR_ARG;
        TransportSetup S;
        int rc = setup_species(b.grid, a, b.d_workspace, b.workspace_bytes, stream, S);
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
    }
    return launch_batch(v, opts, d_batch_ws, batch_ws_bytes, stream);
}

extern "C" int32_t tse_compute_T_dc_batch(const TseBatchHeat* items, int32_t n,
                                          const TseDcOptions* opts, void* d_batch_ws,
                                          size_t batch_ws_bytes, void* stream_) {
    if (!items || n < 1 || !d_batch_ws) return TSE_ERR_ARG;
    cudaStream_t stream = (cudaStream_t)stream_;
    std::vector<BatchItem<TransportForm>> v(n);
    for (int i = 0; i < n; ++i) {
        const TseBatchHeat& b = items[i];
        const TseHeatArgs* a = b.args;
        if (!b.grid || !a || !b.d_status || !b.d_workspace || a->max_it < 1 ||
            !finite_dt(a->dt, a->min_dt) || !a->T)
            return TSE_ERR_ARG;
        TransportSetup S;
        int rc = setup_heat(b.grid, a, b.d_workspace, b.workspace_bytes, stream, S);
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
    }
    return launch_batch(v, opts, d_batch_ws, batch_ws_bytes, stream);
}
