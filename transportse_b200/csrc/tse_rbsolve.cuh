// Persistent red-black solver loop shared by the pressure and transport
// solves (tse.py:699-740 for compute_P, 877-914 for compute_C, 1045-1079 for
// compute_T).
//
// One cooperative launch runs the whole `while not converged` loop of the
// reference on the device: red half-sweep, grid barrier, black half-sweep,
// per-block partial sums of (new - old)^2 and old^2, grid barrier, the L2
// test, dt growth on convergence, or dt halving with a reset to the entry
// state after max_it sub-iterations.  Every block evaluates the L2 from the
// same partials in the same order, so all blocks take the same branch.
//
// Work mapping: block b, thread t owns compact cells m = b*blockDim + t +
// s*gridDim*blockDim of each colour for the whole solve, in the sweeps and in
// the reset alike, so a block only ever re-reads its own writes except for
// the other colour's values, which it loads through L2 (ld.cg).
#pragma once

#include "tse_common.cuh"

namespace tse {

struct SolveCtl {
    Layout L;
    long long Ncal;             // padded per-colour array length
    double dt, inc_it, max_dt, min_dt, conv;
    int max_it;
    int pressure_schedule;      // 1: L2 every it below 50, then every 10th
    int stop_on_first;          // 1: converged after one it (omega == 0)
    int plain_sweep;            // 1: plain-load kernel even where the staged one fits
    double* X[2];               // solution per colour
    const uint8_t* mask[2];
    double* partials;           // 2 doubles per block
    GridBarrier* bar;
    TseSolveStatus* status;
};

constexpr int kMaxBlocks = 16384;

template <class Form>
__global__ void __launch_bounds__(kBlock, 3) rb_solve_kernel(Form F, SolveCtl c) {
    __shared__ double sh[kBlock / 32];
    __shared__ double s_diff;
    const unsigned nb = gridDim.x;
    const long long tid0 = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long stride = (long long)nb * blockDim.x;
    const long long Nc = c.L.Nc;
    const bool leader = (blockIdx.x == 0 && threadIdx.x == 0);

    double t = 0.0, dt = c.dt, diff = 1e100;
    int converged = 0, num_it = 0, num_sub_it = 0, halvings = 0, err = 0, nev = 0;

    while (!converged) {
        num_it += 1;
        num_sub_it += 1;
        double d2 = 0.0, o2 = 0.0;
        const bool check = c.pressure_schedule ? (num_it < 50 || num_it % 10 == 0) : true;
        for (int col = 0; col < 2; ++col) {
            double* Xw = c.X[col];
            const double* Xo = c.X[1 - col];
            const uint8_t* msk = c.mask[col];
            for (long long m = tid0; m < Nc; m += stride) {
                const uint8_t f = msk[m];
                const double xold = Xw[m];
                o2 = o2 + xold * xold;
                if (f & F_ACTIVE) {
                    const double xn = F.update(col, m, f, xold, Xo);
                    Xw[m] = xn;
                    const double d = xn - xold;
                    d2 = d2 + d * d;
                }
            }
            if (col == 1 && check) {
                // per-block partial sums, published by the barrier below
                double b1 = block_sum<kBlock>(d2, sh);
                double b2 = block_sum<kBlock>(o2, sh);
                if (threadIdx.x == 0) {
                    c.partials[2 * blockIdx.x] = b1;
                    c.partials[2 * blockIdx.x + 1] = b2;
                }
            }
            if (!grid_sync(c.bar, nb)) { err = 1; break; }
        }
        if (err) break;
        diff = 1e100;
        if (check) {
            double s1 = 0.0, s2 = 0.0;
            for (unsigned b = threadIdx.x; b < nb; b += blockDim.x) {
                s1 = s1 + __ldcg(c.partials + 2 * b);
                s2 = s2 + __ldcg(c.partials + 2 * b + 1);
            }
            s1 = block_sum<kBlock>(s1, sh);
            s2 = block_sum<kBlock>(s2, sh);
            if (threadIdx.x == 0) {
                double l2 = sqrt(s1) / sqrt(s2 + 1e-200);
                s_diff = (l2 != l2) ? 1.0 : l2;
            }
            __syncthreads();
            diff = s_diff;
            // the next iteration's partial writes come after the next
            // half-sweep barrier, which every block reaches only after this
            // read: one partials buffer is enough
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
                for (int col = 0; col < 2; ++col)
                    for (long long m = tid0; m < Nc; m += stride) F.reassemble(col, m, dt);
                if (!grid_sync(c.bar, nb)) { err = 1; break; }
            }
            if (dt <= c.min_dt) break;
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
        s->error = err ? TSE_STATUS_BARRIER_TIMEOUT : TSE_STATUS_OK;
        s->n_events = nev < 8 ? nev : 8;
        s->cycles = 0;
    }
}

// Launch the persistent loop with as many co-resident blocks as useful.
template <class Form>
inline int launch_rb_solve(const Form& F, SolveCtl& ctl, cudaStream_t stream) {
    static int cached_dev = -1, cached_per_sm = 0, cached_sms = 0;
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev != cached_dev) {
        cudaDeviceGetAttribute(&cached_sms, cudaDevAttrMultiProcessorCount, dev);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&cached_per_sm, rb_solve_kernel<Form>,
                                                      kBlock, 0);
        cached_dev = dev;
    }
    long long maxb = (long long)cached_sms * (cached_per_sm > 0 ? cached_per_sm : 1);
    // at least 4 cells per thread per half-sweep, at most the co-resident set
    long long want = (ctl.L.Nc + (long long)kBlock * 4 - 1) / ((long long)kBlock * 4);
    if (want < 1) want = 1;
    long long nb = want < maxb ? want : maxb;
    if (nb > kMaxBlocks) nb = kMaxBlocks;
    void* args[] = {(void*)&F, (void*)&ctl};
    cudaError_t e = cudaLaunchCooperativeKernel((const void*)rb_solve_kernel<Form>, dim3((unsigned)nb),
                                                dim3(kBlock), args, 0, stream);
    return e == cudaSuccess ? TSE_OK : TSE_ERR_LAUNCH;
}

}  // namespace tse
