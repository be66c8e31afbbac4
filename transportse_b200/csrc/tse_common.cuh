// Shared device helpers for the TRANSPORTSE sm_100a kernels.
//
// FP64 kernels that must reproduce the reference bit for bit are compiled
// with --fmad=false and keep the reference's left-to-right operation order
// (tse.py evaluates each expression in Python/numba without contraction).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/tse_cuda.h"

namespace tse {

constexpr int kBlock = 256;
constexpr unsigned long long kBarrierTimeoutNs = 4000000000ull;  // 4 s

// ---------------------------------------------------------------- helpers
// harm (tse.py:297-310): spacing-weighted harmonic mean, 0 if either is 0.
__device__ __forceinline__ double harm2(double H1, double H2, double d1, double d2) {
    if (H1 != 0.0 && H2 != 0.0) return (d1 + d2) / (d1 / H1 + d2 / H2);
    return 0.0;
}
// amean (tse.py:284-294)
__device__ __forceinline__ double amean2(double X1, double X2, double d1, double d2) {
    return (X1 * d1 + X2 * d2) / (d1 + d2);
}
// Python builtin min(q, 0) / max(q, 0): keep q unless 0 compares strictly
// smaller / larger (tse.py:811-861 and 952-1027).
__device__ __forceinline__ double min0(double q) { return (0.0 < q) ? 0.0 : q; }
__device__ __forceinline__ double max0(double q) { return (0.0 > q) ? 0.0 : q; }
__device__ __forceinline__ double pymin(double a, double b) { return (b < a) ? b : a; }
// NaN-propagating max/min (numpy.max / numpy.min semantics)
__device__ __forceinline__ double nmax(double a, double b) {
    return (a != a) ? a : ((b != b) ? b : ((b > a) ? b : a));
}
__device__ __forceinline__ double nmin(double a, double b) {
    return (a != a) ? a : ((b != b) ? b : ((b < a) ? b : a));
}

// The grid coordinates of linear index t = (i*ny + j)*nz + k (nz may be a
// padded column height): 32-bit divisions while t fits, which is every grid
// below 2^32 cells -- a 64-bit division is several times the instructions.
__device__ __forceinline__ void grid_coords(long long t, int ny, int nz, int& i, int& j, int& k,
                                            long long& row) {
    if (t <= 0xffffffffLL) {
        const unsigned u = (unsigned)t, r = u / (unsigned)nz;
        k = (int)(u - r * (unsigned)nz);
        row = r;
        const unsigned ii = r / (unsigned)ny;
        j = (int)(r - ii * (unsigned)ny);
        i = (int)ii;
    } else {
        row = t / nz;
        k = (int)(t - row * nz);
        const long long ii = row / ny;
        j = (int)(row - ii * ny);
        i = (int)ii;
    }
}

__device__ __forceinline__ uint64_t globaltimer() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ double ld_cg(const double* p) { return __ldcg(p); }

__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned* p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// ------------------------------------------------------------ grid barrier
// Sense (generation) barrier across the blocks of one cooperative launch.
// Every wait is bounded in time; on timeout the block raises `error` and all
// waiting blocks leave their wait, so no block spins forever.
struct GridBarrier {
    unsigned count;
    unsigned gen;
    int error;
    int pad;
};

__device__ __forceinline__ bool grid_sync(GridBarrier* b, unsigned nblocks,
                                          unsigned long long timeout_ns = kBarrierTimeoutNs) {
    __syncthreads();
    if (nblocks == 1) return true;
    __shared__ int s_ok;
    if (threadIdx.x == 0) {
        int ok = 1;
        unsigned g = ld_acquire_u32(&b->gen);
        __threadfence();
        unsigned arrived = atomicAdd(&b->count, 1u);
        if (arrived == nblocks - 1) {
            atomicExch(&b->count, 0u);
            __threadfence();
            atomicAdd(&b->gen, 1u);
        } else {
            uint64_t t0 = globaltimer();
            unsigned spins = 0;
            while (ld_acquire_u32(&b->gen) == g) {
                if (*(volatile int*)&b->error) { ok = 0; break; }
                if ((++spins & 255u) == 0u && globaltimer() - t0 > timeout_ns) {
                    atomicExch(&b->error, 1);
                    ok = 0;
                    break;
                }
                __nanosleep(64);
            }
        }
        __threadfence();
        s_ok = ok;
    }
    __syncthreads();
    return s_ok != 0;
}

__device__ __forceinline__ void red_release_add(unsigned* p, unsigned v) {
    asm volatile("red.release.gpu.global.add.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Device-wide barrier of the staged and fused sweeps: each block adds 1 to a counter
// that is zeroed before the launch and never reset in it (release, no value
// returned), and barrier k of the launch is passed once the counter reaches
// k * nb (acquire).  No returning atomic, reset or generation flip sits
// between the last arrival and the waiters' release.  Bounded like
// grid_sync: on timeout (or another block's error) the error flag is raised
// and false returned.
__device__ __forceinline__ bool count_sync(unsigned* counter, unsigned target, GridBarrier* bar,
                                           unsigned long long timeout_ns = kBarrierTimeoutNs) {
    __syncthreads();
    __shared__ int s_ok;
    if (threadIdx.x == 0) {
        int ok = 1;
        red_release_add(counter, 1u);
        // wrap-safe: blocks are never more than one barrier apart
        if ((int)(ld_acquire_u32(counter) - target) < 0) {
            const uint64_t t0 = globaltimer();
            unsigned spins = 0;
            while ((int)(ld_acquire_u32(counter) - target) < 0) {
                if (*(volatile int*)&bar->error) { ok = 0; break; }
                if ((++spins & 255u) == 0u && globaltimer() - t0 > timeout_ns) {
                    atomicExch(&bar->error, 1);
                    ok = 0;
                    break;
                }
                __nanosleep(32);
            }
        }
        s_ok = ok;
    }
    __syncthreads();
    return s_ok != 0;
}

// ---------------------------------------------------------- block reduces
template <int NT>
__device__ __forceinline__ double block_sum(double v, double* sh) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = v + __shfl_down_sync(0xffffffffu, v, o);
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    __syncthreads();
    if (l == 0) sh[w] = v;
    __syncthreads();
    double r = 0.0;
    if (threadIdx.x == 0) {
        r = sh[0];
        for (int i = 1; i < NT / 32; ++i) r = r + sh[i];
    }
    return r;  // valid in thread 0
}

template <int NT>
__device__ __forceinline__ double block_nmax(double v, double* sh) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = nmax(v, __shfl_down_sync(0xffffffffu, v, o));
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    __syncthreads();
    if (l == 0) sh[w] = v;
    __syncthreads();
    double r = 0.0;
    if (threadIdx.x == 0) {
        r = sh[0];
        for (int i = 1; i < NT / 32; ++i) r = nmax(r, sh[i]);
    }
    return r;
}

template <int NT>
__device__ __forceinline__ double block_nmin(double v, double* sh) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = nmin(v, __shfl_down_sync(0xffffffffu, v, o));
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    __syncthreads();
    if (l == 0) sh[w] = v;
    __syncthreads();
    double r = 0.0;
    if (threadIdx.x == 0) {
        r = sh[0];
        for (int i = 1; i < NT / 32; ++i) r = nmin(r, sh[i]);
    }
    return r;
}

// ---------------------------------------------------- colour-split layout
// Red (colour 0) cells have (i + j + k) even and are swept first, as the GP
// mask of tse.py:170-176 orders them.  Each colour is stored compactly:
// with nzp = nz rounded up to even and H = nzp / 2, cell (i, j, k) of either
// colour has compact index m = ((i * ny + j) * nzp + k) >> 1.  Neighbours of
// the other colour sit at m +- ny*H (x), m +- H (y), and for z at
// m + (k & 1) (k+1) and m - 1 + (k & 1) (k-1).  A padding cell (k == nz,
// only when nz is odd) is inactive.
struct Layout {
    int nx, ny, nz, nzp, H;
    long long Nc;   // cells per colour
    long long SX;   // ny * H
};

__host__ __device__ inline Layout make_layout(int nx, int ny, int nz) {
    Layout L;
    L.nx = nx;
    L.ny = ny;
    L.nz = nz;
    L.nzp = nz + (nz & 1);
    L.H = L.nzp / 2;
    L.SX = (long long)ny * L.H;
    L.Nc = (long long)nx * L.SX;
    return L;
}

// per-cell flag byte of the compact layout
enum : uint8_t {
    F_ACTIVE = 1, F_XP = 2, F_XM = 4, F_YP = 8, F_YM = 16, F_ZP = 32, F_ZM = 64, F_KODD = 128
};

__device__ __forceinline__ uint8_t neighbour_flags(int i, int j, int k, int nx, int ny, int nz) {
    uint8_t f = 0;
    if (i < nx - 1) f |= F_XP;
    if (i > 0) f |= F_XM;
    if (j < ny - 1) f |= F_YP;
    if (j > 0) f |= F_YM;
    if (k < nz - 1) f |= F_ZP;
    if (k > 0) f |= F_ZM;
    if (k & 1) f |= F_KODD;
    return f;
}

__device__ __forceinline__ long long compact_index(int i, int j, int k, const Layout& L) {
    return (((long long)i * L.ny + j) * L.nzp + k) >> 1;
}

inline size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

// Number of co-resident blocks a cooperative launch of `kernel` may use.
template <typename K>
inline int coop_blocks(K kernel, int block, size_t smem, long long work_items,
                       int items_per_thread_min) {
    int dev = 0, sms = 0, per_sm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, block, smem);
    long long maxb = (long long)sms * (per_sm > 0 ? per_sm : 1);
    long long want = (work_items + (long long)block * items_per_thread_min - 1) /
                     ((long long)block * items_per_thread_min);
    if (want < 1) want = 1;
    return (int)(want < maxb ? want : maxb);
}

}  // namespace tse
