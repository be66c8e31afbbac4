// Bulk asynchronous copies (cp.async.bulk, global -> shared), their
// mbarriers, L2 eviction hints and the bounded waits the staged sweeps build
// on.  Shared by the FP32 correction sweeps and the FP64 persistent solves.
#pragma once

#include "tse_common.cuh"

namespace tse {

__device__ __forceinline__ unsigned smem_u32(const void* p) {
    return static_cast<unsigned>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

// the stage's single arrival, adding `bytes` to its transaction count
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
                 "r"(bytes)
                 : "memory");
}

// adds `bytes` to the transaction count without arriving
__device__ __forceinline__ void mbar_add_tx(uint64_t* bar, unsigned bytes) {
    asm volatile("mbarrier.expect_tx.relaxed.cta.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)),
                 "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, unsigned parity) {
    unsigned done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return done != 0;
}

// bulk copy global -> this CTA's shared memory; 16-byte aligned, size % 16 == 0
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, unsigned bytes, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
        ::"r"(smem_u32(dst)), "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}

// L2 eviction priority.  Per iteration a sweep streams each cell's
// coefficients once (far more than L2 holds), while the solution arrays (the
// FP32 corrections, or the FP64 solution) are reread by the next phase's
// windows: the stream is marked evict-first and the solution evict-last, so
// the solution stays in L2 instead of being pushed out by the stream.
#ifndef TSE_TMA_HINTS
#define TSE_TMA_HINTS 1
#endif
__device__ __forceinline__ uint64_t l2_evict_first() {
    uint64_t p;
    asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
    return p;
}
__device__ __forceinline__ uint64_t l2_evict_last() {
    uint64_t p;
    asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
    return p;
}

__device__ __forceinline__ void bulk_g2s_hint(void* dst, const void* src, unsigned bytes, uint64_t* bar,
                                              uint64_t policy) {
#if TSE_TMA_HINTS
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint"
        " [%0], [%1], %2, [%3], %4;"
        ::"r"(smem_u32(dst)), "l"(src), "r"(bytes), "r"(smem_u32(bar)), "l"(policy)
        : "memory");
#else
    bulk_g2s(dst, src, bytes, bar);
#endif
}

__device__ __forceinline__ void st_hint(float* p, float v, uint64_t policy) {
#if TSE_TMA_HINTS
    asm volatile("st.global.L2::cache_hint.f32 [%0], %1, %2;" ::"l"(p), "f"(v), "l"(policy) : "memory");
#else
    *p = v;
#endif
}

__device__ __forceinline__ void st_hint(double* p, double v, uint64_t policy) {
#if TSE_TMA_HINTS
    asm volatile("st.global.L2::cache_hint.f64 [%0], %1, %2;" ::"l"(p), "d"(v), "l"(policy) : "memory");
#else
    *p = v;
#endif
}

// orders this thread's generic-proxy global accesses with async-proxy copies
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async;" ::: "memory"); }

// bounded wait for a stage; false after kBarrierTimeoutNs
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, unsigned parity) {
    if (mbar_try_wait(bar, parity)) return true;
    const uint64_t t0 = globaltimer();
    unsigned spins = 0;
    while (!mbar_try_wait(bar, parity)) {
        if ((++spins & 63u) == 0u && globaltimer() - t0 > kBarrierTimeoutNs) return false;
    }
    return true;
}

// wait for a phase of `bar`; gives up (false) when the block's error flag is
// raised or after kBarrierTimeoutNs, raising the flag
__device__ __forceinline__ bool mbar_wait_flag(uint64_t* bar, unsigned parity, volatile int* err,
                                               unsigned long long timeout_ns = kBarrierTimeoutNs) {
    if (mbar_try_wait(bar, parity)) return true;
    const uint64_t t0 = globaltimer();
    unsigned spins = 0;
    while (!mbar_try_wait(bar, parity)) {
        if (*err) return false;
        if ((++spins & 63u) == 0u && globaltimer() - t0 > timeout_ns) {
            *err = 1;
            return false;
        }
    }
    return true;
}

}  // namespace tse
