// Shared device helpers: status word, bounded mbarrier waits, 1-D bulk copies.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace ob {

// Bits of the device status word. A kernel that gives up on a bounded wait
// sets kStatusTimeout here and skips the rest of its work instead of hanging;
// the host turns the bit into OB_ERROR_TIMEOUT after the next synchronisation.
constexpr unsigned kStatusTimeout = 1u;
constexpr unsigned kStatusOverflow = 2u;
// An index a valid data structure never holds was found and its access skipped.
constexpr unsigned kStatusInvalid = 4u;

// Upper bound on polls of one mbarrier phase (each poll of try_wait already
// suspends for a hardware-defined interval); well above any legitimate wait.
constexpr uint32_t kSpinLimit = 1u << 24;

__device__ __forceinline__ uint32_t smem_addr(const void *p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count)
                 : "memory");
}

// Makes barrier initialisation visible to the async (TMA) proxy.
__device__ __forceinline__ void fence_barrier_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Orders this thread's earlier generic-proxy shared-memory accesses before
// later async-proxy (bulk copy) writes to the same memory.
__device__ __forceinline__ void fence_proxy_async_shared() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)),
                 "r"(bytes)
                 : "memory");
}

// One-dimensional bulk copy global -> this CTA's shared memory, completing on
// `bar`. dst, src and bytes must be multiples of 16 bytes.
__device__ __forceinline__ void bulk_copy_g2s(void *dst, const void *src, uint32_t bytes,
                                              uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::
            "r"(smem_addr(dst)),
        "l"(src), "r"(bytes), "r"(smem_addr(bar))
        : "memory");
}

// Waits for the given phase parity of `bar`, polling at most kSpinLimit times.
// Returns false (and records kStatusTimeout) if the phase never completes.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, uint32_t parity,
                                                  unsigned *status) {
    const uint32_t addr = smem_addr(bar);
    for (uint32_t poll = 0; poll < kSpinLimit; ++poll) {
        uint32_t done;
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
            " selp.u32 %0, 1, 0, p;\n}\n"
            : "=r"(done)
            : "r"(addr), "r"(parity)
            : "memory");
        if (done) {
            return true;
        }
    }
    if (status != nullptr) {
        atomicOr(status, kStatusTimeout);
    }
    return false;
}

// SFU reciprocal square root (PTX rsqrt.approx.ftz.f32).
__device__ __forceinline__ float rsqrt_approx(float x) {
    float y;
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

__host__ __device__ constexpr uint32_t ceil_div(uint64_t a, uint64_t b) {
    return static_cast<uint32_t>((a + b - 1) / b);
}

} // namespace ob
