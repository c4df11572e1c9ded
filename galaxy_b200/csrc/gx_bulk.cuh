// gx_bulk.cuh -- bulk copies (global -> this CTA's shared memory, no
// multicast) completed on an mbarrier, with bounded waits.
//
// A wait gives up after SPIN_LIMIT polls and returns false; the caller then
// raises the context's device error word, waits (again bounded) for its own
// copies in flight and returns, so that a kernel never spins without end.
#pragma once
#include <cstdint>

namespace {
constexpr uint32_t SPIN_LIMIT = 1u << 22;  // try_wait polls before giving up

__device__ __forceinline__ uint32_t su32(const void* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint64_t* b, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(su32(b)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_fence_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ bool mbar_try(uint64_t* b, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(su32(b)), "r"(parity)
        : "memory");
    return ok != 0;
}
__device__ __forceinline__ bool mbar_wait(uint64_t* b, uint32_t parity) {
    for (uint32_t i = 0; i < SPIN_LIMIT; i++)
        if (mbar_try(b, parity)) return true;
    return false;
}
__device__ __forceinline__ void mbar_arrive(uint64_t* b) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(su32(b)) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* b, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(su32(b)), "r"(bytes)
                 : "memory");
}
// global -> own shared memory, no multicast; both addresses 16-byte aligned,
// bytes a multiple of 16
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* b) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            su32(dst)),
        "l"(src), "r"(bytes), "r"(su32(b))
        : "memory");
}
}  // namespace
