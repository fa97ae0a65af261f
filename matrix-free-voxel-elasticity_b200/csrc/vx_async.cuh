// Asynchronous copies and CTA-scope mbarriers shared by the streaming kernels.
#pragma once

#include "vx_common.cuh"

namespace vx {

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
// cp.async of 4, 8 or 16 bytes (L1-allocating)
template <int BYTES>
__device__ __forceinline__ void cp_async(void* dst, const void* src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], %2;" ::"r"(smem_u32(dst)), "l"(src), "n"(BYTES) : "memory");
}
// 16 bytes, L1 bypassed (streamed data)
__device__ __forceinline__ void cp_async_cg16(void* dst, const void* src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
    asm volatile("{\n\t.reg .b64 st;\n\tmbarrier.arrive.shared::cta.b64 st, [%0];\n\t}" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, unsigned parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Device fault flag of the streaming kernels: set when a bounded wait ran out (never in a correct
// run).  Read and cleared by vx_device_status.
__device__ int g_stream_fault;
constexpr int STREAM_WAIT_LIMIT = 1 << 22;

// Bounded wait of a whole warp for the phase `parity` of `bar` (the outcome is warp-uniform); gives
// up early once another warp of the CTA aborted.  Returns false when the wait ran out or the CTA
// aborted; running out raises the fault flag and aborts the CTA.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, unsigned parity, volatile int* abort_flag) {
    for (int i = 0; i < STREAM_WAIT_LIMIT; ++i) {
        const bool ok = mbar_try_wait(bar, parity);
        if (__all_sync(0xffffffffu, ok)) return true;
        if (__any_sync(0xffffffffu, *abort_flag != 0)) return false;
    }
    if ((threadIdx.x & 31) == 0) {
        atomicExch(&g_stream_fault, 1);
        *abort_flag = 1;
    }
    __syncwarp();
    return false;
}

}  // namespace vx
