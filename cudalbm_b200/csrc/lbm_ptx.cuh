// lbm_ptx.cuh -- inline-PTX helpers shared by the step kernels and the
// closure network: shared-memory addresses, mbarriers (bounded waits), the CTA
// barrier, and the TMA tile load of the moment planes.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdint>

namespace lbm {

__device__ __forceinline__ unsigned smem_u32(const void *p)
{
    return static_cast<unsigned>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, unsigned parity)
{
    unsigned ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
__device__ __forceinline__ uint64_t global_ns()
{
    uint64_t t;
    asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
    return t;
}
// Bounded wait: gives up after `limit_ns` and reports false.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, unsigned parity, uint64_t limit_ns)
{
    if (mbar_try_wait(bar, parity))
        return true;
    const uint64_t t0 = global_ns();
    for (;;) {
        for (int k = 0; k < 32; k++)
            if (mbar_try_wait(bar, parity))
                return true;
        if (global_ns() - t0 > limit_ns)
            return false;
    }
}
// CTA-wide barrier.  Each warp first reconverges (__syncwarp), then the CTA
// synchronises; a warp split across divergent paths when it reaches a CTA
// barrier can be released only in part.
__device__ __forceinline__ void cta_sync()
{
    __syncwarp();
    asm volatile("barrier.sync 0;" ::: "memory");
}

// Thread-0 work as predicated instructions executed by the whole warp, so
// that no branch splits warp 0 (every thread calls these; only those with
// `pred` act).
//   TMA issue: make earlier ordinary reads of the slot visible to the async
//   proxy, arm the slot's mbarrier with the plane's bytes, start the copy.
__device__ __forceinline__ void tma_issue_if(bool pred, void *dst, const CUtensorMap *map, int c0, int c1, int c2,
                                             int c3, uint64_t *bar, unsigned bytes)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.u32 p, %8, 0;\n\t"
        "@p fence.proxy.async.shared::cta;\n\t"
        "@p mbarrier.arrive.expect_tx.shared::cta.b64 _, [%6], %7;\n\t"
        "@p cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], "
        "[%6];\n\t}" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(smem_u32(bar)), "r"(bytes),
        "r"(unsigned(pred))
        : "memory");
}
//   mbarrier set-up: count 1 (the arming thread), then publish the init.
__device__ __forceinline__ void mbar_init_if(bool pred, uint64_t *bar)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.u32 p, %1, 0;\n\t"
        "@p mbarrier.init.shared::cta.b64 [%0], 1;\n\t}" ::"r"(smem_u32(bar)),
        "r"(unsigned(pred))
        : "memory");
}
__device__ __forceinline__ void fence_mbar_init_if(bool pred)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.u32 p, %0, 0;\n\t"
        "@p fence.mbarrier_init.release.cluster;\n\t}" ::"r"(unsigned(pred))
        : "memory");
}

}  // namespace lbm
