// tc_tma.cuh -- tensor-memory-accelerator tile loads (cp.async.bulk.tensor)
// completing on a shared-memory mbarrier, for tiles of this GPU's own
// memory.  No cluster multicast is used anywhere.  Every wait is bounded: it
// gives up after a fixed number of polls and reports it.
#pragma once

#include <cuda.h>
#include <cstdint>

#include "tc_cpasync.cuh"

namespace tc {

__device__ __forceinline__ void mbar_init(uint64_t *bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_addr(bar)), "r"(count)
                 : "memory");
}
// make the initialised barriers visible to the tensor-copy unit
__device__ __forceinline__ void mbar_fence_init() {
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
}
// order this thread's earlier generic-proxy shared accesses before later
// async-proxy (tensor copy) accesses to the same shared memory
__device__ __forceinline__ void fence_proxy_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_addr(bar)),
                 "r"(bytes)
                 : "memory");
}
// one 3-D tile of the tensor map into shared memory; completion counted on bar
__device__ __forceinline__ void tma_load_3d(void *dst, const CUtensorMap *map, int x, int y, int z,
                                            uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3, %4}], [%5];\n" ::"r"(smem_addr(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(smem_addr(bar))
        : "memory");
}
// wait for the barrier's phase `parity` to complete; false after `limit`
// polls without completion
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, unsigned parity, unsigned limit) {
    for (unsigned i = 0; i < limit; ++i) {
        unsigned done = 0;
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
            " selp.u32 %0, 1, 0, p;\n}\n"
            : "=r"(done)
            : "r"(smem_addr(bar)), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

}  // namespace tc
