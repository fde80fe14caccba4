// mbarrier, 1D bulk-copy (TMA) and bounded-wait helpers shared by the staged kernels of the 2D and 3D engines.  Every
// bulk copy reads this GPU's own global memory into the issuing CTA's shared memory (no multicast), with 16-byte
// aligned addresses and sizes; every wait is bounded by %globaltimer.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#define TB_WAIT_NS 2000000000ull          // bound of one mbarrier wait (2 s): then the error flag is set

__device__ __forceinline__ uint32_t tb_smem_addr(const void *ptr) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(ptr));
}

__device__ __forceinline__ void tb_mbar_init(uint64_t *bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(tb_smem_addr(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void tb_mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(tb_smem_addr(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool tb_mbar_try_wait(uint64_t *bar, uint32_t parity) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(tb_smem_addr(bar)), "r"(parity)
        : "memory");
    return done != 0;
}

__device__ __forceinline__ uint64_t tb_globaltimer() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Wait for the mbarrier phase of `parity`, at most TB_WAIT_NS; warp-uniform result.
__device__ __forceinline__ bool tb_mbar_wait(uint64_t *bar, uint32_t parity) {
    bool done = tb_mbar_try_wait(bar, parity);
    if (!done) {
        const uint64_t t0 = tb_globaltimer();
        while (!(done = tb_mbar_try_wait(bar, parity)))
            if (tb_globaltimer() - t0 > TB_WAIT_NS) break;
    }
    return __all_sync(0xffffffffu, done);
}

// One bulk copy global -> shared completing on `bar` (16-byte aligned addresses, bytes a multiple of 16).
__device__ __forceinline__ void tb_bulk_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     tb_smem_addr(dst)),
                 "l"(src), "r"(bytes), "r"(tb_smem_addr(bar))
                 : "memory");
}

__device__ __forceinline__ void tb_fence_proxy_async() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

