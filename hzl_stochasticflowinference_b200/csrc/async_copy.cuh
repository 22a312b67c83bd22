// Bulk asynchronous global->shared copies (the TMA bulk-copy engine of sm_90/sm_100a) with
// mbarrier completion, shared->global copies in bulk async-groups, and the waits on them.  Every wait is bounded: a wait that gives up
// reports failure so the caller can set STATUS_TIMEOUT and leave the kernel instead of hanging.
#pragma once
#include <cstdint>

namespace hzlb {

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t arrivals) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(arrivals)
                 : "memory");
}
__device__ __forceinline__ void mbar_init_fence() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
// Orders this thread's earlier generic-proxy shared-memory accesses before later async-proxy
// (bulk copy) writes to the same buffer.
__device__ __forceinline__ void fence_proxy_async_shared() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
// One arrival that also raises the barrier's expected transaction count by `bytes`.
__device__ __forceinline__ void mbar_arrive_expect(uint64_t *bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
                 "r"(bytes)
                 : "memory");
}
// Bulk copy of `bytes` (multiple of 16; both addresses 16-byte aligned) completing on `bar`.
__device__ __forceinline__ void bulk_copy_g2s(void *dst, const void *src, uint32_t bytes,
                                              uint64_t *bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, "
                 "[%3];" ::"r"(smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}
// Bulk copy shared -> global of `bytes` (multiple of 16; both addresses 16-byte aligned), in
// this thread's current bulk async-group.  Whole 16-byte chunks reach L2 as full sectors, so
// no partially written sector waits there for a fill from DRAM.
__device__ __forceinline__ void bulk_copy_s2g(void *dst, const void *src, uint32_t bytes) {
    asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;" ::"l"(dst),
                 "r"(smem_u32(src)), "r"(bytes)
                 : "memory");
}
// Tiled tensor copy shared -> global of one box of `map` at coordinates (x, y, z), in this
// thread's current bulk async-group (the map lies in kernel-parameter space).
__device__ __forceinline__ void tensor_store_3d(const void *map, const void *src, int x, int y,
                                                int z) {
    asm volatile("cp.async.bulk.tensor.3d.global.shared::cta.bulk_group [%0, {%2, %3, %4}], [%1];"
                 ::"l"(map), "r"(smem_u32(src)), "r"(x), "r"(y), "r"(z)
                 : "memory");
}
__device__ __forceinline__ void bulk_commit() {
    asm volatile("cp.async.bulk.commit_group;" ::: "memory");
}
// Waits until every committed shared -> global copy of this thread has read its source.
__device__ __forceinline__ void bulk_wait_read_all() {
    asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
}
// Waits until every committed shared -> global copy of this thread has completed.
__device__ __forceinline__ void bulk_wait_all() {
    asm volatile("cp.async.bulk.wait_group 0;" ::: "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
    uint32_t done;
    asm volatile("{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
                 " selp.u32 %0, 1, 0, p;\n}"
                 : "=r"(done)
                 : "r"(smem_u32(bar)), "r"(parity)
                 : "memory");
    return done != 0;
}
__device__ __forceinline__ uint64_t global_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
// Waits for the phase with the given parity to complete; gives up (false) after `limit_ns`
// nanoseconds of the global timer (one second by default), or at the latest after 2^26 polls,
// so a phase that never completes costs about a second, never a hang.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, uint32_t parity,
                                                  uint64_t limit_ns = 1000000000ull) {
    if (mbar_try_wait(bar, parity))
        return true;
    const uint64_t start = global_ns();
    for (uint32_t i = 0; i < (1u << 26); ++i) {
        if (mbar_try_wait(bar, parity))
            return true;
        if ((i & 63) == 63 && global_ns() - start > limit_ns)
            return false;
    }
    return false;
}

} // namespace hzlb
