// sbf_flush.cuh -- per-thread staging ring for 32-byte bulk OR-reductions
// into the filter's shards, shared by the tile kernels (sbf_tile.cuh) and
// the run-time compiled generic kernels (sbf_generic.cuh).
#pragma once

#include "sbf_device.cuh"
#include "sbf_internal.h"

namespace sbf {

// A run's four word masks are merged into its shard with one 32-byte TMA
// bulk reduction (cp.reduce.async.bulk .or.b64) from a shared-memory staging
// slot: one L2 sector operation instead of four 8-byte atomics.  Each thread
// cycles through kFlushSlots slots; before reusing a slot it waits until the
// bulk operation issued kFlushSlots flushes earlier has read it.
struct FlushRing {
    uint64_t* slot0;  // this thread's slot 0; slot k at slot0 + k * kThreads * 4
    uint32_t count;
};

__device__ __forceinline__ void flush_run(uint64_t* words, uint32_t shard, const uint64_t a[4],
                                          FlushRing& ring) {
    static_assert(kFlushSlots == 8, "wait_group.read immediate below assumes 8 slots");
    uint64_t* slot = ring.slot0 + (ring.count & (kFlushSlots - 1)) * (kThreads * 4);
    asm volatile("cp.async.bulk.wait_group.read 7;" ::: "memory");
    *reinterpret_cast<ulonglong2*>(slot) = make_ulonglong2(a[0], a[1]);
    *reinterpret_cast<ulonglong2*>(slot + 2) = make_ulonglong2(a[2], a[3]);
    fence_proxy_async_smem();
    asm volatile(
        "cp.reduce.async.bulk.global.shared::cta.bulk_group.or.b64 [%0], [%1], 32;" ::"l"(
            words + static_cast<uint64_t>(shard) * 4),
        "r"(smem_addr(slot))
        : "memory");
    asm volatile("cp.async.bulk.commit_group;" ::: "memory");
    ++ring.count;
}

// flush_run as predicated instructions: the insert kernels call it for every
// window with `pred` set where a run ends, so no lane of a warp branches (some
// lane ends a run on almost every window).
__device__ __forceinline__ void flush_run_if(uint32_t pred, uint64_t* words, uint32_t shard,
                                             const uint64_t a[4], FlushRing& ring) {
    static_assert(kFlushSlots == 8, "wait_group.read immediate below assumes 8 slots");
    uint64_t* slot = ring.slot0 + (ring.count & (kFlushSlots - 1)) * (kThreads * 4);
    const uint64_t* g = words + static_cast<uint64_t>(shard) * 4;
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.u32 p, %0, 0;\n\t"
        "@p cp.async.bulk.wait_group.read 7;\n\t"
        "@p st.shared.v2.u64 [%1], {%2, %3};\n\t"
        "@p st.shared.v2.u64 [%1+16], {%4, %5};\n\t"
        "@p fence.proxy.async.shared::cta;\n\t"
        "@p cp.reduce.async.bulk.global.shared::cta.bulk_group.or.b64 [%6], [%1], 32;\n\t"
        "@p cp.async.bulk.commit_group;\n\t}" ::"r"(pred),
        "r"(smem_addr(slot)), "l"(a[0]), "l"(a[1]), "l"(a[2]), "l"(a[3]), "l"(g)
        : "memory");
    ring.count += pred;
}

__device__ __forceinline__ void flush_ring_drain() {
    // Every bulk reduction issued by this thread has completed (its global
    // writes performed and its shared-memory slot read).
    asm volatile("cp.async.bulk.wait_group 0;" ::: "memory");
}

}  // namespace sbf
