// Bulk asynchronous copies between global and shared memory (the TMA unit): the untiled
// one-dimensional form (cp.async.bulk) for kernels whose tiles are contiguous blocks, and
// the tiled tensor form for boxes of strided blocks.
//
//  loads   one elected thread arms an mbarrier with the byte count and issues the copy;
//          every consumer waits on the barrier's phase (bounded: a wait that runs out
//          returns false, the kernel records it and leaves).
//  stores  the writing threads fence their shared-memory writes into the async proxy,
//          a barrier orders them before the elected thread's copy, and the copy's
//          reads of shared memory are awaited before the buffer is reused or the CTA
//          exits.
// Addresses must be 16-byte aligned and sizes multiples of 16 bytes.  No form with
// cluster multicast is used: every copy moves this CTA's own tile of this GPU's memory.
#pragma once
#include <cstdint>

namespace pfc {

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
// makes the initialisation visible to the async proxy (the bulk copies' completion)
__device__ __forceinline__ void mbar_init_fence() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.release.cta.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
                 "r"(bytes)
                 : "memory");
}

// global -> shared, completion counted on bar
__device__ __forceinline__ void bulk_load(void* smem_dst, const void* gsrc, unsigned bytes, uint64_t* bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(smem_dst)),
                 "l"(gsrc), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}

// Waits for the completion of phase `parity` of bar; false when `limit` polls (each of
// which may suspend the thread for a while) did not see it.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, unsigned parity, unsigned limit) {
    const uint32_t a = smem_u32(bar);
    for (unsigned i = 0; i < limit; ++i) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(a), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

// this thread's shared-memory writes become visible to a following bulk store
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// shared -> global, in the current bulk group
__device__ __forceinline__ void bulk_store(void* gdst, const void* smem_src, unsigned bytes) {
    asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;" ::"l"(gdst), "r"(smem_u32(smem_src)),
                 "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
// the issuing thread waits until every committed store has read its shared memory
__device__ __forceinline__ void bulk_wait_read() { asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory"); }

// Tiled tensor copies (cp.async.bulk.tensor) of one box of a five-dimensional tensor map
// passed as a __grid_constant__ kernel parameter; c0 is the innermost coordinate (kept a
// multiple of 16 bytes by the callers: always 0 here).  No multicast form.
__device__ __forceinline__ void tma_load5(void* smem_dst, const void* tmap, int c0, int c1, int c2, int c3, int c4,
                                          uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.5d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, "
        "%5, %6}], [%7];" ::"r"(smem_u32(smem_dst)),
        "l"(reinterpret_cast<uint64_t>(tmap)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(c4), "r"(smem_u32(bar))
        : "memory");
}
__device__ __forceinline__ void tma_store5(const void* tmap, const void* smem_src, int c0, int c1, int c2, int c3,
                                           int c4) {
    asm volatile(
        "cp.async.bulk.tensor.5d.global.shared::cta.tile.bulk_group [%0, {%1, %2, %3, %4, %5}], [%6];" ::"l"(
            reinterpret_cast<uint64_t>(tmap)),
        "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(c4), "r"(smem_u32(smem_src))
        : "memory");
}

// Polls of mbar_wait before a device wait counts as lost (each poll may suspend for up
// to about a microsecond: seconds in total, far beyond any copy's latency).
constexpr unsigned kWaitPolls = 1u << 22;
// Bit of the stepper's device status word that a timed-out wait sets.
constexpr int kFlagWaitTimeout = 2;

}  // namespace pfc
