// pf3d_tma.cuh -- tensor-memory-accelerator (TMA) plane loads and the
// shared-memory barriers (mbarrier) they complete on, for sm_100a.
//
// A z-marching tile stages each plane of its input phase field (the tile plus
// its halo) with one cp.async.bulk.tensor load issued by a single thread; the
// load signals a per-slot mbarrier with its byte count, and every thread that
// reads the slot waits on that barrier's phase.  No load here uses cluster
// multicast: every tensor map covers this GPU's own memory.
//
// Every wait is bounded: after kWaitLimit polls it gives up and reports
// failure, and the caller records an error status for the host instead of
// spinning for ever.
#pragma once
#include <cstdint>
#include <cuda.h>

namespace pf3d {

// polls of mbarrier.try_wait before a wait gives up (each poll may suspend
// the thread for a hardware-chosen interval; a plane load takes microseconds)
constexpr int kWaitLimit = 1 << 22;

// error codes a kernel leaves in the context's status word
constexpr int kErrTmaTimeout = 1;

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

// makes the initialised barriers visible to the asynchronous proxy (TMA)
__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }

// orders this CTA's earlier generic-proxy accesses of shared memory before
// later asynchronous-proxy writes (a TMA load into a slot threads have read)
__device__ __forceinline__ void fence_proxy_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void mbar_arrive_expect_tx(uint32_t bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}

// 3-D tiled load of the tensor map's box at element coordinates (x, y, z)
// into shared memory at dst; completes `bar`'s transaction count.  x times
// the element size must be a multiple of 16 bytes; y, z and a negative x
// start are free (elements outside the tensor read as zero).
__device__ __forceinline__ void tma_load_3d(uint32_t dst, const CUtensorMap* tm, int x, int y, int z, uint32_t bar)
{
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
        "[%5];" ::"r"(dst),
        "l"(tm), "r"(x), "r"(y), "r"(z), "r"(bar)
        : "memory");
}

// waits for the phase of `bar` with the given parity; false after kWaitLimit polls
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity)
{
    for (int i = 0; i < kWaitLimit; ++i) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(bar), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

__device__ __forceinline__ void prefetch_tensormap(const CUtensorMap* tm)
{
    asm volatile("prefetch.tensormap [%0];" ::"l"(tm) : "memory");
}

}  // namespace pf3d
