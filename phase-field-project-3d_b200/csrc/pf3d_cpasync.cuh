// pf3d_cpasync.cuh -- element-wise asynchronous global-to-shared copies
// (cp.async, Ampere and later) used to prefetch the next plane of the
// z-marching windows while the current plane is computed.
#pragma once

namespace pf3d {

__device__ __forceinline__ void cp_async_elem(void* smem, const void* gmem, int bytes)
{
    unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    if (bytes == 8)
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem));
    else
        asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(gmem));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }
// all but the most recently committed group have landed
__device__ __forceinline__ void cp_async_wait_prev() { asm volatile("cp.async.wait_group 1;\n" ::: "memory"); }

}  // namespace pf3d
