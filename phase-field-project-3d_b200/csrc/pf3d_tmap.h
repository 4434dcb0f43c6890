// pf3d_tmap.h -- host side of the TMA plane loads: the tensor map of one
// pitched field (Fortran order, i fastest), encoded through the driver's
// cuTensorMapEncodeTiled (reached through the runtime, no -lcuda).
#pragma once
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>
#include <mutex>

namespace pf3d {

inline PFN_cuTensorMapEncodeTiled_v12000 tmap_encoder()
{
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
        cudaGetLastError();
    });
    return fn;
}

// Tensor map of an nx x ny x nz field of es-byte elements at `base` with row
// pitch px elements (plane stride px*ny), read in boxes of box_x x box_y x 1
// cells; cells outside the field read as zero.  0 on success.
inline int encode_field_map(CUtensorMap* tm, const void* base, int es, int nx, int ny, int nz, long long px,
                            int box_x, int box_y)
{
    auto enc = tmap_encoder();
    if (!enc) return -1;
    const cuuint64_t dims[3] = {(cuuint64_t)nx, (cuuint64_t)ny, (cuuint64_t)nz};
    const cuuint64_t strides[2] = {(cuuint64_t)(px * es), (cuuint64_t)(px * ny * es)};
    const cuuint32_t box[3] = {(cuuint32_t)box_x, (cuuint32_t)box_y, 1};
    const cuuint32_t estr[3] = {1, 1, 1};
    const CUresult r = enc(tm, es == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3,
                           const_cast<void*>(base), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                           CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                           CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS ? 0 : (int)r;
}

// the phase-field box of the march kernels' 32 x TY tiles: the tile plus a
// 2-cell halo, widened in x so that its start is 16-byte aligned
inline int march_box_x(int es) { return 32 + 2 * (es == 8 ? 2 : 4); }
inline int march_box_y(int tile_y) { return tile_y + 4; }

}  // namespace pf3d
