// pf3d_march32b.cu -- FP32 instantiation of the TMA-staged z-marching passes
// over a batch's work list.
#include "pf3d_march.cuh"

namespace pf3d {
template cudaError_t launch_march_batch<float>(const BatchDomain*, const CUtensorMap*, const BatchStep*, const BatchItem*, const int*, int, bool, bool, int, int, int, int, int*, int*, cudaStream_t);
}  // namespace pf3d
