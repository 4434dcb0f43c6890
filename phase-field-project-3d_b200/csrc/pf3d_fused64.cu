// pf3d_fused64.cu -- FP64 instantiation of the fused z-marching passes.
// The fused passes use the fast form of the per-cell arithmetic (explicit
// multiply-adds; FP64 throughout; results within 1e-12 of the reference form).
#include "pf3d_fused.cuh"
#include "pf3d_fused_pair.cuh"

namespace pf3d {
template cudaError_t launch_fused_first<double>(const DomainDesc&, const StepArgs&, const Fields&, bool, int, int, cudaStream_t);
template cudaError_t launch_fused_last<double>(const DomainDesc&, const StepArgs&, const Fields&, int, int, cudaStream_t);
template cudaError_t launch_fused_batch<double>(const BatchDomain*, const BatchStep*, const BatchItem*, const int*, int, bool, bool, int, int, int, cudaStream_t);
template cudaError_t launch_fused_first_pair<double>(const DomainDesc&, const StepArgs&, const Fields&, bool, int, cudaStream_t);
template cudaError_t launch_fused_last_pair<double>(const DomainDesc&, const StepArgs&, const Fields&, int, cudaStream_t);
template cudaError_t launch_fused_batch_pair<double>(const BatchDomain*, const BatchStep*, const BatchItem*, const int*, int, bool, int, int, cudaStream_t);
}  // namespace pf3d
