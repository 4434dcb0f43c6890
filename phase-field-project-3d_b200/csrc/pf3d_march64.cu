// pf3d_march64.cu -- FP64 instantiation of the TMA-staged z-marching passes
// (single domain).  Built without automatic multiply-add contraction, like
// every unit that inlines the per-cell arithmetic.
#include "pf3d_march.cuh"

namespace pf3d {
template cudaError_t launch_march_first<double>(const CUtensorMap&, const DomainDesc&, const StepArgs&, const Fields&, bool, int, int, int, int*, cudaStream_t);
template cudaError_t launch_march_last<double>(const CUtensorMap&, const DomainDesc&, const StepArgs&, const Fields&, int, int, int, int*, cudaStream_t);
}  // namespace pf3d
