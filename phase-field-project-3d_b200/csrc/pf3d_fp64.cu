// pf3d_fp64.cu -- FP64 per-subroutine kernels (reference form), diagnostics and
// staging conversions.
// Built with --fmad=false: the reference's gfortran arithmetic on x86-64 has
// no fused multiply-add, so neither may this form.
#include "pf3d_simple.cuh"
#include "pf3d_init.cuh"

namespace pf3d {
template cudaError_t launch_heat<double>(const DomainDesc&, const StepArgs&, const Fields&, cudaStream_t);
template cudaError_t launch_phase<double>(const DomainDesc&, const StepArgs&, const void*, const void*, void*, void*, cudaStream_t);
template cudaError_t launch_solute<double>(const DomainDesc&, const StepArgs&, const void*, const void*, void*, cudaStream_t);
template cudaError_t launch_copy_inner<double>(const DomainDesc&, const void*, void*, cudaStream_t);
template cudaError_t launch_diag<double>(const DomainDesc&, const void*, const void*, double*, int, double*, cudaStream_t);
template cudaError_t launch_convert_in<double>(const DomainDesc&, const double*, void*, long long, long long, cudaStream_t);
template cudaError_t launch_convert_out<double>(const DomainDesc&, const void*, double*, long long, long long, cudaStream_t);
template <>
cudaError_t launch_init_seeded<double>(const DomainDesc& d, const InitArgs& a, const double* sites, void* phi, void* c,
                                  void* Tf, void* dpp, cudaStream_t st)
{
    return launch_init_seeded_impl<double>(d, a, sites, phi, c, Tf, dpp, st);
}
}  // namespace pf3d
