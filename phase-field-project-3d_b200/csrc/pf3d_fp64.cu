// pf3d_fp64.cu -- FP64 per-subroutine kernels (reference form), diagnostics and
// staging conversions.
// Built with --fmad=false: the reference's gfortran arithmetic on x86-64 has
// no fused multiply-add, so neither may this form.
#include "pf3d_simple.cuh"
#include "pf3d_init.cuh"
#include "pf3d_track.cuh"
#include "pf3d_frame.cuh"

namespace pf3d {
template cudaError_t launch_heat<double>(const DomainDesc&, const StepArgs&, const Fields&, cudaStream_t);
template cudaError_t launch_phase<double>(const DomainDesc&, const StepArgs&, const void*, const void*, void*, void*, cudaStream_t);
template cudaError_t launch_solute<double>(const DomainDesc&, const StepArgs&, const void*, const void*, void*, cudaStream_t);
template cudaError_t launch_copy_inner<double>(const DomainDesc&, const void*, void*, cudaStream_t);
template cudaError_t launch_diag<double>(const DomainDesc&, const void*, const void*, const void*, const void*, double*, int, double*, cudaStream_t);
template cudaError_t launch_convert_in<double>(const DomainDesc&, const double*, void*, long long, long long, cudaStream_t);
template cudaError_t launch_convert_out<double>(const DomainDesc&, const void*, double*, long long, long long, cudaStream_t);
template <>
cudaError_t launch_init_seeded<double>(const DomainDesc& d, const InitArgs& a, const double* sites, void* phi, void* c,
                                  void* Tf, void* dpp, cudaStream_t st)
{
    return launch_init_seeded_impl<double>(d, a, sites, phi, c, Tf, dpp, st);
}
template <>
cudaError_t launch_track<double>(const DomainDesc& d, const void* phi, unsigned long long* scratch, double* out,
                             cudaStream_t st)
{
    return launch_track_impl<double>(d, phi, scratch, out, st);
}
template <>
cudaError_t launch_shift_frame<double>(const DomainDesc& d, int kd, const void* phi_o, const void* c_o, void* phi_n,
                                   void* c_n, cudaStream_t st)
{
    return launch_shift_frame_impl<double>(d, kd, phi_o, c_o, phi_n, c_n, st);
}
template <>
cudaError_t launch_fill<double>(void* a, long long n, double v, cudaStream_t st)
{
    return launch_fill_impl<double>(a, n, v, st);
}
}  // namespace pf3d
