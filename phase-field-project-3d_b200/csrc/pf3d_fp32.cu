// pf3d_fp32.cu -- FP32 instantiation of every kernel (fields and stencils in FP32;
// diagnostics still accumulate in FP64).
#include "pf3d_simple.cuh"
#include "pf3d_init.cuh"
#include "pf3d_track.cuh"
#include "pf3d_frame.cuh"
#include "pf3d_fused.cuh"
#include "pf3d_fused_pair.cuh"

namespace pf3d {
template cudaError_t launch_heat<float>(const DomainDesc&, const StepArgs&, const Fields&, cudaStream_t);
template cudaError_t launch_phase<float>(const DomainDesc&, const StepArgs&, const void*, const void*, void*, void*, cudaStream_t);
template cudaError_t launch_solute<float>(const DomainDesc&, const StepArgs&, const void*, const void*, void*, cudaStream_t);
template cudaError_t launch_copy_inner<float>(const DomainDesc&, const void*, void*, cudaStream_t);
template cudaError_t launch_fused_first<float>(const DomainDesc&, const StepArgs&, const Fields&, bool, int, int, cudaStream_t);
template cudaError_t launch_fused_last<float>(const DomainDesc&, const StepArgs&, const Fields&, int, int, cudaStream_t);
template cudaError_t launch_diag<float>(const DomainDesc&, const void*, const void*, const void*, const void*, double*, int, double*, cudaStream_t);
template cudaError_t launch_convert_in<float>(const DomainDesc&, const double*, void*, long long, long long, cudaStream_t);
template cudaError_t launch_convert_out<float>(const DomainDesc&, const void*, double*, long long, long long, cudaStream_t);
template cudaError_t launch_fused_batch<float>(const BatchDomain*, const BatchStep*, const BatchItem*, const int*, int, bool, bool, int, int, int, cudaStream_t);
template <>
cudaError_t launch_init_seeded<float>(const DomainDesc& d, const InitArgs& a, const double* sites, void* phi, void* c,
                                  void* Tf, void* dpp, cudaStream_t st)
{
    return launch_init_seeded_impl<float>(d, a, sites, phi, c, Tf, dpp, st);
}
template <>
cudaError_t launch_track<float>(const DomainDesc& d, const void* phi, unsigned long long* scratch, double* out,
                             cudaStream_t st)
{
    return launch_track_impl<float>(d, phi, scratch, out, st);
}
template <>
cudaError_t launch_shift_frame<float>(const DomainDesc& d, int kd, const void* phi_o, const void* c_o, void* phi_n,
                                   void* c_n, cudaStream_t st)
{
    return launch_shift_frame_impl<float>(d, kd, phi_o, c_o, phi_n, c_n, st);
}
template <>
cudaError_t launch_fill<float>(void* a, long long n, double v, cudaStream_t st)
{
    return launch_fill_impl<float>(a, n, v, st);
}
template cudaError_t launch_fused_first_pair<float>(const DomainDesc&, const StepArgs&, const Fields&, bool, int, cudaStream_t);
template cudaError_t launch_fused_last_pair<float>(const DomainDesc&, const StepArgs&, const Fields&, int, cudaStream_t);
template cudaError_t launch_fused_batch_pair<float>(const BatchDomain*, const BatchStep*, const BatchItem*, const int*, int, bool, int, int, cudaStream_t);
}  // namespace pf3d
