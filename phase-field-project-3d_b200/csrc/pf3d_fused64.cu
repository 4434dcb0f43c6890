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

__global__ void k_math_log(const double* __restrict__ x, double* __restrict__ own, double* __restrict__ lib,
                           long long n)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const double v = x[i];
        own[i] = Ar<double>::lg(v);
        lib[i] = log(v);
    }
}

cudaError_t launch_math_log(const double* x, double* own, double* lib, long long n, cudaStream_t st)
{
    if (n <= 0) return cudaSuccess;
    const long long want = (n + 255) / 256;
    const int grid = (int)(want < 148 * 8 ? want : 148 * 8);
    k_math_log<<<grid, 256, 0, st>>>(x, own, lib, n);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? cudaStreamSynchronize(st) : e;
}
}  // namespace pf3d
