// pf3d_frame.cuh -- moving frame on the device.
//
// The reference moves its frame by hand: it writes a Tecplot snapshot, and a
// new run reads it back with tipo_inicial = 4 and a shift of k_desl planes
// (entrada.f90:284-321, ler_restart): plane k of the file goes to k - k_desl,
// the k_desl top planes become liquid (phi = 0) with the concentration of the
// file's top plane in that column, conc_soluto_new = conc_soluto_old, and the
// rest of the state is entrada's initial fill (phase_field_new = 0, TOLD =
// TNEW = T0, DPP = 0, entrada.f90:239-262).  Here the same state is produced
// on the device from the context's current fields, with no file in between.
#pragma once
#include "pf3d_launch.h"

namespace pf3d {

// phi_n / c_n <- phi_o / c_o shifted down by kd planes, liquid on top
template <typename T>
__global__ void k_shift_frame(DomainDesc d, int kd, const T* __restrict__ phi_o, const T* __restrict__ c_o,
                              T* __restrict__ phi_n, T* __restrict__ c_n)
{
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y;
    if (x >= d.nx) return;
    const long long col = (long long)x + (long long)y * d.px;
    const T c_top = c_o[col + (long long)(d.nz - 1) * d.plane];
    for (int z = blockIdx.z; z < d.nz; z += gridDim.z) {
        const long long dst = col + (long long)z * d.plane;
        const int zs = z + kd;
        if (zs < d.nz) {
            const long long src = col + (long long)zs * d.plane;
            phi_n[dst] = phi_o[src];
            c_n[dst] = c_o[src];
        } else {
            phi_n[dst] = (T)0;
            c_n[dst] = c_top;
        }
    }
}

// every element of a field (padding included) <- v
template <typename T>
__global__ void k_fill(T* __restrict__ a, long long n, T v)
{
    for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x)
        a[q] = v;
}

template <typename T>
cudaError_t launch_shift_frame_impl(const DomainDesc& d, int kd, const void* phi_o, const void* c_o, void* phi_n,
                                    void* c_n, cudaStream_t st)
{
    const int gz = d.nz < 64 ? d.nz : 64;
    dim3 grid((d.nx + 127) / 128, d.ny, gz);
    k_shift_frame<T><<<grid, 128, 0, st>>>(d, kd, (const T*)phi_o, (const T*)c_o, (T*)phi_n, (T*)c_n);
    return cudaGetLastError();
}

template <typename T>
cudaError_t launch_fill_impl(void* a, long long n, double v, cudaStream_t st)
{
    k_fill<T><<<1184, 256, 0, st>>>((T*)a, n, (T)v);
    return cudaGetLastError();
}

// instantiated in the precision units
template <typename T>
cudaError_t launch_shift_frame(const DomainDesc& d, int kd, const void* phi_o, const void* c_o, void* phi_n,
                               void* c_n, cudaStream_t st);
template <typename T>
cudaError_t launch_fill(void* a, long long n, double v, cudaStream_t st);

}  // namespace pf3d
