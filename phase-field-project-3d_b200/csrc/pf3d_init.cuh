// pf3d_init.cuh -- device-side seeded initial state.
//
// The reference fills its fields on the host (entrada.f90:226-262).  For
// batched and served runs the state is created on the device instead, with
// the recipe of the synthetic workloads (pf3d/init.py): a solid slab of
// cells k <= 4 carrying hemispherical bumps, phi = (1 - tanh(2 d / w)) / 2
// with d the signed distance (cells) to slab U bumps and w the interface
// width in cells; c = C0 (1 - (1 - Ke) phi); T = T0; DPP = 0.
#pragma once
#include "pf3d_launch.h"

namespace pf3d {

struct InitArgs {
    int n_bumps;
    int kmax;          // planes above kmax have phi = 0 exactly (tanh saturates)
    double slab_top;   // 4.5
    double bump_r;     // 3
    double width;      // interface width in cells
    double C0, Ke, T0;
};

template <typename T>
__global__ void k_init_seeded(DomainDesc d, InitArgs a, const double* __restrict__ sites, T* __restrict__ phi,
                              T* __restrict__ c, T* __restrict__ Tf, T* __restrict__ dpp)
{
    const long long n = (long long)d.nx * d.ny * d.nz;
    for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
        const int x = (int)(q % d.nx);
        const long long r = q / d.nx;
        const int y = (int)(r % d.ny);
        const int z = (int)(r / d.ny);
        const double i = x + 1, j = y + 1, k = z + 1;
        double p = 0.0;
        if (z < a.kmax) {
            const double dz = k - a.slab_top;
            double dist = dz;
            for (int b = 0; b < a.n_bumps; ++b) {
                const double di = i - sites[2 * b], dj = j - sites[2 * b + 1];
                // (di^2 + dj^2) + dz^2 without contraction, like the host recipe
                const double s2 = __dadd_rn(__dadd_rn(__dmul_rn(di, di), __dmul_rn(dj, dj)), __dmul_rn(dz, dz));
                const double db = sqrt(s2) - a.bump_r;
                dist = fmin(dist, db);
            }
            p = __dmul_rn(0.5, 1.0 - tanh(__dmul_rn(2.0, dist) / a.width));
        }
        const long long id = (long long)x + (long long)y * d.px + (long long)z * d.plane;
        phi[id] = (T)p;
        c[id] = (T)__dmul_rn(a.C0, 1.0 - __dmul_rn(1.0 - a.Ke, p));
        Tf[id] = (T)a.T0;
        dpp[id] = (T)0;
    }
}

template <typename T>
cudaError_t launch_init_seeded_impl(const DomainDesc& d, const InitArgs& a, const double* sites, void* phi, void* c,
                               void* Tf, void* dpp, cudaStream_t st)
{
    k_init_seeded<T><<<1184, 256, 0, st>>>(d, a, sites, (T*)phi, (T*)c, (T*)Tf, (T*)dpp);
    return cudaGetLastError();
}

// instantiated in the precision units
template <typename T>
cudaError_t launch_init_seeded(const DomainDesc& d, const InitArgs& a, const double* sites, void* phi, void* c,
                               void* Tf, void* dpp, cudaStream_t st);

}  // namespace pf3d
