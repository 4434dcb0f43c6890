// pf3d_track.cuh -- on-device solidification tracking.
//
// Solid fraction = mean(phi >= 0.5) and tip position = the highest plane k
// (1-based) where some (i, j) column has phi >= 0.5, interpolated linearly to
// the 0.5 crossing with the plane above from the two planes' maxima: the "tip
// height, phi >= 0.5" of the reference's run log (docs/run6/README.md:54-62)
// as the tracking loop of karma/karma3d.f90:291-298 evaluates it once per
// output, here without copying the field to the host.
//
// One pass over phi: each CTA reduces a band of rows of one plane to the
// plane's maximum (an order-preserving 64-bit key, so atomicMax is exact and
// order independent) and its count of solid cells (integer, exact); a one-thread
// kernel then scans the plane maxima from the top.  The result equals the same
// metric evaluated on the downloaded field bit for bit.
#pragma once
#include "pf3d_launch.h"

namespace pf3d {

// order-preserving key of a double: key(a) < key(b) iff a < b (finite values)
__device__ __forceinline__ unsigned long long track_key(double v)
{
    const long long b = __double_as_longlong(v);
    return b < 0 ? ~(unsigned long long)b : ((unsigned long long)b | 0x8000000000000000ull);
}
__device__ __forceinline__ double track_unkey(unsigned long long k)
{
    const unsigned long long b = (k & 0x8000000000000000ull) ? (k & 0x7fffffffffffffffull) : ~k;
    return __longlong_as_double((long long)b);
}

// block (32, 8): threads stride x by 32 and rows by 8 * gridDim.x; blockIdx.y = plane
template <typename T>
__global__ void __launch_bounds__(256) k_track(DomainDesc d, const T* __restrict__ phi,
                                               unsigned long long* __restrict__ pmax,
                                               unsigned long long* __restrict__ count)
{
    const int z = blockIdx.y;
    const T* pl = phi + (long long)z * d.plane;
    unsigned long long best = 0;
    unsigned int n = 0;
    for (int y = blockIdx.x * 8 + threadIdx.y; y < d.ny; y += gridDim.x * 8) {
        const T* row = pl + (long long)y * d.px;
        for (int x = threadIdx.x; x < d.nx; x += 32) {
            const double v = (double)row[x];
            const unsigned long long k = track_key(v);
            best = k > best ? k : best;
            n += (v >= 0.5) ? 1u : 0u;
        }
    }
    for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long b2 = __shfl_xor_sync(0xffffffffu, best, o);
        best = b2 > best ? b2 : best;
        n += __shfl_xor_sync(0xffffffffu, n, o);
    }
    __shared__ unsigned long long sb[8];
    __shared__ unsigned int sn[8];
    if (threadIdx.x == 0) {
        sb[threadIdx.y] = best;
        sn[threadIdx.y] = n;
    }
    __syncthreads();
    if (threadIdx.x == 0 && threadIdx.y == 0) {
        unsigned long long b = sb[0];
        unsigned long long tot = sn[0];
        for (int w = 1; w < 8; ++w) {
            b = sb[w] > b ? sb[w] : b;
            tot += sn[w];
        }
        atomicMax(&pmax[z], b);
        if (tot) atomicAdd(count, tot);
    }
}

// out = {solid fraction, tip position (cells, 1-based k; 0 when no plane is
// solid), solid cell count}.  A template (on the field type) so that each
// precision unit has its own instance.
template <typename T>
__global__ void k_track_final(int nz, long long cells, const unsigned long long* __restrict__ pmax,
                              const unsigned long long* __restrict__ count, double* __restrict__ out)
{
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    int k = -1;
    for (int z = nz - 1; z >= 0; --z)
        if (track_unkey(pmax[z]) >= 0.5) { k = z; break; }
    double tip = 0.0;
    if (k >= 0) {
        if (k + 1 >= nz) {
            tip = (double)(k + 1);
        } else {
            const double lo = track_unkey(pmax[k]), hi = track_unkey(pmax[k + 1]);
            const double frac = lo > hi ? (lo - 0.5) / (lo - hi) : 0.0;
            tip = (double)(k + 1) + frac;
        }
    }
    const unsigned long long n = *count;
    out[0] = (double)n / (double)cells;
    out[1] = tip;
    out[2] = (double)n;
}

// scratch: pmax[nz], count[1]; out[3] device doubles
template <typename T>
cudaError_t launch_track_impl(const DomainDesc& d, const void* phi, unsigned long long* scratch, double* out,
                              cudaStream_t st)
{
    cudaError_t e = cudaMemsetAsync(scratch, 0, ((size_t)d.nz + 1) * sizeof(unsigned long long), st);
    if (e != cudaSuccess) return e;
    const int rows = (d.ny + 7) / 8;
    int gx = (592 + d.nz - 1) / d.nz;          // about 4 CTAs per SM in total
    gx = gx < 1 ? 1 : (gx > rows ? rows : gx);
    k_track<T><<<dim3(gx, d.nz), dim3(32, 8), 0, st>>>(d, (const T*)phi, scratch, scratch + d.nz);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    k_track_final<T><<<1, 32, 0, st>>>(d.nz, (long long)d.nx * d.ny * d.nz, scratch, scratch + d.nz, out);
    return cudaGetLastError();
}

// instantiated in the precision units
template <typename T>
cudaError_t launch_track(const DomainDesc& d, const void* phi, unsigned long long* scratch, double* out,
                         cudaStream_t st);

}  // namespace pf3d
