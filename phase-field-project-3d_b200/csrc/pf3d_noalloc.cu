// pf3d_noalloc.cu -- diagnostics that allocate no device memory.
//
// pf_diagnosticos needs a scratch buffer for its per-block partial sums, and
// a pf_ctx allocates that buffer with cudaMalloc.  Some callers cannot let a
// library allocate device memory: a program whose device memory is owned by
// another runtime (for example the reference's OpenMP target-offload build,
// which maps its fields with `target enter data` and can hand their device
// addresses to C through `use_device_addr`, but keeps every allocation inside
// the OpenMP runtime), or a solver that runs under a fixed device-memory
// budget and forbids allocations inside its time loop.  For them,
// pf_diagnosticos_noalloc takes the caller's device pointers and uses a
// file-scope static device array as its scratch instead.
//
// The scratch holds up to PF_NOALLOC_MAX_PLANES rows of partials (4096; the
// array is 4097 x 8 doubles, about 256 KiB, held by every device that loads
// the library until the process exits).  Each z plane is split into S equal
// runs of cells, S = min(4096 / nz, planes cells / 1024) but at least 1, and
// one CTA reduces each run into its row, so a shallow domain still spreads
// over the whole GPU (16 planes of 4096 x 4096 cells give 4096 CTAs of 64 Ki
// cells each); the domain may therefore have at most 4096 planes.  The split
// depends only on nx, ny and nz, so the summation order -- and the result --
// is the same on every call.  Every call shares the array and leaves its
// contents behind; each call writes every partial it later reads (rows
// 0 .. nz*S-1 and the result row) before reading it, so nothing needs
// clearing, but two calls whose work overlaps on the GPU race on the array.
#include <cuda_runtime.h>
#include <cfloat>
#include <cmath>
#include <cstring>
#include <mutex>
#include <string>
#include "../../include/pf3d.h"

namespace pf3d {
int set_last_error_global(int code, const std::string& msg);   // pf3d_api.cu
}

namespace {

constexpr int kMaxPlanes = PF_NOALLOC_MAX_PLANES;
constexpr int kRow = 8;           // l2, l2 comp, max, min, sol, sol comp, fe, fe comp
constexpr int kMaxDevices = 64;

// rows 0 .. kMaxPlanes-1: partials of each run of cells; row kMaxPlanes: the result
static __device__ __align__(256) double g_diag_scratch[(kMaxPlanes + 1) * kRow];

std::mutex g_setup_mu;
double* g_scratch_addr[kMaxDevices];   // device address of g_diag_scratch per device

struct NSum {
    double s, c;
    __device__ __forceinline__ void add(double v)
    {
        double t = __dadd_rn(s, v);
        if (fabs(s) >= fabs(v)) c = __dadd_rn(c, __dadd_rn(__dsub_rn(s, t), v));
        else c = __dadd_rn(c, __dadd_rn(__dsub_rn(v, t), s));
        s = t;
    }
    __device__ __forceinline__ void merge(double os, double oc)
    {
        add(os);
        c = __dadd_rn(c, oc);
    }
};

// max / min that return NaN when either argument is NaN, as pf_diagnosticos
// reports them (fmax/fmin would drop a NaN and show finite extremes)
__device__ __forceinline__ double nan_max(double a, double b) { return (a > b || a != a) ? a : b; }
__device__ __forceinline__ double nan_min(double a, double b) { return (a < b || a != a) ? a : b; }

struct PlaneArgs {
    int nx, ny, nz;
    int runs;              // S: runs of cells per plane, one CTA and one row each
    long long run;         // cells per run (the last run of a plane may be shorter)
    long long px, plane;
    double dx, dy, dz, E0, W0;
};

// one CTA per run of cells of one z plane (row blockIdx.x = z * S + s),
// fixed reduction order (diag_body.inc:8-22 per cell)
template <typename T>
__global__ void __launch_bounds__(256) k_diag_plane(PlaneArgs a, const T* __restrict__ phi, const T* __restrict__ c,
                                                   double* __restrict__ part)
{
    const int row = blockIdx.x;
    const int z = row / a.runs, s = row % a.runs;
    NSum l2{0, 0}, sol{0, 0}, fe{0, 0};
    double mx = -DBL_MAX, mn = DBL_MAX;
    const long long ncell = (long long)a.nx * a.ny;
    const long long q0 = (long long)s * a.run;
    const long long q1 = q0 + a.run < ncell ? q0 + a.run : ncell;
    for (long long q = q0 + threadIdx.x; q < q1; q += blockDim.x) {
        const int x = (int)(q % a.nx), y = (int)(q / a.nx);
        const long long id = (long long)x + (long long)y * a.px + (long long)z * a.plane;
        const double p = (double)phi[id];
        l2.add(__dmul_rn(p, p));
        mx = nan_max(mx, p);
        mn = nan_min(mn, p);
        sol.add((double)c[id]);
        const double w = __dmul_rn(__dmul_rn(__dmul_rn(__dmul_rn(a.W0, p), p), __dsub_rn(1.0, p)), __dsub_rn(1.0, p));
        double g2 = 0.0;
        if (x > 0 && x < a.nx - 1 && y > 0 && y < a.ny - 1 && z > 0 && z < a.nz - 1) {
            const double gx = __dmul_rn(__dsub_rn((double)phi[id + 1], (double)phi[id - 1]), 0.5) / a.dx;
            const double gy = __dmul_rn(__dsub_rn((double)phi[id + a.px], (double)phi[id - a.px]), 0.5) / a.dy;
            const double gz = __dmul_rn(__dsub_rn((double)phi[id + a.plane], (double)phi[id - a.plane]), 0.5) / a.dz;
            g2 = __dadd_rn(__dadd_rn(__dmul_rn(gx, gx), __dmul_rn(gy, gy)), __dmul_rn(gz, gz));
        }
        const double e = __dadd_rn(__dmul_rn(__dmul_rn(__dmul_rn(0.5, a.E0), a.E0), g2), w);
        fe.add(__dmul_rn(__dmul_rn(__dmul_rn(e, a.dx), a.dy), a.dz));
    }
    __shared__ double sh[8][kRow];
    double v[kRow] = {l2.s, l2.c, mx, mn, sol.s, sol.c, fe.s, fe.c};
    for (int off = 16; off > 0; off >>= 1) {
        double o[kRow];
        for (int k = 0; k < kRow; ++k) o[k] = __shfl_down_sync(0xffffffffu, v[k], off);
        NSum s1{v[0], v[1]}; s1.merge(o[0], o[1]); v[0] = s1.s; v[1] = s1.c;
        v[2] = nan_max(v[2], o[2]); v[3] = nan_min(v[3], o[3]);
        NSum s2{v[4], v[5]}; s2.merge(o[4], o[5]); v[4] = s2.s; v[5] = s2.c;
        NSum s3{v[6], v[7]}; s3.merge(o[6], o[7]); v[6] = s3.s; v[7] = s3.c;
    }
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0)
        for (int k = 0; k < kRow; ++k) sh[w][k] = v[k];
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int k = 0; k < kRow; ++k) v[k] = sh[0][k];
        for (int ww = 1; ww < (int)(blockDim.x >> 5); ++ww) {
            NSum s1{v[0], v[1]}; s1.merge(sh[ww][0], sh[ww][1]); v[0] = s1.s; v[1] = s1.c;
            v[2] = nan_max(v[2], sh[ww][2]); v[3] = nan_min(v[3], sh[ww][3]);
            NSum s2{v[4], v[5]}; s2.merge(sh[ww][4], sh[ww][5]); v[4] = s2.s; v[5] = s2.c;
            NSum s3{v[6], v[7]}; s3.merge(sh[ww][6], sh[ww][7]); v[6] = s3.s; v[7] = s3.c;
        }
        for (int k = 0; k < kRow; ++k) part[(long long)row * kRow + k] = v[k];
    }
}

__global__ void k_diag_plane_final(const double* __restrict__ part, int rows, double* __restrict__ res)
{
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    NSum l2{0, 0}, sol{0, 0}, fe{0, 0};
    double mx = -DBL_MAX, mn = DBL_MAX;
    for (int r = 0; r < rows; ++r) {
        const double* p = part + (long long)r * kRow;
        l2.merge(p[0], p[1]);
        mx = nan_max(mx, p[2]);
        mn = nan_min(mn, p[3]);
        sol.merge(p[4], p[5]);
        fe.merge(p[6], p[7]);
    }
    res[0] = sqrt(__dadd_rn(l2.s, l2.c));
    res[1] = mx;
    res[2] = mn;
    res[3] = __dadd_rn(sol.s, sol.c);
    res[4] = __dadd_rn(fe.s, fe.c);
}

// device address of the static scratch on the current device, looked up once
// per device with that device current
int scratch_address(double** out)
{
    int dev = -1;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess || dev < 0)
        return pf3d::set_last_error_global(PF_E_NODEV, std::string("pf_diagnosticos_noalloc: no current CUDA device: ") +
                                                           cudaGetErrorString(e));
    if (dev >= kMaxDevices)
        return pf3d::set_last_error_global(PF_E_ARG, "pf_diagnosticos_noalloc: device index above 63");
    std::lock_guard<std::mutex> lk(g_setup_mu);
    if (!g_scratch_addr[dev]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_diag_scratch);
        if (e != cudaSuccess || !p)
            return pf3d::set_last_error_global(PF_E_CUDA, std::string("pf_diagnosticos_noalloc: cudaGetSymbolAddress: ") +
                                                              cudaGetErrorString(e));
        g_scratch_addr[dev] = static_cast<double*>(p);
    }
    *out = g_scratch_addr[dev];
    return PF_OK;
}

}  // namespace

extern "C" int pf_diagnosticos_noalloc(const void* phase_field, const void* conc_soluto, int nx, int ny, int nz,
                                       int pitch, int precision, double dx, double dy, double dz, double E0,
                                       double W0, void* stream, double out[5])
{
    if (!phase_field || !conc_soluto || !out)
        return pf3d::set_last_error_global(PF_E_ARG, "pf_diagnosticos_noalloc: null pointer argument");
    if (nx < 1 || ny < 1 || nz < 1 || pitch < nx)
        return pf3d::set_last_error_global(PF_E_ARG, "pf_diagnosticos_noalloc: need nx, ny, nz >= 1 and pitch >= nx");
    if (nz > kMaxPlanes)
        return pf3d::set_last_error_global(
            PF_E_ARG, "pf_diagnosticos_noalloc: nz = " + std::to_string(nz) + " exceeds the " +
                          std::to_string(kMaxPlanes) + " planes its static scratch holds; use pf_diagnosticos");
    if (precision != PF_FP64 && precision != PF_FP32)
        return pf3d::set_last_error_global(PF_E_ARG, "pf_diagnosticos_noalloc: precision must be 64 or 32");
    double* scratch = nullptr;
    int rc = scratch_address(&scratch);
    if (rc != PF_OK) return rc;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    PlaneArgs a;
    a.nx = nx; a.ny = ny; a.nz = nz;
    const long long ncell = (long long)nx * ny;
    long long runs = ncell / 1024;                       // at least 1024 cells a CTA
    if (runs > kMaxPlanes / nz) runs = kMaxPlanes / nz;  // at most kMaxPlanes rows
    if (runs < 1) runs = 1;
    a.runs = (int)runs;
    a.run = (ncell + runs - 1) / runs;
    const int rows = nz * a.runs;
    a.px = pitch;
    a.plane = (long long)pitch * ny;
    a.dx = dx; a.dy = dy; a.dz = dz; a.E0 = E0; a.W0 = W0;
    double* res = scratch + (long long)kMaxPlanes * kRow;
    if (precision == PF_FP64)
        k_diag_plane<double><<<rows, 256, 0, st>>>(a, (const double*)phase_field, (const double*)conc_soluto, scratch);
    else
        k_diag_plane<float><<<rows, 256, 0, st>>>(a, (const float*)phase_field, (const float*)conc_soluto, scratch);
    k_diag_plane_final<<<1, 32, 0, st>>>(scratch, rows, res);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(out, res, 5 * sizeof(double), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess)
        return pf3d::set_last_error_global(PF_E_CUDA, std::string("pf_diagnosticos_noalloc: ") + cudaGetErrorString(e));
    return PF_OK;
}
