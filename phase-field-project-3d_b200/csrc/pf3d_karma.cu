// pf3d_karma.cu -- C-ABI of the quantitative Karma model (include/pf3d.h,
// "Karma model"): one domain of phi and U resident in HBM, the two passes of
// pf3d_karma.cuh per step, the tip search and the seed on the device.
#include <cuda_runtime.h>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>
#include "../../include/pf3d.h"
#include "pf3d_karma.cuh"

using namespace pf3d;

namespace pf3d {
int set_last_error_global(int code, const std::string& msg);
}

namespace {
constexpr double kA1 = 0.8839, kA2 = 0.6267;            // karma3d.f90:98
constexpr double kAt = 0.35355339059327373;             // karma3d.f90:99
constexpr int kTY = 8, kZChunk = 64;

int kerr(int code, const std::string& msg) { return set_last_error_global(code, "pf_karma: " + msg); }

template <typename T>
KarmaK<T> karma_constants(const pf_karma_params& p)
{
    // each as the reference's expression evaluates it in FP64, then stored in T
    const double idx = 1.0 / p.dx;
    KarmaK<T> c;
    c.idx = (T)idx;
    c.q = (T)(0.25 * idx);
    c.h = (T)(0.5 * idx);
    c.om3 = (T)(1.0 - 3.0 * p.eps4);
    c.e4 = (T)(4.0 * p.eps4);
    c.e16 = (T)(16.0 * p.eps4);
    c.lambda = (T)p.lambda;
    c.dt = (T)p.dt;
    c.Fnoise = (T)p.Fnoise;
    c.sqdt = (T)std::sqrt(p.dt);
    c.omk = (T)(1.0 - p.k);
    c.Ahalf1 = (T)(0.5 * (1.0 + p.k));
    c.Ahalf2 = (T)(0.5 * (1.0 - p.k));
    c.D = (T)(kA2 * p.lambda);
    c.at = (T)kAt;
    return c;
}

// karma3d.f90:130-144 on the device: an eighth of a sphere of radius R0 at
// the corner, phi = -tanh((r - R0)/sqrt(2)) at the centres (i - 1/2) dx,
// U = -Omega
template <typename T>
__global__ void k_karma_seed(KarmaDesc d, double dx, double R0, double Omega, T* __restrict__ phi, T* __restrict__ U)
{
    const long long n = (long long)d.nx * d.ny * d.nz;
    for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
        const int x = (int)(q % d.nx);
        const long long r2 = q / d.nx;
        const int y = (int)(r2 % d.ny), z = (int)(r2 / d.ny);
        const double xx = __dmul_rn((double)(x + 1) - 0.5, dx);
        const double yy = __dmul_rn((double)(y + 1) - 0.5, dx);
        const double zz = __dmul_rn((double)(z + 1) - 0.5, dx);
        const double r = sqrt(__dadd_rn(__dadd_rn(__dmul_rn(xx, xx), __dmul_rn(yy, yy)), __dmul_rn(zz, zz)));
        const long long id = (long long)x + (long long)y * d.px + (long long)z * d.plane;
        phi[id] = (T)(-tanh(__ddiv_rn(__dsub_rn(r, R0), sqrt(2.0))));
        U[id] = (T)(-Omega);
    }
}
}  // namespace

struct pf_karma {
    pf_karma_params p;
    pf_karma_derived dv;
    int prec;
    size_t es;
    KarmaDesc d;
    size_t field_bytes;
    void* base;
    void* phi[2];
    void* U[2];
    void* dphi;
    int* d_tip;
    int* h_tip;   // pinned
    int cur;      // which phi/U buffer holds the state
    int it;       // steps done
    cudaStream_t own_stream, stream;
};

extern "C" {

int pf_karma_derived_of(const pf_karma_params* p, pf_karma_derived* out)
{
    if (!p || !out) return kerr(PF_E_ARG, "bad argument");
    // karma3d.f90:118-124, in the reference's order
    out->D = kA2 * p->lambda;
    out->cl0 = (p->Tm - p->TP) / p->mliq;
    out->Omega = (out->cl0 - p->C0) / ((1.0 - p->k) * out->cl0);
    out->Gam = p->sigma * p->Tm / p->dH;
    out->d0 = out->Gam / (p->mliq * (1.0 - p->k) * out->cl0);
    out->W = p->lambda / kA1 * out->d0;
    out->tau0 = kA2 * p->lambda * out->W * out->W / p->Dl;
    return PF_OK;
}

int pf_karma_create(const pf_karma_params* p, int precision, pf_karma** out)
{
    if (!out) return kerr(PF_E_ARG, "out is null");
    *out = nullptr;
    if (!p || p->nx < 1 || p->ny < 1 || p->nz < 1) return kerr(PF_E_ARG, "grid extents must be >= 1");
    if (precision != PF_FP64 && precision != PF_FP32) return kerr(PF_E_ARG, "precision must be 64 or 32");
    if (!(p->dx > 0.0) || !(p->dt > 0.0)) return kerr(PF_E_ARG, "dx and dt must be > 0");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev < 1) {
        cudaGetLastError();
        return kerr(PF_E_NODEV, "no CUDA device");
    }
    pf_karma* k = new pf_karma();
    k->p = *p;
    pf_karma_derived_of(p, &k->dv);
    k->prec = precision;
    k->es = precision == PF_FP64 ? 8 : 4;
    const long long px = ((long long)p->nx + 31) / 32 * 32;
    k->d.nx = p->nx;
    k->d.ny = p->ny;
    k->d.nz = p->nz;
    k->d.px = px;
    k->d.plane = px * p->ny;
    k->d.it = 0;
    k->field_bytes = ((size_t)px * p->ny * p->nz * k->es + 255) / 256 * 256;
    cudaError_t e = cudaMalloc(&k->base, 5 * k->field_bytes + 256);
    if (e != cudaSuccess) {
        cudaGetLastError();
        delete k;
        return kerr(PF_E_NOMEM, std::string("cudaMalloc: ") + cudaGetErrorString(e));
    }
    char* b = (char*)k->base;
    k->phi[0] = b;
    k->phi[1] = b + k->field_bytes;
    k->U[0] = b + 2 * k->field_bytes;
    k->U[1] = b + 3 * k->field_bytes;
    k->dphi = b + 4 * k->field_bytes;
    k->d_tip = (int*)(b + 5 * k->field_bytes);
    if ((e = cudaMemset(k->base, 0, 5 * k->field_bytes + 256)) != cudaSuccess ||
        (e = cudaMallocHost(&k->h_tip, 2 * sizeof(int))) != cudaSuccess ||
        (e = cudaStreamCreateWithFlags(&k->own_stream, cudaStreamNonBlocking)) != cudaSuccess) {
        cudaFree(k->base);
        delete k;
        return kerr(PF_E_CUDA, std::string("set-up: ") + cudaGetErrorString(e));
    }
    k->stream = k->own_stream;
    *out = k;
    return PF_OK;
}

int pf_karma_destroy(pf_karma* k)
{
    if (!k) return PF_OK;
    cudaStreamSynchronize(k->stream);
    cudaFree(k->base);
    cudaFreeHost(k->h_tip);
    cudaStreamDestroy(k->own_stream);
    delete k;
    return PF_OK;
}

int pf_karma_set_stream(pf_karma* k, void* stream)
{
    if (!k) return kerr(PF_E_ARG, "null handle");
    k->stream = stream ? (cudaStream_t)stream : k->own_stream;
    return PF_OK;
}

int pf_karma_get_it(const pf_karma* k, int* it)
{
    if (!k || !it) return kerr(PF_E_ARG, "bad argument");
    *it = k->it;
    return PF_OK;
}

int pf_karma_set_it(pf_karma* k, int it)
{
    if (!k || it < 0) return kerr(PF_E_ARG, "bad argument");
    k->it = it;
    return PF_OK;
}

static void* karma_field(pf_karma* k, int field)
{
    switch (field) {
    case PF_KARMA_PHI: return k->phi[k->cur];
    case PF_KARMA_U: return k->U[k->cur];
    case PF_KARMA_DPHI: return k->dphi;
    }
    return nullptr;
}

int pf_karma_upload(pf_karma* k, int field, const double* host)
{
    if (!k || !host || (field != PF_KARMA_PHI && field != PF_KARMA_U)) return kerr(PF_E_ARG, "bad argument");
    const pf_karma_params& p = k->p;
    const size_t n = (size_t)p.nx * p.ny * p.nz;
    const void* src = host;
    std::vector<float> tmp;
    if (k->prec == PF_FP32) {
        tmp.resize(n);
        for (size_t q = 0; q < n; ++q) tmp[q] = (float)host[q];
        src = tmp.data();
    }
    cudaError_t e = cudaMemcpy2DAsync(karma_field(k, field), (size_t)k->d.px * k->es, src, (size_t)p.nx * k->es,
                                      (size_t)p.nx * k->es, (size_t)p.ny * p.nz, cudaMemcpyHostToDevice, k->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(k->stream);
    if (e != cudaSuccess) return kerr(PF_E_CUDA, std::string("upload: ") + cudaGetErrorString(e));
    return PF_OK;
}

int pf_karma_download(pf_karma* k, int field, double* host)
{
    if (!k || !host || field < PF_KARMA_PHI || field > PF_KARMA_DPHI) return kerr(PF_E_ARG, "bad argument");
    const pf_karma_params& p = k->p;
    const size_t n = (size_t)p.nx * p.ny * p.nz;
    std::vector<float> tmp;
    void* dst = host;
    if (k->prec == PF_FP32) {
        tmp.resize(n);
        dst = tmp.data();
    }
    cudaError_t e = cudaMemcpy2DAsync(dst, (size_t)p.nx * k->es, karma_field(k, field), (size_t)k->d.px * k->es,
                                      (size_t)p.nx * k->es, (size_t)p.ny * p.nz, cudaMemcpyDeviceToHost, k->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(k->stream);
    if (e != cudaSuccess) return kerr(PF_E_CUDA, std::string("download: ") + cudaGetErrorString(e));
    if (k->prec == PF_FP32)
        for (size_t q = 0; q < n; ++q) host[q] = (double)tmp[q];
    return PF_OK;
}

int pf_karma_seed(pf_karma* k)
{
    if (!k) return kerr(PF_E_ARG, "null handle");
    cudaError_t e;
    if (k->prec == PF_FP64)
        k_karma_seed<double><<<1184, 256, 0, k->stream>>>(k->d, k->p.dx, k->p.R0, k->dv.Omega,
                                                          (double*)k->phi[k->cur], (double*)k->U[k->cur]);
    else
        k_karma_seed<float><<<1184, 256, 0, k->stream>>>(k->d, k->p.dx, k->p.R0, k->dv.Omega,
                                                         (float*)k->phi[k->cur], (float*)k->U[k->cur]);
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemsetAsync(k->dphi, 0, k->field_bytes, k->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(k->stream);
    if (e != cudaSuccess) return kerr(PF_E_CUDA, std::string("seed: ") + cudaGetErrorString(e));
    k->it = 0;
    return PF_OK;
}

}  // extern "C"

template <typename T>
static cudaError_t karma_steps(pf_karma* k, int n)
{
    const KarmaK<T> c = karma_constants<T>(k->p);
    const dim3 block(32, kTY);
    const dim3 grid((k->d.nx + 31) / 32, (k->d.ny + kTY - 1) / kTY, (k->d.nz + kZChunk - 1) / kZChunk);
    for (int s = 0; s < n; ++s) {
        KarmaDesc d = k->d;
        d.it = k->it + 1;
        const int a = k->cur, b = 1 - k->cur;
        k_karma_phase<T, kTY><<<grid, block, 0, k->stream>>>(d, c, (const T*)k->phi[a], (const T*)k->U[a],
                                                             (T*)k->dphi, kZChunk);
        k_karma_solute<T, kTY><<<grid, block, 0, k->stream>>>(d, c, (const T*)k->phi[a], (const T*)k->U[a],
                                                              (const T*)k->dphi, (T*)k->phi[b], (T*)k->U[b],
                                                              kZChunk);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
        k->cur = b;
        k->it += 1;
    }
    return cudaSuccess;
}

extern "C" {

int pf_karma_step(pf_karma* k, int n_steps)
{
    if (!k || n_steps < 0) return kerr(PF_E_ARG, "bad argument");
    cudaError_t e = k->prec == PF_FP64 ? karma_steps<double>(k, n_steps) : karma_steps<float>(k, n_steps);
    if (e != cudaSuccess) return kerr(PF_E_CUDA, std::string("step: ") + cudaGetErrorString(e));
    return PF_OK;
}

int pf_karma_tip(pf_karma* k, int* tip_x, int* tip_d)
{
    if (!k || !tip_x || !tip_d) return kerr(PF_E_ARG, "bad argument");
    if (k->prec == PF_FP64)
        k_karma_tip<double><<<1, 256, 0, k->stream>>>(k->d, (const double*)k->phi[k->cur], k->d_tip);
    else
        k_karma_tip<float><<<1, 256, 0, k->stream>>>(k->d, (const float*)k->phi[k->cur], k->d_tip);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(k->h_tip, k->d_tip, 2 * sizeof(int), cudaMemcpyDeviceToHost, k->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(k->stream);
    if (e != cudaSuccess) return kerr(PF_E_CUDA, std::string("tip: ") + cudaGetErrorString(e));
    *tip_x = k->h_tip[0];
    *tip_d = k->h_tip[1];
    return PF_OK;
}

int pf_karma_sync(pf_karma* k)
{
    if (!k) return kerr(PF_E_ARG, "null handle");
    cudaError_t e = cudaStreamSynchronize(k->stream);
    if (e != cudaSuccess) return kerr(PF_E_CUDA, std::string("sync: ") + cudaGetErrorString(e));
    return PF_OK;
}

}  // extern "C"
