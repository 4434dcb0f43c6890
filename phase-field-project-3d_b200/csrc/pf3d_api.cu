// pf3d_api.cu -- C-ABI of the B200 phase-field step (include/pf3d.h).
//
// A pf_ctx is one domain resident in HBM: the seven fields of the
// reference (principal.f90:61-63) in pitched FP64 or FP32 storage, one
// stream, and the host scalars the reference keeps in module variables
// (TP, M0, it, time).  The per-subroutine entry points launch the
// one-thread-per-cell kernels; pf_step launches the fused z-marching passes.
#include <cuda_runtime.h>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <thread>
#include <vector>
#include "../../include/pf3d.h"
#include "pf3d_launch.h"
#include "pf3d_scalar.h"
#include "pf3d_hostdesc.h"
#include "pf3d_init.cuh"
#include "pf3d_ckpt.h"
#include "pf3d_tma.cuh"
#include "pf3d_tmap.h"

using namespace pf3d;

namespace {
std::mutex g_err_mu;
std::string g_err;   // last error of calls without a context

int set_global_err(int code, const std::string& msg)
{
    std::lock_guard<std::mutex> lk(g_err_mu);
    g_err = msg;
    return code;
}
}  // namespace

namespace pf3d {
// lets other translation units report through pf_last_error(NULL)
int set_last_error_global(int code, const std::string& msg) { return set_global_err(code, msg); }
}  // namespace pf3d

struct pf_ctx {
    pf_grid g;
    pf_params p;
    int prec;          // 64 or 32
    size_t es;         // element size
    pf_derived dv;
    pf_state st;
    DomainDesc dd;
    void* fld[7];      // device pointer of each field id
    void* base;
    size_t field_bytes;
    double* d_part;
    int nblk;
    double* d_out;
    double* h_out;     // pinned
    double* d_stage;
    size_t stage_elems;
    unsigned long long* d_track;   // tracking scratch: nz plane maxima + count
    double* d_track_out;           // 3 tracking results
    // asynchronous checkpoint writer: fields copied into ckpt_host on the
    // stream, then written to the file by ckpt_thr once ckpt_ev has passed
    std::thread ckpt_thr;
    void* ckpt_host;
    size_t ckpt_host_bytes;
    cudaEvent_t ckpt_ev;
    int ckpt_rc;
    std::string ckpt_err;
    cudaStream_t own_stream;
    cudaStream_t stream;
    int fused, tile_y, zchunk, ktiming, paired;
    int kernel;              // PF_OPT_KERNEL: 1 TMA-staged march passes, 0 the cp.async passes
    int nslot;               // PF_OPT_NSLOT: window mode of the march passes (0: 3)
    CUtensorMap tmap[2];     // tensor maps of the two phase-field buffers (32 x 8 march tiles)
    void* tmap_buf[2];       // their base addresses
    int tmap_ok;
    int* d_status;           // kernel status word: 0, or the code a kernel left there
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> ev_first, ev_last;
    std::string err;
    int device;
};

static int ctx_err(pf_ctx* c, int code, const std::string& msg)
{
    if (c) c->err = msg;
    set_global_err(code, msg);
    return code;
}

static int cuda_check(pf_ctx* c, cudaError_t e, const char* what)
{
    if (e == cudaSuccess) return PF_OK;
    return ctx_err(c, PF_E_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

#define CK(call, what)                                  \
    do {                                                \
        int rc_ = cuda_check(ctx, (call), what);        \
        if (rc_ != PF_OK) return rc_;                   \
    } while (0)

static inline bool is64(const pf_ctx* c) { return c->prec == PF_FP64; }

extern "C" {

int pf_version(void) { return PF3D_VERSION; }

const char* pf_last_error(const pf_ctx* ctx)
{
    if (ctx) return ctx->err.c_str();
    std::lock_guard<std::mutex> lk(g_err_mu);
    return g_err.c_str();
}

long long pf_ctx_bytes(const pf_grid* g, int precision)
{
    if (!g || g->nx < 1 || g->ny < 1 || g->nz < 1) return -1;
    size_t es = (precision == PF_FP32) ? 4 : 8;
    size_t fb = round_up((size_t)pitch_of(g->nx) * g->ny * g->nz * es + 64, 256);
    return (long long)(7 * fb);
}

int pf_create(const pf_grid* g, const pf_params* p, int precision, pf_ctx** out)
{
    if (!out) return set_global_err(PF_E_ARG, "out is null");
    *out = nullptr;
    std::string why;
    int rc = validate(g, p, precision, why);
    if (rc != PF_OK) return set_global_err(rc, why);
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return set_global_err(PF_E_NODEV, "no CUDA device visible");
    }
    pf_ctx* ctx = new pf_ctx();
    ctx->g = *g;
    ctx->p = *p;
    ctx->prec = precision;
    ctx->es = (precision == PF_FP32) ? 4 : 8;
    setup_derived(*g, *p, ctx->dv);
    ctx->st.it = 0;
    ctx->st.TP = initial_tp(*p);
    ctx->st.M0 = p->M0;
    ctx->st.time = 0.0f;
    equilibrium(*p, ctx->st.TP, &ctx->st.Cs_eq, &ctx->st.Cl_eq);
    const int px = pitch_of(g->nx);
    fill_desc(*g, *p, ctx->dv, px, ctx->dd);
    ctx->fused = 1;
    ctx->tile_y = 8;
    ctx->zchunk = 64;
    ctx->ktiming = 0;
    ctx->paired = 1;
    cudaGetDevice(&ctx->device);
    // one allocation: 7 fields + diagnostics partials
    ctx->field_bytes = round_up((size_t)px * g->ny * g->nz * ctx->es + 64, 256);
    ctx->nblk = 592;
    const size_t track_words = round_up((size_t)g->nz + 1, 4) + 4;
    size_t total = 7 * ctx->field_bytes + (size_t)ctx->nblk * kDiagRow * sizeof(double) + 8 * sizeof(double) +
                   track_words * sizeof(unsigned long long) + 16;
    cudaError_t e = cudaMalloc(&ctx->base, total);
    if (e != cudaSuccess) {
        cudaGetLastError();
        delete ctx;
        return set_global_err(PF_E_NOMEM, std::string("cudaMalloc of ") + std::to_string(total) + " bytes: " + cudaGetErrorString(e));
    }
    for (int f = 0; f < 7; ++f) ctx->fld[f] = (char*)ctx->base + (size_t)f * ctx->field_bytes;
    ctx->d_part = (double*)((char*)ctx->base + 7 * ctx->field_bytes);
    ctx->d_out = ctx->d_part + (size_t)ctx->nblk * kDiagRow;
    ctx->d_track = (unsigned long long*)(ctx->d_out + 8);
    ctx->d_track_out = (double*)(ctx->d_track + round_up((size_t)g->nz + 1, 4));
    ctx->d_status = (int*)(ctx->d_track_out + 4);
    if ((e = cudaMemset(ctx->base, 0, total)) != cudaSuccess ||
        (e = cudaMallocHost(&ctx->h_out, 8 * sizeof(double))) != cudaSuccess ||
        (e = cudaStreamCreateWithFlags(&ctx->own_stream, cudaStreamNonBlocking)) != cudaSuccess) {
        cudaFree(ctx->base);
        delete ctx;
        return set_global_err(PF_E_CUDA, std::string("context set-up: ") + cudaGetErrorString(e));
    }
    ctx->stream = ctx->own_stream;
    // tensor maps of the phase-field buffers for the TMA plane loads; without
    // them (driver entry point missing) the step uses the cp.async passes
    ctx->kernel = 1;
    ctx->nslot = 0;
    ctx->tmap_ok = 1;
    for (int b = 0; b < 2; ++b) {
        ctx->tmap_buf[b] = ctx->fld[b == 0 ? PF_PHASE_OLD : PF_PHASE_NEW];
        if (encode_field_map(&ctx->tmap[b], ctx->tmap_buf[b], (int)ctx->es, g->nx, g->ny, g->nz, px,
                             march_box_x((int)ctx->es), march_box_y(8)) != 0)
            ctx->tmap_ok = 0;
    }
    *out = ctx;
    return PF_OK;
}

static void drop_events(pf_ctx* ctx)
{
    for (auto& pr : ctx->ev_first) { cudaEventDestroy(pr.first); cudaEventDestroy(pr.second); }
    for (auto& pr : ctx->ev_last) { cudaEventDestroy(pr.first); cudaEventDestroy(pr.second); }
    ctx->ev_first.clear();
    ctx->ev_last.clear();
}

int pf_destroy(pf_ctx* ctx)
{
    if (!ctx) return PF_OK;
    if (ctx->ckpt_thr.joinable()) ctx->ckpt_thr.join();
    if (ctx->ckpt_host) cudaFreeHost(ctx->ckpt_host);
    if (ctx->ckpt_ev) cudaEventDestroy(ctx->ckpt_ev);
    cudaStreamSynchronize(ctx->stream);
    drop_events(ctx);
    if (ctx->d_stage) cudaFree(ctx->d_stage);
    cudaFree(ctx->base);
    cudaFreeHost(ctx->h_out);
    cudaStreamDestroy(ctx->own_stream);
    delete ctx;
    return PF_OK;
}

int pf_get_derived(const pf_ctx* ctx, pf_derived* out)
{
    if (!ctx || !out) return PF_E_ARG;
    *out = ctx->dv;
    return PF_OK;
}

int pf_get_state(const pf_ctx* ctx, pf_state* out)
{
    if (!ctx || !out) return PF_E_ARG;
    *out = ctx->st;
    return PF_OK;
}

int pf_set_state(pf_ctx* ctx, const pf_state* st)
{
    if (!ctx || !st) return PF_E_ARG;
    ctx->st = *st;
    return PF_OK;
}

// the kernel status word, after the stream has drained: PF_E_KERNEL when a
// kernel reported a failure (the word is cleared after it is reported)
static int kernel_status(pf_ctx* ctx)
{
    int code = 0;
    CK(cudaMemcpyAsync(&code, ctx->d_status, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream), "status read");
    CK(cudaStreamSynchronize(ctx->stream), "status read");
    if (code == 0) return PF_OK;
    CK(cudaMemsetAsync(ctx->d_status, 0, sizeof(int), ctx->stream), "status reset");
    return ctx_err(ctx, PF_E_KERNEL, "a kernel reported failure code " + std::to_string(code) +
                                         (code == kErrTmaTimeout ? " (a TMA plane load did not arrive in time)" : ""));
}

int pf_sync(pf_ctx* ctx)
{
    if (!ctx) return PF_E_ARG;
    CK(cudaStreamSynchronize(ctx->stream), "pf_sync");
    return kernel_status(ctx);
}

int pf_set_stream(pf_ctx* ctx, void* stream)
{
    if (!ctx) return PF_E_ARG;
    ctx->stream = stream ? (cudaStream_t)stream : ctx->own_stream;
    return PF_OK;
}

int pf_set_option(pf_ctx* ctx, int opt, int value)
{
    if (!ctx) return PF_E_ARG;
    switch (opt) {
    case PF_OPT_FUSED: ctx->fused = value ? 1 : 0; return PF_OK;
    case PF_OPT_TILE_Y:
        if (value != 4 && value != 8 && value != 16) return ctx_err(ctx, PF_E_ARG, "tile_y must be 4, 8 or 16");
        ctx->tile_y = value;
        return PF_OK;
    case PF_OPT_ZCHUNK:
        if (value < 0) return ctx_err(ctx, PF_E_ARG, "zchunk must be >= 0");
        ctx->zchunk = value;
        return PF_OK;
    case PF_OPT_KTIMING: ctx->ktiming = value ? 1 : 0; return PF_OK;
    case PF_OPT_PAIRED:
        if (value < 0 || value > 2) return ctx_err(ctx, PF_E_ARG, "paired must be 0, 1 or 2");
        ctx->paired = value;
        return PF_OK;
    case PF_OPT_KERNEL:
        if (value < 0 || value > 1) return ctx_err(ctx, PF_E_ARG, "kernel must be 0 or 1");
        ctx->kernel = value;
        return PF_OK;
    case PF_OPT_NSLOT:
        if (value != 0 && value != 3 && value != 4 && value != 5)
            return ctx_err(ctx, PF_E_ARG, "window mode must be 0, 3, 4 or 5");
        ctx->nslot = value;
        return PF_OK;
    }
    return ctx_err(ctx, PF_E_ARG, "unknown option");
}

int pf_get_option(const pf_ctx* ctx, int opt, int* value)
{
    if (!ctx || !value) return PF_E_ARG;
    switch (opt) {
    case PF_OPT_FUSED: *value = ctx->fused; return PF_OK;
    case PF_OPT_TILE_Y: *value = ctx->tile_y; return PF_OK;
    case PF_OPT_ZCHUNK: *value = ctx->zchunk; return PF_OK;
    case PF_OPT_KTIMING: *value = ctx->ktiming; return PF_OK;
    case PF_OPT_PAIRED: *value = ctx->paired; return PF_OK;
    case PF_OPT_KERNEL: *value = ctx->kernel; return PF_OK;
    case PF_OPT_NSLOT: *value = ctx->nslot; return PF_OK;
    }
    return PF_E_ARG;
}

// ---- data residency ----

static int ensure_stage(pf_ctx* ctx)
{
    if (ctx->d_stage) return PF_OK;
    size_t plane = (size_t)ctx->g.nx * ctx->g.ny;
    size_t want = (size_t)1 << 24;  // 16 Mi doubles = 128 MiB
    if (want < plane) want = plane;
    ctx->stage_elems = want;
    CK(cudaMalloc(&ctx->d_stage, want * sizeof(double)), "staging buffer");
    return PF_OK;
}

int pf_upload(pf_ctx* ctx, int field, const double* host)
{
    if (!ctx || !host || field < 0 || field > 6) return ctx_err(ctx, PF_E_ARG, "pf_upload: bad argument");
    const pf_grid& g = ctx->g;
    if (is64(ctx)) {
        CK(cudaMemcpy2DAsync(ctx->fld[field], (size_t)ctx->dd.px * 8, host, (size_t)g.nx * 8, (size_t)g.nx * 8,
                             (size_t)g.ny * g.nz, cudaMemcpyHostToDevice, ctx->stream),
           "pf_upload copy");
    } else {
        int rc = ensure_stage(ctx);
        if (rc) return rc;
        size_t plane = (size_t)g.nx * g.ny;
        long long zper = (long long)(ctx->stage_elems / plane);
        for (long long z0 = 0; z0 < g.nz; z0 += zper) {
            long long nzc = std::min<long long>(zper, g.nz - z0);
            CK(cudaMemcpyAsync(ctx->d_stage, host + z0 * plane, nzc * plane * sizeof(double), cudaMemcpyHostToDevice,
                               ctx->stream),
               "pf_upload copy");
            CK(launch_convert_in<float>(ctx->dd, ctx->d_stage, ctx->fld[field], z0, nzc, ctx->stream), "pf_upload convert");
        }
    }
    CK(cudaStreamSynchronize(ctx->stream), "pf_upload sync");
    return PF_OK;
}

int pf_download(pf_ctx* ctx, int field, double* host)
{
    if (!ctx || !host || field < 0 || field > 6) return ctx_err(ctx, PF_E_ARG, "pf_download: bad argument");
    const pf_grid& g = ctx->g;
    if (is64(ctx)) {
        CK(cudaMemcpy2DAsync(host, (size_t)g.nx * 8, ctx->fld[field], (size_t)ctx->dd.px * 8, (size_t)g.nx * 8,
                             (size_t)g.ny * g.nz, cudaMemcpyDeviceToHost, ctx->stream),
           "pf_download copy");
    } else {
        int rc = ensure_stage(ctx);
        if (rc) return rc;
        size_t plane = (size_t)g.nx * g.ny;
        long long zper = (long long)(ctx->stage_elems / plane);
        for (long long z0 = 0; z0 < g.nz; z0 += zper) {
            long long nzc = std::min<long long>(zper, g.nz - z0);
            CK(launch_convert_out<float>(ctx->dd, ctx->fld[field], ctx->d_stage, z0, nzc, ctx->stream), "pf_download convert");
            CK(cudaMemcpyAsync(host + z0 * plane, ctx->d_stage, nzc * plane * sizeof(double), cudaMemcpyDeviceToHost,
                               ctx->stream),
               "pf_download copy");
        }
    }
    CK(cudaStreamSynchronize(ctx->stream), "pf_download sync");
    return kernel_status(ctx);
}

int pf_probe(pf_ctx* ctx, int field, int i, int j, int k, double* value)
{
    if (!ctx || !value || field < 0 || field > 6) return ctx_err(ctx, PF_E_ARG, "pf_probe: bad argument");
    if (i < 1 || i > ctx->g.nx || j < 1 || j > ctx->g.ny || k < 1 || k > ctx->g.nz)
        return ctx_err(ctx, PF_E_ARG, "pf_probe: index out of range");
    size_t off = (size_t)(i - 1) + (size_t)ctx->dd.px * ((size_t)(j - 1) + (size_t)ctx->g.ny * (size_t)(k - 1));
    CK(cudaMemcpyAsync(ctx->h_out, (char*)ctx->fld[field] + off * ctx->es, ctx->es, cudaMemcpyDeviceToHost, ctx->stream),
       "pf_probe copy");
    CK(cudaStreamSynchronize(ctx->stream), "pf_probe sync");
    if (is64(ctx)) *value = ctx->h_out[0];
    else { float f; std::memcpy(&f, ctx->h_out, 4); *value = (double)f; }
    return PF_OK;
}

// ---- per-subroutine entry points ----

static Fields fields_of(const pf_ctx* ctx)
{
    Fields f;
    f.phi_old = ctx->fld[PF_PHASE_OLD];
    f.phi_new = ctx->fld[PF_PHASE_NEW];
    f.c_old = ctx->fld[PF_CONC_OLD];
    f.c_new = ctx->fld[PF_CONC_NEW];
    f.T_old = ctx->fld[PF_TOLD];
    f.T_new = ctx->fld[PF_TNEW];
    f.dpp = ctx->fld[PF_DPP];
    f.phi_mid = nullptr;
    return f;
}

int pf_temperatura(pf_ctx* ctx, double TP)
{
    if (!ctx) return PF_E_ARG;
    StepArgs s = make_step_args(ctx->p, ctx->dv, ctx->st.it, TP, TP, ctx->st.M0);
    Fields f = fields_of(ctx);
    CK(is64(ctx) ? launch_heat<double>(ctx->dd, s, f, ctx->stream) : launch_heat<float>(ctx->dd, s, f, ctx->stream),
       "temperatura");
    return PF_OK;
}

int pf_equacao_campo_fase(pf_ctx* ctx, int it, double TP, double M0, double* Cs_eq, double* Cl_eq)
{
    if (!ctx) return PF_E_ARG;
    StepArgs s = make_step_args(ctx->p, ctx->dv, it, TP, TP, M0);
    double Cs, Cl;
    equilibrium(ctx->p, TP, &Cs, &Cl);
    ctx->st.Cs_eq = Cs;
    ctx->st.Cl_eq = Cl;
    if (Cs_eq) *Cs_eq = Cs;
    if (Cl_eq) *Cl_eq = Cl;
    Fields f = fields_of(ctx);
    CK(is64(ctx) ? launch_phase<double>(ctx->dd, s, f.phi_old, f.c_old, f.phi_new, f.dpp, ctx->stream)
                 : launch_phase<float>(ctx->dd, s, f.phi_old, f.c_old, f.phi_new, f.dpp, ctx->stream),
       "equacao_campo_fase");
    return PF_OK;
}

int pf_copy_phase_new_to_old(pf_ctx* ctx)
{
    if (!ctx) return PF_E_ARG;
    CK(cudaMemcpyAsync(ctx->fld[PF_PHASE_OLD], ctx->fld[PF_PHASE_NEW], ctx->field_bytes, cudaMemcpyDeviceToDevice,
                       ctx->stream),
       "copy phase new->old");
    return PF_OK;
}

int pf_concentracao_soluto(pf_ctx* ctx)
{
    if (!ctx) return PF_E_ARG;
    StepArgs s = make_step_args(ctx->p, ctx->dv, ctx->st.it, ctx->st.TP, ctx->st.TP, ctx->st.M0);
    Fields f = fields_of(ctx);
    if (is64(ctx)) {
        CK(launch_solute<double>(ctx->dd, s, f.phi_old, f.c_old, f.c_new, ctx->stream), "concentracao_soluto");
        CK(launch_copy_inner<double>(ctx->dd, f.c_new, f.c_old, ctx->stream), "concentracao_soluto old=new");
    } else {
        CK(launch_solute<float>(ctx->dd, s, f.phi_old, f.c_old, f.c_new, ctx->stream), "concentracao_soluto");
        CK(launch_copy_inner<float>(ctx->dd, f.c_new, f.c_old, ctx->stream), "concentracao_soluto old=new");
    }
    return PF_OK;
}

int pf_auxiliar(const pf_ctx* ctx, double TP, double Cs_eq, double Cl_eq, double* M0)
{
    if (!ctx || !M0) return PF_E_ARG;
    return pf_auxiliar_scalar(&ctx->p, ctx->dv.E0, ctx->dv.W0, TP, Cs_eq, Cl_eq, M0);
}

static int run_diag(pf_ctx* ctx, const void* phi, const void* c, const void* Tw, double out[5])
{
    const void* dp = ctx->fld[PF_DPP];
    CK(is64(ctx) ? launch_diag<double>(ctx->dd, phi, c, Tw, dp, ctx->d_part, ctx->nblk, ctx->d_out, ctx->stream)
                 : launch_diag<float>(ctx->dd, phi, c, Tw, dp, ctx->d_part, ctx->nblk, ctx->d_out, ctx->stream),
       "diagnosticos");
    CK(cudaMemcpyAsync(ctx->h_out, ctx->d_out, 6 * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream), "diag copy");
    CK(cudaStreamSynchronize(ctx->stream), "diag sync");
    std::memcpy(out, ctx->h_out, 5 * sizeof(double));
    const int rc = kernel_status(ctx);
    if (rc != PF_OK) return rc;
    if (ctx->h_out[5] != 0.0)
        return ctx_err(ctx, PF_E_NONFINITE, "diagnosticos: " + std::to_string((long long)ctx->h_out[5]) +
                                                " cells hold a non-finite phi, c, T or DPP (the run has blown up)");
    return PF_OK;
}

int pf_diagnosticos(pf_ctx* ctx, double out[5])
{
    if (!ctx || !out) return PF_E_ARG;
    return run_diag(ctx, ctx->fld[PF_PHASE_NEW], ctx->fld[PF_CONC_NEW], ctx->fld[PF_TNEW], out);
}

int pf_track(pf_ctx* ctx, double out[3])
{
    if (!ctx || !out) return PF_E_ARG;
    CK(is64(ctx) ? launch_track<double>(ctx->dd, ctx->fld[PF_PHASE_OLD], ctx->d_track, ctx->d_track_out, ctx->stream)
                 : launch_track<float>(ctx->dd, ctx->fld[PF_PHASE_OLD], ctx->d_track, ctx->d_track_out, ctx->stream),
       "pf_track");
    CK(cudaMemcpyAsync(ctx->h_out, ctx->d_track_out, 3 * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream),
       "track copy");
    CK(cudaStreamSynchronize(ctx->stream), "track sync");
    std::memcpy(out, ctx->h_out, 3 * sizeof(double));
    return PF_OK;
}

// ---- checkpoints ----

int pf_checkpoint_wait(pf_ctx* ctx)
{
    if (!ctx) return PF_E_ARG;
    if (ctx->ckpt_thr.joinable()) ctx->ckpt_thr.join();
    const int rc = ctx->ckpt_rc;
    ctx->ckpt_rc = PF_OK;
    if (rc != PF_OK) return ctx_err(ctx, rc, "pf_checkpoint_save: " + ctx->ckpt_err);
    return PF_OK;
}

static int ckpt_host_buffer(pf_ctx* ctx, size_t bytes)
{
    if (ctx->ckpt_host_bytes >= bytes) return PF_OK;
    if (ctx->ckpt_host) cudaFreeHost(ctx->ckpt_host);
    ctx->ckpt_host = nullptr;
    ctx->ckpt_host_bytes = 0;
    CK(cudaMallocHost(&ctx->ckpt_host, bytes), "checkpoint host buffer");
    ctx->ckpt_host_bytes = bytes;
    return PF_OK;
}

int pf_checkpoint_save(pf_ctx* ctx, const char* path)
{
    if (!ctx || !path) return PF_E_ARG;
    int rc = pf_checkpoint_wait(ctx);   // one writer at a time
    if (rc != PF_OK) return rc;
    const pf_grid& g = ctx->g;
    const size_t row = (size_t)g.nx * ctx->es;
    const size_t fbytes = row * g.ny * g.nz;
    if ((rc = ckpt_host_buffer(ctx, 4 * fbytes)) != PF_OK) return rc;
    if (!ctx->ckpt_ev) CK(cudaEventCreateWithFlags(&ctx->ckpt_ev, cudaEventDisableTiming), "checkpoint event");
    for (int i = 0; i < 4; ++i)
        CK(cudaMemcpy2DAsync((char*)ctx->ckpt_host + i * fbytes, row, ctx->fld[kCkptFields[i]],
                             (size_t)ctx->dd.px * ctx->es, row, (size_t)g.ny * g.nz, cudaMemcpyDeviceToHost,
                             ctx->stream),
           "checkpoint copy");
    CK(cudaEventRecord(ctx->ckpt_ev, ctx->stream), "checkpoint event");
    // the host state of the copied fields: later steps are enqueued after them
    const CkptHeader h = ckpt_header(g, ctx->prec, ctx->st, ctx->p);
    const std::string file(path);
    void* data = ctx->ckpt_host;
    cudaEvent_t ev = ctx->ckpt_ev;
    ctx->ckpt_thr = std::thread([ctx, h, file, data, fbytes, ev]() {
        cudaError_t e = cudaEventSynchronize(ev);
        if (e != cudaSuccess) {
            ctx->ckpt_err = std::string("copy: ") + cudaGetErrorString(e);
            ctx->ckpt_rc = PF_E_CUDA;
            return;
        }
        std::string why = ckpt_write(file, h, data, fbytes);
        if (!why.empty()) {
            ctx->ckpt_err = why;
            ctx->ckpt_rc = PF_E_STATE;
        }
    });
    return PF_OK;
}

int pf_checkpoint_load(pf_ctx* ctx, const char* path)
{
    if (!ctx || !path) return PF_E_ARG;
    int rc = pf_checkpoint_wait(ctx);
    if (rc != PF_OK) return rc;
    std::FILE* f = std::fopen(path, "rb");
    if (!f) return ctx_err(ctx, PF_E_ARG, std::string("pf_checkpoint_load: cannot open ") + path);
    CkptHeader h;
    std::string why = ckpt_read_header(f, ctx->g, ctx->prec, ctx->p, &h);
    const pf_grid& g = ctx->g;
    const size_t row = (size_t)g.nx * ctx->es;
    const size_t fbytes = row * g.ny * g.nz;
    if (why.empty() && ckpt_host_buffer(ctx, 4 * fbytes) != PF_OK) why = "cannot allocate the host buffer";
    if (why.empty() && std::fread(ctx->ckpt_host, fbytes, 4, f) != 4) why = "checkpoint shorter than its fields";
    std::fclose(f);
    if (!why.empty()) return ctx_err(ctx, PF_E_ARG, "pf_checkpoint_load: " + why);
    for (int i = 0; i < 4; ++i)
        CK(cudaMemcpy2DAsync(ctx->fld[kCkptFields[i]], (size_t)ctx->dd.px * ctx->es,
                             (const char*)ctx->ckpt_host + i * fbytes, row, row, (size_t)g.ny * g.nz,
                             cudaMemcpyHostToDevice, ctx->stream),
           "checkpoint upload");
    CK(cudaStreamSynchronize(ctx->stream), "checkpoint sync");
    ctx->st = ckpt_state(h);
    return PF_OK;
}

// ---- moving frame ----

int pf_shift_frame(pf_ctx* ctx, int k_desl)
{
    if (!ctx) return PF_E_ARG;
    if (k_desl < 0 || k_desl >= ctx->g.nz)
        return ctx_err(ctx, PF_E_ARG, "pf_shift_frame: the shift must be in [0, nz)");   // entrada.f90:292
    const long long n = (long long)ctx->field_bytes / (long long)ctx->es;
    void*& po = ctx->fld[PF_PHASE_OLD];
    void*& pn = ctx->fld[PF_PHASE_NEW];
    void*& co = ctx->fld[PF_CONC_OLD];
    void*& cn = ctx->fld[PF_CONC_NEW];
    CK(is64(ctx) ? launch_shift_frame<double>(ctx->dd, k_desl, po, co, pn, cn, ctx->stream)
                 : launch_shift_frame<float>(ctx->dd, k_desl, po, co, pn, cn, ctx->stream),
       "pf_shift_frame");
    std::swap(po, pn);
    std::swap(co, cn);
    CK(cudaMemcpyAsync(cn, co, ctx->field_bytes, cudaMemcpyDeviceToDevice, ctx->stream), "shift: c_new");
    CK(cudaMemsetAsync(pn, 0, ctx->field_bytes, ctx->stream), "shift: phi_new");
    CK(cudaMemsetAsync(ctx->fld[PF_DPP], 0, ctx->field_bytes, ctx->stream), "shift: DPP");
    for (int fidx : {PF_TOLD, PF_TNEW})
        CK(is64(ctx) ? launch_fill<double>(ctx->fld[fidx], n, ctx->p.T0, ctx->stream)
                     : launch_fill<float>(ctx->fld[fidx], n, ctx->p.T0, ctx->stream),
           "shift: T");
    return PF_OK;
}

int pf_swap(pf_ctx* ctx)
{
    if (!ctx) return PF_E_ARG;
    std::swap(ctx->fld[PF_PHASE_OLD], ctx->fld[PF_PHASE_NEW]);
    std::swap(ctx->fld[PF_TOLD], ctx->fld[PF_TNEW]);
    std::swap(ctx->fld[PF_CONC_OLD], ctx->fld[PF_CONC_NEW]);
    return PF_OK;
}

// ---- fused step ----

static cudaEvent_t new_event()
{
    cudaEvent_t e;
    cudaEventCreate(&e);
    return e;
}

static int one_step(pf_ctx* ctx)
{
    const pf_params& p = ctx->p;
    const int it = ctx->st.it + 1;
    const double dt = ctx->dv.DELTA_T;
    ctx->st.time = (float)(dt + (double)ctx->st.time);          // principal.f90:96 (REAL(4) time)
    const double TP_heat = ctx->st.TP;                          // temperatura sees the previous TP
    const double TP = step_tp(p, dt, it, ctx->st.TP);           // principal.f90:104
    const StepArgs s = make_step_args(ctx->p, ctx->dv, it, TP_heat, TP, ctx->st.M0);
    const int nsw = p.n_varreduras;
    void* A = ctx->fld[PF_PHASE_OLD];
    void* B = ctx->fld[PF_PHASE_NEW];
    Fields f = fields_of(ctx);
    void* final_phi;
    void* other_phi;
    const bool march = ctx->fused && ctx->kernel == 1 && ctx->tmap_ok && ctx->tile_y == 8;
    if (march) {
        // TMA-staged passes: two cells per thread unless PF_OPT_PAIRED says
        // otherwise (default: FP32 only) or the deck draws the smooth noise
        const int lanes = ((ctx->paired == 2 || (ctx->paired == 1 && !is64(ctx))) && p.ruido_tipo != 2) ? 2 : 1;
        const int nslot = ctx->nslot ? ctx->nslot : 3;
        auto tm_of = [ctx](const void* buf) -> const CUtensorMap& {
            return ctx->tmap[buf == ctx->tmap_buf[0] ? 0 : 1];
        };
        cudaEvent_t e0 = nullptr, e1 = nullptr;
        f.phi_mid = B;
        if (ctx->ktiming) { e0 = new_event(); e1 = new_event(); cudaEventRecord(e0, ctx->stream); }
        CK(is64(ctx) ? launch_march_first<double>(tm_of(A), ctx->dd, s, f, nsw == 1, lanes, nslot, ctx->zchunk,
                                                  ctx->d_status, ctx->stream)
                     : launch_march_first<float>(tm_of(A), ctx->dd, s, f, nsw == 1, lanes, nslot, ctx->zchunk,
                                                 ctx->d_status, ctx->stream),
           nsw == 1 ? "march step (single sweep)" : "march heat + sweep 1");
        if (ctx->ktiming) { cudaEventRecord(e1, ctx->stream); ctx->ev_first.push_back({e0, e1}); }
        if (nsw == 1) {
            final_phi = B;
            other_phi = A;
        } else {
            void* cur = B;   // phase after the sweeps so far
            void* oth = A;   // free buffer
            for (int sw = 2; sw <= nsw - 1; ++sw) {
                // no DPP: it carries the step's noise from the first to the last pass
                CK(is64(ctx) ? launch_phase<double>(ctx->dd, s, cur, f.c_old, oth, nullptr, ctx->stream)
                             : launch_phase<float>(ctx->dd, s, cur, f.c_old, oth, nullptr, ctx->stream),
                   "middle sweep");
                std::swap(cur, oth);
            }
            Fields f2 = f;
            f2.phi_mid = cur;
            f2.phi_new = oth;
            if (ctx->ktiming) { e0 = new_event(); e1 = new_event(); cudaEventRecord(e0, ctx->stream); }
            CK(is64(ctx) ? launch_march_last<double>(tm_of(cur), ctx->dd, s, f2, lanes, nslot, ctx->zchunk,
                                                     ctx->d_status, ctx->stream)
                         : launch_march_last<float>(tm_of(cur), ctx->dd, s, f2, lanes, nslot, ctx->zchunk,
                                                    ctx->d_status, ctx->stream),
               "march last sweep + solute");
            if (ctx->ktiming) { cudaEventRecord(e1, ctx->stream); ctx->ev_last.push_back({e0, e1}); }
            final_phi = oth;
            other_phi = cur;
        }
    } else if (ctx->fused) {
        // two cells per thread on 32 x 8 tiles; the smooth noise keeps one
        const bool pair = (ctx->paired == 2 || (ctx->paired == 1 && !is64(ctx))) && ctx->tile_y == 8 &&
                          p.ruido_tipo != 2 && !ctx->dd.do_heat_lap;
        if (nsw == 1) {
            f.phi_mid = B;
            cudaEvent_t e0 = nullptr, e1 = nullptr;
            if (ctx->ktiming) { e0 = new_event(); e1 = new_event(); cudaEventRecord(e0, ctx->stream); }
            CK(pair ? (is64(ctx) ? launch_fused_first_pair<double>(ctx->dd, s, f, true, ctx->zchunk, ctx->stream)
                                 : launch_fused_first_pair<float>(ctx->dd, s, f, true, ctx->zchunk, ctx->stream))
                    : (is64(ctx) ? launch_fused_first<double>(ctx->dd, s, f, true, ctx->tile_y, ctx->zchunk, ctx->stream)
                                 : launch_fused_first<float>(ctx->dd, s, f, true, ctx->tile_y, ctx->zchunk, ctx->stream)),
               "fused step (single sweep)");
            if (ctx->ktiming) { cudaEventRecord(e1, ctx->stream); ctx->ev_first.push_back({e0, e1}); }
            final_phi = B;
            other_phi = A;
        } else {
            f.phi_mid = B;
            cudaEvent_t e0 = nullptr, e1 = nullptr;
            if (ctx->ktiming) { e0 = new_event(); e1 = new_event(); cudaEventRecord(e0, ctx->stream); }
            CK(pair ? (is64(ctx) ? launch_fused_first_pair<double>(ctx->dd, s, f, false, ctx->zchunk, ctx->stream)
                                 : launch_fused_first_pair<float>(ctx->dd, s, f, false, ctx->zchunk, ctx->stream))
                    : (is64(ctx) ? launch_fused_first<double>(ctx->dd, s, f, false, ctx->tile_y, ctx->zchunk, ctx->stream)
                                 : launch_fused_first<float>(ctx->dd, s, f, false, ctx->tile_y, ctx->zchunk, ctx->stream)),
               "fused heat + sweep 1");
            if (ctx->ktiming) { cudaEventRecord(e1, ctx->stream); ctx->ev_first.push_back({e0, e1}); }
            void* cur = B;   // phase after the sweeps so far
            void* oth = A;   // free buffer
            for (int sw = 2; sw <= nsw - 1; ++sw) {
                // no DPP: it carries the step's noise from the first to the last pass
                CK(is64(ctx) ? launch_phase<double>(ctx->dd, s, cur, f.c_old, oth, nullptr, ctx->stream)
                             : launch_phase<float>(ctx->dd, s, cur, f.c_old, oth, nullptr, ctx->stream),
                   "middle sweep");
                std::swap(cur, oth);
            }
            Fields f2 = f;
            f2.phi_mid = cur;
            f2.phi_new = oth;
            if (ctx->ktiming) { e0 = new_event(); e1 = new_event(); cudaEventRecord(e0, ctx->stream); }
            CK(pair ? (is64(ctx) ? launch_fused_last_pair<double>(ctx->dd, s, f2, ctx->zchunk, ctx->stream)
                                 : launch_fused_last_pair<float>(ctx->dd, s, f2, ctx->zchunk, ctx->stream))
                    : (is64(ctx) ? launch_fused_last<double>(ctx->dd, s, f2, ctx->tile_y, ctx->zchunk, ctx->stream)
                                 : launch_fused_last<float>(ctx->dd, s, f2, ctx->tile_y, ctx->zchunk, ctx->stream)),
               "fused last sweep + solute");
            if (ctx->ktiming) { cudaEventRecord(e1, ctx->stream); ctx->ev_last.push_back({e0, e1}); }
            final_phi = oth;
            other_phi = cur;
        }
    } else {
        // per-subroutine kernels in the reference's order
        CK(is64(ctx) ? launch_heat<double>(ctx->dd, s, f, ctx->stream) : launch_heat<float>(ctx->dd, s, f, ctx->stream),
           "temperatura");
        void* in = A;
        void* out = B;
        for (int sw = 1; sw <= nsw; ++sw) {
            if (sw > 1) std::swap(in, out);   // the copy new -> old, by exchange
            CK(is64(ctx) ? launch_phase<double>(ctx->dd, s, in, f.c_old, out, f.dpp, ctx->stream)
                         : launch_phase<float>(ctx->dd, s, in, f.c_old, out, f.dpp, ctx->stream),
               "equacao_campo_fase");
        }
        CK(is64(ctx) ? launch_solute<double>(ctx->dd, s, in, f.c_old, f.c_new, ctx->stream)
                     : launch_solute<float>(ctx->dd, s, in, f.c_old, f.c_new, ctx->stream),
           "concentracao_soluto");
        final_phi = out;
        other_phi = in;
    }
    // swap (principal.f90:200-226) by exchanging buffers
    ctx->fld[PF_PHASE_OLD] = final_phi;
    ctx->fld[PF_PHASE_NEW] = other_phi;
    std::swap(ctx->fld[PF_CONC_OLD], ctx->fld[PF_CONC_NEW]);
    std::swap(ctx->fld[PF_TOLD], ctx->fld[PF_TNEW]);
    // auxiliar (principal.f90:157): M0 for the next step
    double Cs, Cl;
    equilibrium(p, TP, &Cs, &Cl);
    double M0n;
    pf_auxiliar_scalar(&p, ctx->dv.E0, ctx->dv.W0, TP, Cs, Cl, &M0n);
    ctx->st.M0 = M0n;
    ctx->st.TP = TP;
    ctx->st.Cs_eq = Cs;
    ctx->st.Cl_eq = Cl;
    ctx->st.it = it;
    return PF_OK;
}

int pf_step(pf_ctx* ctx, int n_steps)
{
    if (!ctx || n_steps < 0) return ctx_err(ctx, PF_E_ARG, "pf_step: bad argument");
    for (int n = 0; n < n_steps; ++n) {
        int rc = one_step(ctx);
        if (rc) return rc;
    }
    return PF_OK;
}

int pf_step_diag(pf_ctx* ctx, int n_steps, double out[5])
{
    int rc = pf_step(ctx, n_steps);
    if (rc) return rc;
    // after the exchange the final state sits in the "old" buffers
    return run_diag(ctx, ctx->fld[PF_PHASE_OLD], ctx->fld[PF_CONC_OLD], ctx->fld[PF_TOLD], out);
}

int pf_init_seeded(pf_ctx* ctx, int n_bumps, const double* sites)
{
    if (!ctx || n_bumps < 0 || n_bumps > 4096 || (n_bumps > 0 && !sites))
        return ctx_err(ctx, PF_E_ARG, "pf_init_seeded: bad argument (at most 4096 bumps)");
    int rc = ensure_stage(ctx);
    if (rc) return rc;
    InitArgs a;
    a.n_bumps = n_bumps;
    a.slab_top = 4.5;
    a.bump_r = 3.0;
    a.width = ctx->p.Thin_Interface;
    a.kmax = std::min(ctx->g.nz, (int)(a.slab_top + a.bump_r + 20.0 * a.width / 2.0) + 2);
    a.C0 = ctx->p.C0;
    a.Ke = (double)ctx->p.Ke;
    a.T0 = ctx->p.T0;
    if (n_bumps)
        CK(cudaMemcpyAsync(ctx->d_stage, sites, 2 * n_bumps * sizeof(double), cudaMemcpyHostToDevice, ctx->stream),
           "bump sites");
    Fields f = fields_of(ctx);
    CK(is64(ctx) ? launch_init_seeded<double>(ctx->dd, a, ctx->d_stage, f.phi_old, f.c_old, f.T_old, f.dpp, ctx->stream)
                 : launch_init_seeded<float>(ctx->dd, a, ctx->d_stage, f.phi_old, f.c_old, f.T_old, f.dpp, ctx->stream),
       "pf_init_seeded");
    CK(cudaStreamSynchronize(ctx->stream), "pf_init_seeded sync");
    return PF_OK;
}

int pf_kernel_times(pf_ctx* ctx, long* n_first, double* ms_first, long* n_last, double* ms_last, int reset)
{
    if (!ctx) return PF_E_ARG;
    CK(cudaStreamSynchronize(ctx->stream), "pf_kernel_times sync");
    double a = 0, b = 0;
    for (auto& pr : ctx->ev_first) { float ms = 0; cudaEventElapsedTime(&ms, pr.first, pr.second); a += ms; }
    for (auto& pr : ctx->ev_last) { float ms = 0; cudaEventElapsedTime(&ms, pr.first, pr.second); b += ms; }
    if (n_first) *n_first = (long)ctx->ev_first.size();
    if (ms_first) *ms_first = a;
    if (n_last) *n_last = (long)ctx->ev_last.size();
    if (ms_last) *ms_last = b;
    if (reset) drop_events(ctx);
    return PF_OK;
}

int pf_math_log(const double* x, long long n, double* own, double* lib)
{
    if (n < 0 || (n > 0 && (!x || !own || !lib)) || n > (1LL << 28))
        return ctx_err(nullptr, PF_E_ARG, "pf_math_log: bad argument");
    if (n == 0) return PF_OK;
    const size_t bytes = (size_t)n * sizeof(double);
    double* d = nullptr;
    if (int rc = cuda_check(nullptr, cudaMalloc(&d, 3 * bytes), "pf_math_log alloc")) return rc;
    cudaError_t e = cudaMemcpy(d, x, bytes, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = launch_math_log(d, d + n, d + 2 * n, n, 0);
    if (e == cudaSuccess) e = cudaMemcpy(own, d + n, bytes, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(lib, d + 2 * n, bytes, cudaMemcpyDeviceToHost);
    cudaFree(d);
    return cuda_check(nullptr, e, "pf_math_log");
}

}  // extern "C"
