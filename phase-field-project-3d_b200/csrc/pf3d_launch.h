// pf3d_launch.h -- host-side launcher declarations.  The definitions are
// templates in pf3d_kernels.cuh, instantiated for double in pf3d_fp64.cu
// (built with --fmad=false) and for float in pf3d_fp32.cu.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>
#include "pf3d_device.cuh"

namespace pf3d {

// Device pointers of one domain.  "old"/"new" follow the reference names.
struct Fields {
    void* phi_old;
    void* phi_new;
    void* c_old;
    void* c_new;
    void* T_old;
    void* T_new;
    void* dpp;
    void* phi_mid;   // fused step: the sweep-1 phase field
};

// Per-subroutine kernels (one thread per cell, reference form).
template <typename T> cudaError_t launch_heat(const DomainDesc& d, const StepArgs& s, const Fields& f, cudaStream_t st);
template <typename T> cudaError_t launch_phase(const DomainDesc& d, const StepArgs& s, const void* phi_in,
                                               const void* c_in, void* phi_out, void* dpp, cudaStream_t st);
template <typename T> cudaError_t launch_solute(const DomainDesc& d, const StepArgs& s, const void* phi_in,
                                                const void* c_in, void* c_out, cudaStream_t st);
template <typename T> cudaError_t launch_copy_inner(const DomainDesc& d, const void* src, void* dst, cudaStream_t st);

// Fused z-marching kernels.
//   first  : temperatura + phase sweep 1 (phi_old -> phi_mid), or with
//            solute as well when there is a single sweep
//   last   : final phase sweep (phi_mid -> phi_new) + solute from phi_mid
//   The first pass of a multi-sweep step leaves the step's noise in the DPP
//   buffer for the last pass; sweeps in between must not write DPP.
template <typename T> cudaError_t launch_fused_first(const DomainDesc& d, const StepArgs& s, const Fields& f,
                                                     bool with_solute, int tile_y, int zchunk, cudaStream_t st);
// the same passes with two cells per thread (32 x 8 tiles, no smooth noise)
template <typename T> cudaError_t launch_fused_first_pair(const DomainDesc& d, const StepArgs& s, const Fields& f,
                                                          bool with_solute, int zchunk, cudaStream_t st);
template <typename T> cudaError_t launch_fused_last_pair(const DomainDesc& d, const StepArgs& s, const Fields& f,
                                                         int zchunk, cudaStream_t st);
template <typename T> cudaError_t launch_fused_last(const DomainDesc& d, const StepArgs& s, const Fields& f,
                                                    int tile_y, int zchunk, cudaStream_t st);

// ---- batches of independent domains (persistent work-list kernels) ----
struct BatchDomain {
    DomainDesc d;
    void* phi[2];    // phase field buffers
    void* c[2];      // solute buffers
    void* T[2];      // temperature buffers
    void* dpp;
};
// per domain and step: the step scalars, whether the domain advances in this
// step, and which buffer of each pair holds the "old" field
struct BatchStep {
    StepArgs s;
    int active;
    int q_phi, q_c, q_T;
    int pad_;
    // the loop constants of this domain and step, KC<T> of the batch's type
    alignas(16) unsigned char kc[sizeof(KC<double>)];
};
struct BatchItem {
    int dom, bx, by, bz;
};
template <typename T> cudaError_t launch_fused_batch(const BatchDomain* doms, const BatchStep* steps,
                                                     const BatchItem* items, const int* n_items, int pass,
                                                     bool one_sweep, bool smooth, int tile_y, int zchunk,
                                                     int n_sm, cudaStream_t st);
// the batch passes with two cells per thread (32 x 8 tiles, no smooth noise,
// no heat diffusion)
template <typename T> cudaError_t launch_fused_batch_pair(const BatchDomain* doms, const BatchStep* steps,
                                                          const BatchItem* items, const int* n_items, int pass,
                                                          bool one_sweep, int zchunk, int n_sm, cudaStream_t st);

// TMA-staged z-marching passes (pf3d_march.cuh): 32 x 8 tiles, the input
// phase field through the tensor map `tm`, `lanes` cells per thread (1 or 2),
// `nslot` node-window planes (3 or 4); a plane load that does not arrive sets
// *err.  Same outputs, bit for bit, as launch_fused_first / _last.
template <typename S> cudaError_t launch_march_first(const CUtensorMap& tm, const DomainDesc& d, const StepArgs& s,
                                                     const Fields& f, bool with_solute, int lanes, int nslot,
                                                     int zchunk, int* err, cudaStream_t st);
template <typename S> cudaError_t launch_march_last(const CUtensorMap& tm, const DomainDesc& d, const StepArgs& s,
                                                    const Fields& f, int lanes, int nslot, int zchunk, int* err,
                                                    cudaStream_t st);
// batch form: tmaps[2 d + b] is the tensor map of buffer b of domain d's
// phase field; *ctr (zero before the launch) hands out the work items
template <typename S> cudaError_t launch_march_batch(const BatchDomain* doms, const CUtensorMap* tmaps,
                                                     const BatchStep* steps, const BatchItem* items,
                                                     const int* n_items, int pass, bool one_sweep, bool smooth,
                                                     int lanes, int nslot, int zchunk, int n_sm, int* ctr,
                                                     int* err, cudaStream_t st);

// Solidification tracking of phi: out[3] = {solid fraction, tip position
// (cells, 1-based), solid cells}; scratch holds nz + 1 words.
template <typename T> cudaError_t launch_track(const DomainDesc& d, const void* phi, unsigned long long* scratch,
                                               double* out, cudaStream_t st);

// Moving frame (restart with a shift of kd planes) into the "new" buffers;
// fill of n elements with v.
template <typename T> cudaError_t launch_shift_frame(const DomainDesc& d, int kd, const void* phi_o, const void* c_o,
                                                     void* phi_n, void* c_n, cudaStream_t st);
template <typename T> cudaError_t launch_fill(void* a, long long n, double v, cudaStream_t st);

// Diagnostics: block partials into part[nblk*kDiagRow], final into out[6]:
// the five values of diagnosticos and the count of cells whose phi or c is
// not finite (the watchdog).
constexpr int kDiagRow = 10;   // l2, l2 comp, max, min, sol, sol comp, fe, fe comp, non-finite cells, pad
// Tw and dpp (may be null): the temperature and DPP fields the watchdog
// also checks for non-finite values.
template <typename T> cudaError_t launch_diag(const DomainDesc& d, const void* phi, const void* c, const void* Tw,
                                              const void* dppw, double* part, int nblk, double* out, cudaStream_t st);

// FP64 host array (Fortran order, nx*ny*nz) <-> pitched device field of T,
// through a device staging buffer of doubles (FP32 contexts only).
template <typename T> cudaError_t launch_convert_in(const DomainDesc& d, const double* stage, void* dst, long long z0,
                                                    long long nz, cudaStream_t st);
template <typename T> cudaError_t launch_convert_out(const DomainDesc& d, const void* src, double* stage, long long z0,
                                                     long long nz, cudaStream_t st);

// Self-check of the fast form's FP64 logarithm: own[i] = pf_log(x[i]),
// lib[i] = the CUDA library's log(x[i]).
cudaError_t launch_math_log(const double* x, double* own, double* lib, long long n, cudaStream_t st);

}  // namespace pf3d
