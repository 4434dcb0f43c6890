// pf3d_simple.cuh -- one-thread-per-cell kernels behind the per-subroutine
// entry points (pf_temperatura, pf_equacao_campo_fase, pf_concentracao_soluto,
// pf_diagnosticos).  Each cell is computed in the reference form (six anisotropy
// nodes per cell, seven solute points per cell); the boundary decoration is
// applied in closed form by the thread that owns the source cell.
#pragma once
#include <cfloat>
#include "pf3d_launch.h"

namespace pf3d {

__device__ __forceinline__ long long cell_off(const DomainDesc& d, int x, int y, int z)
{
    return (long long)x + (long long)y * d.px + (long long)z * d.plane;
}

// ---- temperatura.f90 (TNEW = TOLD; temp_body.inc on 2..N-1) ----
template <typename T>
__global__ void __launch_bounds__(256) k_heat(DomainDesc d, StepArgs s, const T* __restrict__ Told,
                                              const T* __restrict__ phi, const T* __restrict__ dpp,
                                              T* __restrict__ Tnew)
{
    int x = blockIdx.x * 32 + threadIdx.x, y = blockIdx.y * 8 + threadIdx.y, z = blockIdx.z;
    if (x >= d.nx || y >= d.ny) return;
    long long id = cell_off(d, x, y, z);
    bool inner = x >= 1 && x <= d.nx - 2 && y >= 1 && y <= d.ny - 2 && z >= 1 && z <= d.nz - 2;
    if (!inner) { Tnew[id] = Told[id]; return; }
    KC<T> c;
    c.load(d, s);
    T TE = 0, TW = 0, TN = 0, TS = 0, TT = 0, TB = 0;
    if (c.lap) {
        TE = Told[id + 1]; TW = Told[id - 1]; TN = Told[id + d.px]; TS = Told[id - d.px];
        TT = Told[id + d.plane]; TB = Told[id - d.plane];
    }
    Tnew[id] = heat_new<T>(phi[id], dpp[id], TE, TW, TN, TS, TT, TB, c);
}

// ---- equacao_campo_fase.f90 (copy, phase_body.inc on 3..N-2, decoration) ----
template <typename T>
__global__ void __launch_bounds__(256) k_phase(DomainDesc d, StepArgs s, const T* __restrict__ po,
                                               const T* __restrict__ co, T* __restrict__ pn, T* __restrict__ dpp)
{
    int x = blockIdx.x * 32 + threadIdx.x, y = blockIdx.y * 8 + threadIdx.y, z = blockIdx.z;
    if (x >= d.nx || y >= d.ny) return;
    // only cells with every coordinate in [1, N-2] are decoration sources
    if (x < 1 || x > d.nx - 2 || y < 1 || y > d.ny - 2 || z < 1 || z > d.nz - 2) return;
    long long id = cell_off(d, x, y, z);
    T U;
    if (x >= 2 && x <= d.nx - 3 && y >= 2 && y <= d.ny - 3 && z >= 2 && z <= d.nz - 3) {
        constexpr bool FAST = sizeof(T) == 4;   // FP64: the reference form
        KC<T> c;
        c.load(d, s);
        const T* p = po + id;
        const long long sy = d.px, sz = d.plane;
        auto P = [&](int a, int b, int e) -> T { return p[a + b * sy + e * sz]; };
        Nbr<T> nb;
        nb.PP = P(0, 0, 0);
        nb.PN = P(0, 1, 0); nb.PS = P(0, -1, 0); nb.PE = P(1, 0, 0); nb.PW = P(-1, 0, 0);
        nb.PT = P(0, 0, 1); nb.PB = P(0, 0, -1);
        nb.PNE = P(1, 1, 0); nb.PSE = P(1, -1, 0); nb.PNW = P(-1, 1, 0); nb.PSW = P(-1, -1, 0);
        nb.PNT = P(0, 1, 1); nb.PNB = P(0, 1, -1); nb.PST = P(0, -1, 1); nb.PSB = P(0, -1, -1);
        nb.PET = P(1, 0, 1); nb.PEB = P(1, 0, -1); nb.PWT = P(-1, 0, 1); nb.PWB = P(-1, 0, -1);
        Node<T> E = aniso_node<T, FAST>(grad<T, FAST>(P(2, 0, 0), nb.PP, c.dx, c.hx), grad<T, FAST>(P(1, 1, 0), P(1, -1, 0), c.dy, c.hy),
                                  grad<T, FAST>(P(1, 0, 1), P(1, 0, -1), c.dz, c.hz), c);
        Node<T> W = aniso_node<T, FAST>(grad<T, FAST>(nb.PP, P(-2, 0, 0), c.dx, c.hx), grad<T, FAST>(P(-1, 1, 0), P(-1, -1, 0), c.dy, c.hy),
                                  grad<T, FAST>(P(-1, 0, 1), P(-1, 0, -1), c.dz, c.hz), c);
        Node<T> N = aniso_node<T, FAST>(grad<T, FAST>(P(1, 1, 0), P(-1, 1, 0), c.dx, c.hx), grad<T, FAST>(P(0, 2, 0), nb.PP, c.dy, c.hy),
                                  grad<T, FAST>(P(0, 1, 1), P(0, 1, -1), c.dz, c.hz), c);
        Node<T> S = aniso_node<T, FAST>(grad<T, FAST>(P(1, -1, 0), P(-1, -1, 0), c.dx, c.hx), grad<T, FAST>(nb.PP, P(0, -2, 0), c.dy, c.hy),
                                  grad<T, FAST>(P(0, -1, 1), P(0, -1, -1), c.dz, c.hz), c);
        Node<T> Tt = aniso_node<T, FAST>(grad<T, FAST>(P(1, 0, 1), P(-1, 0, 1), c.dx, c.hx), grad<T, FAST>(P(0, 1, 1), P(0, -1, 1), c.dy, c.hy),
                                   grad<T, FAST>(P(0, 0, 2), nb.PP, c.dz, c.hz), c);
        Node<T> B = aniso_node<T, FAST>(grad<T, FAST>(P(1, 0, -1), P(-1, 0, -1), c.dx, c.hx), grad<T, FAST>(P(0, 1, -1), P(0, -1, -1), c.dy, c.hy),
                                  grad<T, FAST>(nb.PP, P(0, 0, -2), c.dz, c.hz), c);
        float ran = phase_ran(c.rt, x + 1, y + 1, z + 1, c.it);
        T ppn = phase_ppnew<T, FAST>(nb, E, W, N, S, Tt, B, co[id], ran, c);
        if (dpp) dpp[id] = ppn - nb.PP;   // the fused step's middle sweeps pass no DPP
        U = clamp01(ppn);
    } else {
        U = po[id];
    }
    int xl, xh, yl, yh, zl, zh;
    fpre_range(x, d.nx, &xl, &xh);
    fpre_range(y, d.ny, &yl, &yh);
    fpre_range(z, d.nz, &zl, &zh);
    for (int zz = zl; zz <= zh; ++zz)
        for (int yy = yl; yy <= yh; ++yy)
            for (int xx = xl; xx <= xh; ++xx) pn[cell_off(d, xx, yy, zz)] = U;
}

// ---- concentracao_soluto.f90 (conc_body.inc on 2..N-1, decoration) ----
template <typename T>
__global__ void __launch_bounds__(256) k_solute(DomainDesc d, StepArgs s, const T* __restrict__ po,
                                                const T* __restrict__ co, T* __restrict__ cn)
{
    int x = blockIdx.x * 32 + threadIdx.x, y = blockIdx.y * 8 + threadIdx.y, z = blockIdx.z;
    if (x >= d.nx || y >= d.ny) return;
    long long id = cell_off(d, x, y, z);
    const int nx = d.nx, ny = d.ny, nz = d.nz;
    bool xin = x >= 1 && x <= nx - 2, yin = y >= 1 && y <= ny - 2, zin = z >= 1 && z <= nz - 2;
    bool inner = xin && yin && zin;
    // only inner cells, or cells one plane from a wall, feed a write
    bool feeds = inner || z == 1 || z == nz - 2 || (zin && (x == 1 || x == nx - 2));
    if (!feeds) return;
    T U;
    if (inner) {
        constexpr bool FAST = sizeof(T) == 4;
        KC<T> c;
        c.load(d, s);
        const long long sy = d.px, sz = d.plane;
        T PP = po[id];
        SolNode<T> nP = sol_node<T, FAST>(PP, co[id], c);
        SolNode<T> nE = sol_node<T, FAST>(po[id + 1], co[id + 1], c);
        SolNode<T> nW = sol_node<T, FAST>(po[id - 1], co[id - 1], c);
        SolNode<T> nN = sol_node<T, FAST>(po[id + sy], co[id + sy], c);
        SolNode<T> nS = sol_node<T, FAST>(po[id - sy], co[id - sy], c);
        SolNode<T> nT = sol_node<T, FAST>(po[id + sz], co[id + sz], c);
        SolNode<T> nB = sol_node<T, FAST>(po[id - sz], co[id - sz], c);
        U = conc_new<T, FAST>(PP, co[id], nP, nE, nW, nN, nS, nT, nB, c);
        cn[id] = U;
    } else {
        U = co[id];
    }
    // last writer wins in the order y, x, z faces (concentracao_soluto.f90:119-124)
    if (z == 1) cn[cell_off(d, x, y, 0)] = U;
    if (z == nz - 2) cn[cell_off(d, x, y, nz - 1)] = U;
    if (zin && x == 1) cn[cell_off(d, 0, y, z)] = U;
    if (zin && x == nx - 2) cn[cell_off(d, nx - 1, y, z)] = U;
    if (zin && xin && y == 1) cn[cell_off(d, x, 0, z)] = U;
    if (zin && xin && y == ny - 2) cn[cell_off(d, x, ny - 1, z)] = U;
}

// conc_soluto_old = conc_soluto_new on 2..N-1 (the wall cells of
// conc_soluto_old keep their values; concentracao_soluto.f90:116)
template <typename T>
__global__ void __launch_bounds__(256) k_copy_inner(DomainDesc d, const T* __restrict__ src, T* __restrict__ dst)
{
    int x = blockIdx.x * 32 + threadIdx.x, y = blockIdx.y * 8 + threadIdx.y, z = blockIdx.z;
    if (x < 1 || x > d.nx - 2 || y < 1 || y > d.ny - 2 || z < 1 || z > d.nz - 2) return;
    long long id = cell_off(d, x, y, z);
    dst[id] = src[id];
}

// ---- diagnosticos.f90 + diag_body.inc ----
// FP64 accumulation with Neumaier compensation; max/min exact and NaN-
// propagating (fmax/fmin would drop a NaN and report finite extremes for a
// blown-up field); plus the watchdog: the count of cells where phi, c, or
// (when given) T or DPP is not finite.  The clamp of the phase update maps a
// NaN or infinite update to 1, so a blow-up can leave phi finite and show
// only in DPP and T.  Partials: kDiagRow doubles per block (pf3d_launch.h).

// max / min that return NaN when either argument is NaN
__device__ __forceinline__ double nan_max(double a, double b) { return (a > b || a != a) ? a : b; }
__device__ __forceinline__ double nan_min(double a, double b) { return (a < b || a != a) ? a : b; }
struct KSum {
    double s, c;
    __device__ __forceinline__ void add(double v)
    {
        double t = s + v;
        if (fabs(s) >= fabs(v)) c += (s - t) + v;
        else c += (v - t) + s;
        s = t;
    }
    __device__ __forceinline__ void merge(double os, double oc)
    {
        add(os);
        c += oc;
    }
};

// The grid walks 32 x 8-column tiles, each marched along z over a chunk of
// kDiagZ planes (a persistent grid: block b takes tiles b, b + gridDim.x,
// ...; the per-thread sums carry across its tiles, so the reduction order is
// fixed by the launch shape).  The march goes in groups of kDiagG planes: a
// thread first issues the reads of the whole group -- phi of the next
// kDiagG planes and c, T, DPP of the group's planes, each cell read once from
// HBM, all in flight together -- then shares the group's phase planes
// through shared memory (one barrier a group) and evaluates its cells, with
// the phase field of the planes above and below in registers (indexed at
// compile time, so no register is moved before its load lands).  Only the
// tile's edge cells read an in-plane neighbour from global memory (L2).  The
// central gradient multiplies by the host-rounded 0.5/dx (within an ulp of
// diag_body.inc's (a-b)*0.5d0/dx, far inside the sums' tolerance).  Within
// a tile a thread sums its column's at most kDiagZ terms in plain FP64
// (every term is nonnegative: phi^2, c and the energy density, so the
// relative error stays below kDiagZ ulps) and adds the column sum to its
// compensated (Neumaier) totals.
constexpr int kDiagZ = 64;
constexpr int kDiagG = 4;   // planes a group
template <typename T>
__global__ void __launch_bounds__(256, 4) k_diag(DomainDesc d, const T* __restrict__ pn, const T* __restrict__ cn,
                                                 const T* __restrict__ tw, const T* __restrict__ dw,
                                                 double* __restrict__ part)
{
    KSum l2{0, 0}, sol{0, 0}, fe{0, 0};
    double mx = -DBL_MAX, mn = DBL_MAX, bad = 0.0;
    const int nx = d.nx, ny = d.ny, nz = d.nz;
    const long long px = d.px, pl = d.plane;
    const double dx = d.dx, dy = d.dy, dz = d.dz, w0 = d.W0, hx = d.hx, hy = d.hy, hz = d.hz;
    const double hE2 = __dmul_rn(__dmul_rn(0.5, d.E0), d.E0);
    __shared__ double sp[2][kDiagG][8][32];   // the group's phase planes, double-buffered by group parity
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    const int ntx = (nx + 31) >> 5, nty = (ny + 7) >> 3, ntz = (nz + kDiagZ - 1) / kDiagZ;
    const long long ntiles = (long long)ntx * nty * ntz;
    long long plk[kDiagG + 1];   // k planes, in elements
#pragma unroll
    for (int k = 0; k <= kDiagG; ++k) plk[k] = (long long)k * pl;
    int g = 0;   // group parity across the whole walk
    for (long long t = blockIdx.x; t < ntiles; t += gridDim.x) {
        const int bx = (int)(t % ntx);
        const long long r = t / ntx;
        const int by = (int)(r % nty), bz = (int)(r / nty);
        const int x = bx * 32 + tx, y = by * 8 + ty;
        const bool own = x < nx && y < ny;
        const bool xy_in = x > 0 && x < nx - 1 && y > 0 && y < ny - 1;
        const int z0 = bz * kDiagZ, z1 = min(z0 + kDiagZ, nz);
        const long long col = own ? (long long)x + (long long)y * px : 0;
        // phase field of this column at planes z-1 (pprev) and z (pcur) of the group's first plane z
        double pprev = (own && z0 > 0) ? (double)pn[col + (long long)(z0 - 1) * pl] : 0.0;
        double pcur = own ? (double)pn[col + (long long)z0 * pl] : 0.0;
        double s_l2 = 0.0, s_sol = 0.0, s_fe = 0.0;   // this column's sums over the chunk
        for (int zb = z0; zb < z1; zb += kDiagG, g ^= 1) {
            const int ng = min(kDiagG, z1 - zb);          // planes in this group (uniform)
            const long long ib = col + (long long)zb * pl;
            double pnx[kDiagG], cv[kDiagG], tv[kDiagG], dv[kDiagG];   // phi of plane zb+k+1; c, T, DPP of zb+k
#pragma unroll
            for (int k = 0; k < kDiagG; ++k) {
                const bool in = own && k < ng;
                pnx[k] = (in && zb + k + 1 < nz) ? (double)pn[ib + plk[k + 1]] : 0.0;
                cv[k] = in ? (double)cn[ib + plk[k]] : 0.0;
                tv[k] = (in && tw) ? (double)tw[ib + plk[k]] : 0.0;
                dv[k] = (in && dw) ? (double)dw[ib + plk[k]] : 0.0;
            }
#pragma unroll
            for (int k = 0; k < kDiagG; ++k) sp[g][k][ty][tx] = (k == 0) ? pcur : pnx[k - 1];
            __syncthreads();
#pragma unroll
            for (int k = 0; k < kDiagG; ++k) {
                if (k >= ng || !own) continue;
                const int z = zb + k;
                const double phi = (k == 0) ? pcur : pnx[k - 1];
                const double pm = (k == 0) ? pprev : ((k == 1) ? pcur : pnx[k - 2]);
                const double pp = pnx[k];
                s_l2 += phi * phi;
                mx = nan_max(mx, phi);
                mn = nan_min(mn, phi);
                s_sol += cv[k];
                bool fin = isfinite(phi) && isfinite(cv[k]);
                if (tw) fin = fin && isfinite(tv[k]);
                if (dw) fin = fin && isfinite(dv[k]);
                if (!fin) bad += 1.0;
                const double w_term = __dmul_rn(__dmul_rn(__dmul_rn(__dmul_rn(w0, phi), phi), 1.0 - phi), 1.0 - phi);
                double grad2 = 0.0;
                if (xy_in && z > 0 && z < nz - 1) {
                    const long long id = ib + plk[k];
                    const double xp = tx < 31 ? sp[g][k][ty][tx + 1] : (double)pn[id + 1];
                    const double xm = tx > 0 ? sp[g][k][ty][tx - 1] : (double)pn[id - 1];
                    const double yp = ty < 7 ? sp[g][k][ty + 1][tx] : (double)pn[id + px];
                    const double ym = ty > 0 ? sp[g][k][ty - 1][tx] : (double)pn[id - px];
                    const double gx = __dmul_rn(xp - xm, hx);
                    const double gy = __dmul_rn(yp - ym, hy);
                    const double gz = __dmul_rn(pp - pm, hz);
                    grad2 = __dadd_rn(__dadd_rn(__dmul_rn(gx, gx), __dmul_rn(gy, gy)), __dmul_rn(gz, gz));
                }
                const double e = __dadd_rn(__dmul_rn(hE2, grad2), w_term);
                s_fe += __dmul_rn(__dmul_rn(__dmul_rn(e, dx), dy), dz);
            }
            if (ng == kDiagG) {   // the next group's planes z-1 and z (a short group ends the chunk)
                pprev = pnx[kDiagG - 2];
                pcur = pnx[kDiagG - 1];
            }
        }
        l2.add(s_l2);
        sol.add(s_sol);
        fe.add(s_fe);
    }
    __shared__ double sh[8][9];
    double v[9] = {l2.s, l2.c, mx, mn, sol.s, sol.c, fe.s, fe.c, bad};
    // warp reduction (fixed order, deterministic for a fixed launch shape)
    for (int off = 16; off > 0; off >>= 1) {
        double o[9];
        for (int q = 0; q < 9; ++q) o[q] = __shfl_down_sync(0xffffffffu, v[q], off);
        KSum a{v[0], v[1]}; a.merge(o[0], o[1]); v[0] = a.s; v[1] = a.c;
        v[2] = nan_max(v[2], o[2]); v[3] = nan_min(v[3], o[3]);
        KSum b{v[4], v[5]}; b.merge(o[4], o[5]); v[4] = b.s; v[5] = b.c;
        KSum e{v[6], v[7]}; e.merge(o[6], o[7]); v[6] = e.s; v[7] = e.c;
        v[8] += o[8];
    }
    int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0)
        for (int q = 0; q < 9; ++q) sh[w][q] = v[q];
    __syncthreads();
    if (threadIdx.x == 0) {
        int nw = blockDim.x >> 5;
        for (int q = 0; q < 9; ++q) v[q] = sh[0][q];
        for (int ww = 1; ww < nw; ++ww) {
            KSum a{v[0], v[1]}; a.merge(sh[ww][0], sh[ww][1]); v[0] = a.s; v[1] = a.c;
            v[2] = nan_max(v[2], sh[ww][2]); v[3] = nan_min(v[3], sh[ww][3]);
            KSum b{v[4], v[5]}; b.merge(sh[ww][4], sh[ww][5]); v[4] = b.s; v[5] = b.c;
            KSum e{v[6], v[7]}; e.merge(sh[ww][6], sh[ww][7]); v[6] = e.s; v[7] = e.c;
            v[8] += sh[ww][8];
        }
        for (int q = 0; q < 9; ++q) part[(long long)blockIdx.x * kDiagRow + q] = v[q];
    }
}

// One warp merges the per-block partials: lane l takes blocks l, l + 32, ...,
// then the lanes merge in a fixed shuffle order (deterministic).
template <typename T>  // templated only so each precision unit owns its copy
__global__ void k_diag_final(const double* __restrict__ part, int nblk, double* __restrict__ out)
{
    if (blockIdx.x != 0 || threadIdx.x >= 32) return;
    KSum l2{0, 0}, sol{0, 0}, fe{0, 0};
    double mx = -DBL_MAX, mn = DBL_MAX, bad = 0.0;
    for (int b = (int)threadIdx.x; b < nblk; b += 32) {
        const double* p = part + (long long)b * kDiagRow;
        l2.merge(p[0], p[1]);
        mx = nan_max(mx, p[2]);
        mn = nan_min(mn, p[3]);
        sol.merge(p[4], p[5]);
        fe.merge(p[6], p[7]);
        bad += p[8];
    }
    double v[9] = {l2.s, l2.c, mx, mn, sol.s, sol.c, fe.s, fe.c, bad};
    for (int off = 16; off > 0; off >>= 1) {
        double o[9];
        for (int q = 0; q < 9; ++q) o[q] = __shfl_down_sync(0xffffffffu, v[q], off);
        KSum a{v[0], v[1]}; a.merge(o[0], o[1]); v[0] = a.s; v[1] = a.c;
        v[2] = nan_max(v[2], o[2]); v[3] = nan_min(v[3], o[3]);
        KSum b{v[4], v[5]}; b.merge(o[4], o[5]); v[4] = b.s; v[5] = b.c;
        KSum e{v[6], v[7]}; e.merge(o[6], o[7]); v[6] = e.s; v[7] = e.c;
        v[8] += o[8];
    }
    if (threadIdx.x == 0) {
        out[0] = sqrt(v[0] + v[1]);
        out[1] = v[2];
        out[2] = v[3];
        out[3] = v[4] + v[5];
        out[4] = v[6] + v[7];
        out[5] = v[8];   // cells with a non-finite phi, c, T or DPP (the watchdog)
    }
}

// ---- host conversion staging (FP32 contexts) ----
template <typename T>
__global__ void k_convert_in(DomainDesc d, const double* __restrict__ stage, T* __restrict__ dst, long long z0, long long nzc)
{
    long long n = (long long)d.nx * d.ny * nzc;
    for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
        int x = (int)(q % d.nx);
        long long r = q / d.nx;
        int y = (int)(r % d.ny);
        long long z = z0 + r / d.ny;
        dst[x + (long long)y * d.px + z * d.plane] = (T)stage[q];
    }
}

template <typename T>
__global__ void k_convert_out(DomainDesc d, const T* __restrict__ src, double* __restrict__ stage, long long z0, long long nzc)
{
    long long n = (long long)d.nx * d.ny * nzc;
    for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
        int x = (int)(q % d.nx);
        long long r = q / d.nx;
        int y = (int)(r % d.ny);
        long long z = z0 + r / d.ny;
        stage[q] = (double)src[x + (long long)y * d.px + z * d.plane];
    }
}

// ---- launchers ----
inline dim3 cell_grid(const DomainDesc& d) { return dim3((d.nx + 31) / 32, (d.ny + 7) / 8, d.nz); }

template <typename T>
cudaError_t launch_heat(const DomainDesc& d, const StepArgs& s, const Fields& f, cudaStream_t st)
{
    k_heat<T><<<cell_grid(d), dim3(32, 8), 0, st>>>(d, s, (const T*)f.T_old, (const T*)f.phi_old, (const T*)f.dpp,
                                                    (T*)f.T_new);
    return cudaGetLastError();
}

template <typename T>
cudaError_t launch_phase(const DomainDesc& d, const StepArgs& s, const void* phi_in, const void* c_in, void* phi_out,
                         void* dpp, cudaStream_t st)
{
    k_phase<T><<<cell_grid(d), dim3(32, 8), 0, st>>>(d, s, (const T*)phi_in, (const T*)c_in, (T*)phi_out, (T*)dpp);
    return cudaGetLastError();
}

template <typename T>
cudaError_t launch_solute(const DomainDesc& d, const StepArgs& s, const void* phi_in, const void* c_in, void* c_out,
                          cudaStream_t st)
{
    k_solute<T><<<cell_grid(d), dim3(32, 8), 0, st>>>(d, s, (const T*)phi_in, (const T*)c_in, (T*)c_out);
    return cudaGetLastError();
}

template <typename T>
cudaError_t launch_copy_inner(const DomainDesc& d, const void* src, void* dst, cudaStream_t st)
{
    k_copy_inner<T><<<cell_grid(d), dim3(32, 8), 0, st>>>(d, (const T*)src, (T*)dst);
    return cudaGetLastError();
}

template <typename T>
cudaError_t launch_diag(const DomainDesc& d, const void* phi, const void* c, const void* Tw, const void* dppw,
                        double* part, int nblk, double* out, cudaStream_t st)
{
    k_diag<T><<<nblk, 256, 0, st>>>(d, (const T*)phi, (const T*)c, (const T*)Tw, (const T*)dppw, part);
    k_diag_final<T><<<1, 32, 0, st>>>(part, nblk, out);
    return cudaGetLastError();
}

template <typename T>
cudaError_t launch_convert_in(const DomainDesc& d, const double* stage, void* dst, long long z0, long long nzc,
                              cudaStream_t st)
{
    k_convert_in<T><<<592, 256, 0, st>>>(d, stage, (T*)dst, z0, nzc);
    return cudaGetLastError();
}

template <typename T>
cudaError_t launch_convert_out(const DomainDesc& d, const void* src, double* stage, long long z0, long long nzc,
                               cudaStream_t st)
{
    k_convert_out<T><<<592, 256, 0, st>>>(d, (const T*)src, stage, z0, nzc);
    return cudaGetLastError();
}

}  // namespace pf3d
