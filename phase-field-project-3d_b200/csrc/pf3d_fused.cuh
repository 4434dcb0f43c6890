// pf3d_fused.cuh -- fused z-marching kernels of the coupled step.
//
// One CTA owns a 32 x TY column tile and a z-chunk and marches along z.  It
// keeps rolling shared-memory windows:
//   sphi  : 5 planes of the input phase field with a 2-cell x/y halo
//           (planes z-2 .. z+2, the next one prefetched with cp.async),
//   snode : 3 planes (z-1, z, z+1) of the anisotropy quantities eps, exy,
//           eyz, ezx at every node of the tile plus a 1-cell ring
//           (phase_body.inc:51-129); each is computed once and read by the
//           six cells around it,
//   ssol  : 3 planes of the per-point solute quantities (Gamma bracket and
//           mu = log(CL/(1-CL)), conc_body.inc:42-144), also computed once.
// A node's value depends only on the phase field around the node, so sharing
// it is bit-identical to the reference's per-cell recomputation.
//
// Template switches select which reference subroutines one pass performs:
//   HEAT : temperatura (TNEW from TOLD, DPP and the centre phase value)
//   DPPW : write DPP (only the last sweep of a step needs to)
//   SOL  : concentracao_soluto from the same input phase field
// Every output is written with the closed-form boundary decoration, so one
// pass replaces the reference's copy + stencil + plane-copy kernels.  The
// per-cell arithmetic is the fast form of pf3d_device.cuh (FAST = true).
#pragma once
#include "pf3d_launch.h"

namespace pf3d {

__device__ __forceinline__ void cp_async_elem(void* smem, const void* gmem, int bytes)
{
    unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    if (bytes == 8)
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem));
    else
        asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(gmem));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

template <typename T, int TY>
struct FusedSmem {
    static constexpr int TX = 32;
    static constexpr int PW = TX + 4, PH = TY + 4;   // phase tile with halo 2
    static constexpr int NW = TX + 2, NH = TY + 2;   // node tile with ring 1
    T phi[5][PH][PW];
    T eps[3][NH][NW], exy[3][NH][NW], eyz[3][NH][NW], ezx[3][NH][NW];
    T br[3][NH][NW], mu[3][NH][NW];
};

template <typename T, int TY, bool HEAT, bool DPPW, bool SOL>
__global__ void __launch_bounds__(32 * TY, (TY <= 8) ? 2 : 1) k_fused(DomainDesc d, StepArgs s, const T* __restrict__ phi_in,
                                                   const T* __restrict__ c_in, T* __restrict__ phi_out,
                                                   T* __restrict__ dpp, T* __restrict__ c_out,
                                                   const T* __restrict__ T_old, T* __restrict__ T_new, int zchunk)
{
    using SM = FusedSmem<T, TY>;
    constexpr int TX = SM::TX, PW = SM::PW, PH = SM::PH, NW = SM::NW, NH = SM::NH;
    constexpr int NT = TX * TY;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    SM& sm = *reinterpret_cast<SM*>(smem_raw);

    const int nx = d.nx, ny = d.ny, nz = d.nz;
    const long long px = d.px, pl = d.plane;
    const int x0 = blockIdx.x * TX, y0 = blockIdx.y * TY;
    const int zb = blockIdx.z * zchunk;
    const int ze = min(zb + zchunk, nz);
    const int tid = threadIdx.x + TX * threadIdx.y;
    const int tx = threadIdx.x, ty = threadIdx.y;
    const int x = x0 + tx, y = y0 + ty;
    const bool own = (x < nx) && (y < ny);

    KC<T> c;
    c.load(d, s);

    auto slot5 = [](int z) { return ((z % 5) + 5) % 5; };
    auto slot3 = [](int z) { return ((z % 3) + 3) % 3; };

    // issue the loads of phase plane z (in-domain elements only)
    auto load_plane = [&](int z) {
        if (z < 0 || z >= nz) return;
        T(*dst)[PW] = sm.phi[slot5(z)];
        const T* src = phi_in + (long long)z * pl;
        for (int ly = ty; ly < PH; ly += TY) {
            const int gy = y0 - 2 + ly;
            if (gy < 0 || gy >= ny) continue;
            const T* row = src + (long long)gy * px;
            int gx = x0 - 2 + tx;
            if (gx >= 0 && gx < nx) cp_async_elem(&dst[ly][tx], row + gx, (int)sizeof(T));
            if (tx < 4) {
                gx = x0 + 30 + tx;
                if (gx < nx) cp_async_elem(&dst[ly][32 + tx], row + gx, (int)sizeof(T));
            }
        }
    };

    // node-tile position of the ring item r (0 <= r < RING): the two full
    // rows above and below the tile, then the two side columns
    constexpr int RING = 2 * NW + 2 * TY;
    auto ring_pos = [](int r, int& lx, int& ly) {
        if (r < NW) { lx = r; ly = 0; return; }
        r -= NW;
        if (r < NW) { lx = r; ly = NH - 1; return; }
        r -= NW;
        if (r < TY) { lx = 0; ly = 1 + r; return; }
        r -= TY;
        lx = NW - 1; ly = 1 + r;
    };

    // anisotropy quantities of node plane zn over the tile + ring
    auto node_plane = [&](int zn) {
        if (zn < 1 || zn > nz - 2) return;
        const T(*pm)[PW] = sm.phi[slot5(zn - 1)];
        const T(*p0)[PW] = sm.phi[slot5(zn)];
        const T(*pp)[PW] = sm.phi[slot5(zn + 1)];
        const int sl = slot3(zn);
        auto one_node = [&](int lx, int ly) {
            int gx = x0 - 1 + lx, gy = y0 - 1 + ly;
            if (gx < 1 || gx > nx - 2 || gy < 1 || gy > ny - 2) return;
            int fx = lx + 1, fy = ly + 1;   // phase-tile coordinates of the node
            T gxv = grad<T, true>(p0[fy][fx + 1], p0[fy][fx - 1], c.dx, c.hx);
            T gyv = grad<T, true>(p0[fy + 1][fx], p0[fy - 1][fx], c.dy, c.hy);
            T gzv = grad<T, true>(pp[fy][fx], pm[fy][fx], c.dz, c.hz);
            Node<T> n = aniso_node<T, true>(gxv, gyv, gzv, c);
            sm.eps[sl][ly][lx] = n.eps;
            sm.exy[sl][ly][lx] = n.exy;
            sm.eyz[sl][ly][lx] = n.eyz;
            sm.ezx[sl][ly][lx] = n.ezx;
        };
        one_node(tx + 1, ty + 1);
        if (tid < RING) {
            int lx, ly;
            ring_pos(tid, lx, ly);
            one_node(lx, ly);
        }
    };

    // solute point quantities of plane zs over the tile + ring
    auto sol_plane = [&](int zs) {
        if (!SOL) return;
        if (zs < 0 || zs > nz - 1) return;
        const T(*p0)[PW] = sm.phi[slot5(zs)];
        const int sl = slot3(zs);
        const T* cz = c_in + (long long)zs * pl;
        auto one_point = [&](int lx, int ly) {
            int gx = x0 - 1 + lx, gy = y0 - 1 + ly;
            if (gx < 0 || gx > nx - 1 || gy < 0 || gy > ny - 1) return;
            SolNode<T> n = sol_node<T, true>(p0[ly + 1][lx + 1], cz[gx + (long long)gy * px], c);
            sm.br[sl][ly][lx] = n.br;
            sm.mu[sl][ly][lx] = n.mu;
        };
        one_point(tx + 1, ty + 1);
        if (tid < RING) {
            int lx, ly;
            ring_pos(tid, lx, ly);
            one_point(lx, ly);
        }
    };

    // ---- prologue: planes zb-2 .. zb+2, nodes zb-1 and zb ----
    for (int z = zb - 2; z <= zb + 2; ++z) load_plane(z);
    cp_async_commit();
    cp_async_wait_all();
    __syncthreads();
    node_plane(zb - 1);
    node_plane(zb);
    sol_plane(zb - 1);
    sol_plane(zb);

    const int fx = tx + 2, fy = ty + 2;   // own cell in the phase tile
    const int nlx = tx + 1, nly = ty + 1; // own cell in the node tile
    const bool xs_src = x >= 1 && x <= nx - 2, ys_src = y >= 1 && y <= ny - 2;
    const bool xs_int = x >= 2 && x <= nx - 3, ys_int = y >= 2 && y <= ny - 3;
    int xl = 0, xh = -1, yl = 0, yh = -1;
    if (own && xs_src) fpre_range(x, nx, &xl, &xh);
    if (own && ys_src) fpre_range(y, ny, &yl, &yh);

    for (int z = zb; z < ze; ++z) {
        node_plane(z + 1);
        sol_plane(z + 1);
        __syncthreads();
        load_plane(z + 3);
        cp_async_commit();

        if (own) {
            const long long id = (long long)x + (long long)y * px + (long long)z * pl;
            const T(*pm)[PW] = sm.phi[slot5(z - 1)];
            const T(*p0)[PW] = sm.phi[slot5(z)];
            const T(*pp)[PW] = sm.phi[slot5(z + 1)];
            const T PPc = p0[fy][fx];
            const bool zin = z >= 1 && z <= nz - 2;

            // ---- temperatura ----
            if (HEAT) {
                if (xs_src && ys_src && zin) {
                    T TE = 0, TW = 0, TN = 0, TS = 0, TT = 0, TB = 0;
                    if (c.lap) {
                        TE = T_old[id + 1]; TW = T_old[id - 1]; TN = T_old[id + px]; TS = T_old[id - px];
                        TT = T_old[id + pl]; TB = T_old[id - pl];
                    }
                    T_new[id] = heat_new<T>(PPc, dpp[id], TE, TW, TN, TS, TT, TB, c);
                } else {
                    T_new[id] = T_old[id];
                }
            }

            // ---- phase sweep ----
            const bool src = xs_src && ys_src && zin;
            if (src) {
                T U;
                const bool interior = xs_int && ys_int && z >= 2 && z <= nz - 3;
                if (interior) {
                    Nbr<T> nb;
                    nb.PP = PPc;
                    nb.PN = p0[fy + 1][fx]; nb.PS = p0[fy - 1][fx];
                    nb.PE = p0[fy][fx + 1]; nb.PW = p0[fy][fx - 1];
                    nb.PT = pp[fy][fx]; nb.PB = pm[fy][fx];
                    nb.PNE = p0[fy + 1][fx + 1]; nb.PSE = p0[fy - 1][fx + 1];
                    nb.PNW = p0[fy + 1][fx - 1]; nb.PSW = p0[fy - 1][fx - 1];
                    nb.PNT = pp[fy + 1][fx]; nb.PNB = pm[fy + 1][fx];
                    nb.PST = pp[fy - 1][fx]; nb.PSB = pm[fy - 1][fx];
                    nb.PET = pp[fy][fx + 1]; nb.PEB = pm[fy][fx + 1];
                    nb.PWT = pp[fy][fx - 1]; nb.PWB = pm[fy][fx - 1];
                    const int s0 = slot3(z), sp = slot3(z + 1), sm1 = slot3(z - 1);
                    Node<T> E, W, N, S, Tt, B;
                    E.eps = sm.eps[s0][nly][nlx + 1]; E.exy = sm.exy[s0][nly][nlx + 1]; E.ezx = sm.ezx[s0][nly][nlx + 1];
                    W.eps = sm.eps[s0][nly][nlx - 1]; W.exy = sm.exy[s0][nly][nlx - 1]; W.ezx = sm.ezx[s0][nly][nlx - 1];
                    N.eps = sm.eps[s0][nly + 1][nlx]; N.exy = sm.exy[s0][nly + 1][nlx]; N.eyz = sm.eyz[s0][nly + 1][nlx];
                    S.eps = sm.eps[s0][nly - 1][nlx]; S.exy = sm.exy[s0][nly - 1][nlx]; S.eyz = sm.eyz[s0][nly - 1][nlx];
                    Tt.eps = sm.eps[sp][nly][nlx]; Tt.eyz = sm.eyz[sp][nly][nlx]; Tt.ezx = sm.ezx[sp][nly][nlx];
                    B.eps = sm.eps[sm1][nly][nlx]; B.eyz = sm.eyz[sm1][nly][nlx]; B.ezx = sm.ezx[sm1][nly][nlx];
                    E.eyz = W.eyz = N.ezx = S.ezx = Tt.exy = B.exy = (T)0;   // unused by the body
                    float ran = phase_ran(c.rt, x + 1, y + 1, z + 1, c.it);
                    T ppn = phase_ppnew<T, true>(nb, E, W, N, S, Tt, B, c_in[id], ran, c);
                    if (DPPW) dpp[id] = ppn - PPc;
                    U = clamp01(ppn);
                } else {
                    U = PPc;
                }
                int zl, zh;
                fpre_range(z, nz, &zl, &zh);
                for (int zz = zl; zz <= zh; ++zz)
                    for (int yy = yl; yy <= yh; ++yy)
                        for (int xx = xl; xx <= xh; ++xx)
                            phi_out[(long long)xx + (long long)yy * px + (long long)zz * pl] = U;
            }

            // ---- solute ----
            if (SOL) {
                const bool xin = xs_src, yin = ys_src;
                const bool inner = xin && yin && zin;
                const bool feeds = inner || z == 1 || z == nz - 2 || (zin && (x == 1 || x == nx - 2));
                if (feeds) {
                    T Uc;
                    if (inner) {
                        const int s0 = slot3(z), sp = slot3(z + 1), sm1 = slot3(z - 1);
                        SolNode<T> nP{sm.br[s0][nly][nlx], sm.mu[s0][nly][nlx]};
                        SolNode<T> nE{sm.br[s0][nly][nlx + 1], sm.mu[s0][nly][nlx + 1]};
                        SolNode<T> nW{sm.br[s0][nly][nlx - 1], sm.mu[s0][nly][nlx - 1]};
                        SolNode<T> nN{sm.br[s0][nly + 1][nlx], sm.mu[s0][nly + 1][nlx]};
                        SolNode<T> nS{sm.br[s0][nly - 1][nlx], sm.mu[s0][nly - 1][nlx]};
                        SolNode<T> nT{sm.br[sp][nly][nlx], sm.mu[sp][nly][nlx]};
                        SolNode<T> nB{sm.br[sm1][nly][nlx], sm.mu[sm1][nly][nlx]};
                        Uc = conc_new<T, true>(PPc, c_in[id], nP, nE, nW, nN, nS, nT, nB, c);
                        c_out[id] = Uc;
                    } else {
                        Uc = c_in[id];
                    }
                    if (z == 1) c_out[id - pl] = Uc;
                    if (z == nz - 2) c_out[id + pl] = Uc;
                    if (zin && x == 1) c_out[id - 1] = Uc;
                    if (zin && x == nx - 2) c_out[id + 1] = Uc;
                    if (zin && xin && y == 1) c_out[id - px] = Uc;
                    if (zin && xin && y == ny - 2) c_out[id + px] = Uc;
                }
            }
        }
        cp_async_wait_all();
        __syncthreads();
    }
}

template <typename T, int TY>
constexpr size_t fused_smem_bytes()
{
    return sizeof(FusedSmem<T, TY>);
}

template <typename T, int TY, bool HEAT, bool DPPW, bool SOL>
cudaError_t launch_fused_t(const DomainDesc& d, const StepArgs& s, const void* phi_in, const void* c_in,
                           void* phi_out, void* dpp, void* c_out, const void* T_old, void* T_new, int zchunk,
                           cudaStream_t st)
{
    auto kern = k_fused<T, TY, HEAT, DPPW, SOL>;
    const size_t smem = fused_smem_bytes<T, TY>();
    static bool configured = false;   // one attribute call per instantiation
    if (!configured) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        configured = true;
    }
    if (zchunk <= 0) zchunk = d.nz;
    dim3 grid((d.nx + 31) / 32, (d.ny + TY - 1) / TY, (d.nz + zchunk - 1) / zchunk);
    kern<<<grid, dim3(32, TY), smem, st>>>(d, s, (const T*)phi_in, (const T*)c_in, (T*)phi_out, (T*)dpp, (T*)c_out,
                                           (const T*)T_old, (T*)T_new, zchunk);
    return cudaGetLastError();
}

template <typename T, bool HEAT, bool DPPW, bool SOL>
cudaError_t launch_fused_ty(const DomainDesc& d, const StepArgs& s, const void* phi_in, const void* c_in,
                            void* phi_out, void* dpp, void* c_out, const void* T_old, void* T_new, int tile_y,
                            int zchunk, cudaStream_t st)
{
    switch (tile_y) {
    case 4: return launch_fused_t<T, 4, HEAT, DPPW, SOL>(d, s, phi_in, c_in, phi_out, dpp, c_out, T_old, T_new, zchunk, st);
    case 16: return launch_fused_t<T, 16, HEAT, DPPW, SOL>(d, s, phi_in, c_in, phi_out, dpp, c_out, T_old, T_new, zchunk, st);
    default: return launch_fused_t<T, 8, HEAT, DPPW, SOL>(d, s, phi_in, c_in, phi_out, dpp, c_out, T_old, T_new, zchunk, st);
    }
}

// first pass of a step: temperatura + sweep 1 (phi_old -> phi_mid); with a
// single sweep it also writes DPP and does the solute step into c_new.
template <typename T>
cudaError_t launch_fused_first(const DomainDesc& d, const StepArgs& s, const Fields& f, bool with_solute, int tile_y,
                               int zchunk, cudaStream_t st)
{
    if (with_solute)
        return launch_fused_ty<T, true, true, true>(d, s, f.phi_old, f.c_old, f.phi_mid, f.dpp, f.c_new, f.T_old,
                                                    f.T_new, tile_y, zchunk, st);
    return launch_fused_ty<T, true, false, false>(d, s, f.phi_old, f.c_old, f.phi_mid, f.dpp, nullptr, f.T_old, f.T_new,
                                                  tile_y, zchunk, st);
}

// last pass: final sweep (phi_mid -> phi_new) with DPP + solute from phi_mid.
template <typename T>
cudaError_t launch_fused_last(const DomainDesc& d, const StepArgs& s, const Fields& f, int tile_y, int zchunk,
                              cudaStream_t st)
{
    return launch_fused_ty<T, false, true, true>(d, s, f.phi_mid, f.c_old, f.phi_new, f.dpp, f.c_new, nullptr, nullptr,
                                                 tile_y, zchunk, st);
}

}  // namespace pf3d
