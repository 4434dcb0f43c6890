// pf3d_fused.cuh -- fused z-marching kernels of the coupled step.
//
// One CTA owns a 32 x TY column tile and a z-chunk and marches along z.  It
// keeps rolling shared-memory windows:
//   sphi  : 6 planes of the input phase field with a 2-cell x/y halo
//           (planes z-2 .. z+3; plane z+4 is fetched with cp.async while
//           plane z is computed, so two planes are always in flight),
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
// Noise: every sweep of a step draws the same noise (same it), so the first
//   pass of a multi-sweep step stores the REAL(4) ran of every interior cell
//   in the DPP buffer after the heat equation has read that cell's DPP, and
//   the last pass reads it back before writing the new DPP (sweeps in between
//   leave DPP alone); a single-sweep pass draws it.
// Every output is written with the closed-form boundary decoration, so one
// pass replaces the reference's copy + stencil + plane-copy kernels.  The
// per-cell arithmetic is the fast form of pf3d_device.cuh (FAST = true).
//
// Latency hiding: the window slots advance incrementally (no modulo), the
// centre values the cell update reads from global memory (c, DPP, T) and the
// concentration values of the next solute plane are loaded one plane ahead
// into registers.
#pragma once
#include "pf3d_launch.h"
#include "pf3d_cpasync.cuh"

namespace pf3d {


template <typename T, int TY>
struct FusedSmem {
    static constexpr int TX = 32;
    static constexpr int PW = TX + 4, PH = TY + 4;   // phase tile with halo 2
    static constexpr int NW = TX + 2, NH = TY + 2;   // node tile with ring 1
    static constexpr int NS = 6;                     // phase planes z-2 .. z+3
    T phi[NS][PH][PW];
    T eps[3][NH][NW], exy[3][NH][NW], eyz[3][NH][NW], ezx[3][NH][NW];
    T br[3][NH][NW], mu[3][NH][NW];
};

// resident CTAs per SM the register budget is sized for.  K = 1: a pass that
// draws the smooth noise (ruido_tipo 2) inline; its trilinear blend of eight
// hashes needs about 128 registers a thread in FP64, which caps it at 16
// warps.  K = 0: every other pass fits 80 registers without spills, so 24
// warps.  FP32 runs 24 warps in both.
template <typename T, int TY, int K>
struct FusedOcc {
    static constexpr int warps = (sizeof(T) == 8) ? (K == 1 ? 16 : 24) : 24;
    static constexpr int v = (warps / TY) > 0 ? (warps / TY) : 1;
};

__device__ __forceinline__ int add6(int a, int k) { int t = a + k; return t >= 6 ? t - 6 : t; }
__device__ __forceinline__ int add3(int a, int k) { int t = a + k; return t >= 3 ? t - 3 : t; }

// One cell of a boundary tile or plane, shared by the one-cell and the
// paired kernels: the heat update (TNEW <- TOLD outside 2..N-1), the phase
// sweep with the closed-form decoration of equacao_campo_fase.f90:151-167
// (the source cell writes its value to all its preimages) and the solute
// update with the face copies of concentracao_soluto.f90:116-124.  phase(),
// heat() and solute() evaluate the cell's arithmetic; [xl, xh] and [yl, yh]
// are the cell's x and y preimage ranges (fpre_range).
template <typename T, bool HEAT, bool DPPW, bool SOL, typename PhaseF, typename HeatF, typename SolF>
__device__ __forceinline__ void boundary_cell(int x, int y, int z, int nx, int ny, int nz, long long px, long long pl,
                                              long long id, T PPc, T cpp, T told, int xl, int xh, int yl, int yh,
                                              T* __restrict__ phi_out, T* __restrict__ dpp, T* __restrict__ c_out,
                                              T* __restrict__ T_new, PhaseF phase, HeatF heat, SolF solute)
{
    const bool xs_src = x >= 1 && x <= nx - 2, ys_src = y >= 1 && y <= ny - 2;
    const bool xs_int = x >= 2 && x <= nx - 3, ys_int = y >= 2 && y <= ny - 3;
    const bool single_xy = x >= 3 && x <= nx - 4 && y >= 3 && y <= ny - 4;
    const bool zin = z >= 1 && z <= nz - 2;

    // ---- temperatura ----
    if (HEAT) T_new[id] = (xs_src && ys_src && zin) ? heat() : told;

    // ---- phase sweep ----
    if (xs_src && ys_src && zin) {
        T U;
        if (xs_int && ys_int && z >= 2 && z <= nz - 3) {
            const T ppn = phase();
            if (DPPW) dpp[id] = ppn - PPc;
            U = clamp01(ppn);
        } else {
            U = PPc;
        }
        if (single_xy && z >= 3 && z <= nz - 4) {
            phi_out[id] = U;   // its only preimage is itself
        } else {
            int zl, zh;
            fpre_range(z, nz, &zl, &zh);
            for (int zz = zl; zz <= zh; ++zz)
                for (int yy = yl; yy <= yh; ++yy)
                    for (int xx = xl; xx <= xh; ++xx)
                        phi_out[(long long)xx + (long long)yy * px + (long long)zz * pl] = U;
        }
    }

    // ---- solute ----
    if (SOL) {
        const bool inner = xs_src && ys_src && zin;
        const bool feeds = inner || z == 1 || z == nz - 2 || (zin && (x == 1 || x == nx - 2));
        if (feeds) {
            T Uc;
            if (inner) {
                Uc = solute();
                c_out[id] = Uc;
            } else {
                Uc = cpp;
            }
            if (z == 1) c_out[id - pl] = Uc;
            if (z == nz - 2) c_out[id + pl] = Uc;
            if (zin && x == 1) c_out[id - 1] = Uc;
            if (zin && x == nx - 2) c_out[id + 1] = Uc;
            if (zin && xs_src && y == 1) c_out[id - px] = Uc;
            if (zin && xs_src && y == ny - 2) c_out[id + px] = Uc;
        }
    }
}

// One 32 x TY x zchunk tile (tile coordinates bx, by, bz) of one domain.
// Ends with a CTA-wide barrier, so the caller may reuse the shared memory.
template <typename T, int TY, bool HEAT, bool DPPW, bool SOL, bool SMOOTH>
__device__ __forceinline__ void fused_tile(const DomainDesc& d, const KC<T>& c, const T* __restrict__ phi_in,
                                           const T* __restrict__ c_in, T* __restrict__ phi_out,
                                           T* __restrict__ dpp, T* __restrict__ c_out,
                                           const T* __restrict__ T_old, T* __restrict__ T_new, int zchunk, int bx,
                                           int by, int bz, unsigned char* smem_raw)
{
    using SM = FusedSmem<T, TY>;
    constexpr int TX = SM::TX, PW = SM::PW, PH = SM::PH, NW = SM::NW, NH = SM::NH;
    constexpr int RING = 2 * NW + 2 * TY;   // ring nodes around the tile
    // noise hand-over: first pass of a multi-sweep step stores, last reads
    constexpr int ran_mode = (HEAT && !DPPW) ? 1 : ((!HEAT && DPPW) ? 2 : 0);
    SM& sm = *reinterpret_cast<SM*>(smem_raw);

    const int nx = d.nx, ny = d.ny, nz = d.nz;
    const long long px = d.px, pl = d.plane;
    const int x0 = bx * TX, y0 = by * TY;
    const int zb = bz * zchunk;
    const int ze = min(zb + zchunk, nz);
    const int tx = threadIdx.x, ty = threadIdx.y;
    const int tid = tx + TX * ty;
    const int x = x0 + tx, y = y0 + ty;
    const bool own = (x < nx) && (y < ny);

    // node-tile position of ring item r: the rows above and below the tile,
    // then the two side columns
    int rlx = 0, rly = 0;
    if (tid < RING) {
        int r = tid;
        if (r < NW) { rlx = r; rly = 0; }
        else if ((r -= NW) < NW) { rlx = r; rly = NH - 1; }
        else if ((r -= NW) < TY) { rlx = 0; rly = 1 + r; }
        else { r -= TY; rlx = NW - 1; rly = 1 + r; }
    }
    // global position of this thread's two node-tile items and whether they
    // are phase nodes (1 .. N-2) / solute points (0 .. N-1)
    const int rgx = x0 - 1 + rlx, rgy = y0 - 1 + rly;       // ring item
    const bool ring = tid < RING;
    const bool in_node = x >= 1 && x <= nx - 2 && y >= 1 && y <= ny - 2;
    const bool rg_node = ring && rgx >= 1 && rgx <= nx - 2 && rgy >= 1 && rgy <= ny - 2;
    const bool in_pt = own;
    const bool rg_pt = ring && rgx >= 0 && rgx <= nx - 1 && rgy >= 0 && rgy <= ny - 1;
    const long long col = (long long)x + (long long)y * px;
    const long long rg_col = (long long)rgx + (long long)rgy * px;

    // issue the loads of phase plane z into window slot sl
    auto load_plane = [&](int z, int sl) {
        if (z < 0 || z >= nz) return;
        T(*dst)[PW] = sm.phi[sl];
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

    // anisotropy quantities of node plane zn from phase slots (zn-1, zn, zn+1)
    auto node_plane = [&](int zn, int sm1, int s0, int sp1, int sl) {
        if (zn < 1 || zn > nz - 2) return;
        const T(*pm)[PW] = sm.phi[sm1];
        const T(*p0)[PW] = sm.phi[s0];
        const T(*pp)[PW] = sm.phi[sp1];
        auto one_node = [&](int lx, int ly) {
            const int fx = lx + 1, fy = ly + 1;   // phase-tile coordinates of the node
            T gxv = grad<T, true>(p0[fy][fx + 1], p0[fy][fx - 1], c.dx, c.hx);
            T gyv = grad<T, true>(p0[fy + 1][fx], p0[fy - 1][fx], c.dy, c.hy);
            T gzv = grad<T, true>(pp[fy][fx], pm[fy][fx], c.dz, c.hz);
            Node<T> n = aniso_node<T, true>(gxv, gyv, gzv, c);
            sm.eps[sl][ly][lx] = n.eps;
            sm.exy[sl][ly][lx] = n.exy;
            sm.eyz[sl][ly][lx] = n.eyz;
            sm.ezx[sl][ly][lx] = n.ezx;
        };
        if (in_node) one_node(tx + 1, ty + 1);
        if (rg_node) one_node(rlx, rly);
    };

    // solute point quantities of plane zs from phase slot s0 and the
    // concentration values ci (own point) and cr (ring point) of that plane
    auto sol_plane = [&](int zs, int s0, int sl, T ci, T cr) {
        if (zs < 0 || zs > nz - 1) return;
        const T(*p0)[PW] = sm.phi[s0];
        if (in_pt) {
            SolNode<T> n = sol_node<T, true>(p0[ty + 2][tx + 2], ci, c);
            sm.br[sl][ty + 1][tx + 1] = n.br;
            sm.mu[sl][ty + 1][tx + 1] = n.mu;
        }
        if (rg_pt) {
            SolNode<T> n = sol_node<T, true>(p0[rly + 1][rlx + 1], cr, c);
            sm.br[sl][rly][rlx] = n.br;
            sm.mu[sl][rly][rlx] = n.mu;
        }
    };
    auto load_c = [&](int zs, T& ci, T& cr) {
        if (!SOL || zs < 0 || zs > nz - 1) return;
        const long long zo = (long long)zs * pl;
        if (in_pt) ci = c_in[col + zo];
        if (rg_pt) cr = c_in[rg_col + zo];
    };

    // ---- prologue: planes zb-2 .. zb+2, nodes zb-1 and zb ----
    int s5 = zb % 6, s3 = zb % 3;   // window slots of plane zb
    for (int k = -2; k <= 3; ++k) load_plane(zb + k, add6(s5, (k + 6) % 6));
    cp_async_commit();
    T cpi = 0, cpr = 0, cqi = 0, cqr = 0;   // c of solute planes z+1 (p) and z+2 (q)
    if (SOL) {
        T ai = 0, ar = 0, bi = 0, br_ = 0;
        load_c(zb - 1, ai, ar);
        load_c(zb, bi, br_);
        load_c(zb + 1, cpi, cpr);
        cp_async_wait_all();
        __syncthreads();
        sol_plane(zb - 1, add6(s5, 5), add3(s3, 2), ai, ar);
        sol_plane(zb, s5, s3, bi, br_);
    } else {
        cp_async_wait_all();
        __syncthreads();
    }
    node_plane(zb - 1, add6(s5, 4), add6(s5, 5), s5, add3(s3, 2));
    node_plane(zb, add6(s5, 5), s5, add6(s5, 1), s3);

    const int fx = tx + 2, fy = ty + 2;   // own cell in the phase tile
    const int nlx = tx + 1, nly = ty + 1; // own cell in the node tile
    const bool xs_src = x >= 1 && x <= nx - 2, ys_src = y >= 1 && y <= ny - 2;
    // CTA-uniform: every column of the tile is in [3, N-4] in x and y
    const bool tile_int = x0 >= 3 && x0 + TX + 3 <= nx && y0 >= 3 && y0 + TY + 3 <= ny;
    int xl = 0, xh = -1, yl = 0, yh = -1;
    if (own && xs_src) fpre_range(x, nx, &xl, &xh);
    if (own && ys_src) fpre_range(y, ny, &yl, &yh);
    long long zoff = (long long)zb * pl;
    // noise hash input of the own cell, carried along z (k = z + 1)
    uint64_t hin = hash_base(x + 1, y + 1, c.it, 1) + (uint64_t)(zb + 1) * kHashK;

    // centre values of the own cell, one plane ahead
    T ncpp = 0, ndpp = 0, ntold = 0;
    if (own && zb < ze) {
        const long long id0 = col + zoff;
        ncpp = c_in[id0];
        if (HEAT) {
            ndpp = dpp[id0];
            ntold = T_old[id0];
        } else if (ran_mode == 2) {
            ndpp = dpp[id0];
        }
    }
    for (int z = zb; z < ze; ++z, zoff += pl, hin += kHashK) {
        const long long id = col + zoff;
        const T cpp = ncpp, dppv = ndpp, told = ntold;
        if (own && z + 1 < ze) {
            ncpp = c_in[id + pl];
            if (HEAT) {
                ndpp = dpp[id + pl];
                ntold = T_old[id + pl];
            } else if (ran_mode == 2) {
                ndpp = dpp[id + pl];
            }
        }
        if (SOL) load_c(z + 2, cqi, cqr);
        node_plane(z + 1, s5, add6(s5, 1), add6(s5, 2), add3(s3, 1));
        if (SOL) sol_plane(z + 1, add6(s5, 1), add3(s3, 1), cpi, cpr);
        __syncthreads();
        load_plane(z + 4, add6(s5, 4));
        cp_async_commit();

        const T(*pm)[PW] = sm.phi[add6(s5, 5)];
        const T(*p0)[PW] = sm.phi[s5];
        const T(*pp)[PW] = sm.phi[add6(s5, 1)];
        const int n0 = s3, np1 = add3(s3, 1), nm1 = add3(s3, 2);

        // phase_body.inc at the own cell: PPNEW
        auto phase_cell = [&](T PPc, T cpp, int z) -> T {
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
            Node<T> E, W, N, S, Tt, B;
            E.eps = sm.eps[n0][nly][nlx + 1]; E.exy = sm.exy[n0][nly][nlx + 1]; E.ezx = sm.ezx[n0][nly][nlx + 1];
            W.eps = sm.eps[n0][nly][nlx - 1]; W.exy = sm.exy[n0][nly][nlx - 1]; W.ezx = sm.ezx[n0][nly][nlx - 1];
            N.eps = sm.eps[n0][nly + 1][nlx]; N.exy = sm.exy[n0][nly + 1][nlx]; N.eyz = sm.eyz[n0][nly + 1][nlx];
            S.eps = sm.eps[n0][nly - 1][nlx]; S.exy = sm.exy[n0][nly - 1][nlx]; S.eyz = sm.eyz[n0][nly - 1][nlx];
            Tt.eps = sm.eps[np1][nly][nlx]; Tt.eyz = sm.eyz[np1][nly][nlx]; Tt.ezx = sm.ezx[np1][nly][nlx];
            B.eps = sm.eps[nm1][nly][nlx]; B.eyz = sm.eyz[nm1][nly][nlx]; B.ezx = sm.ezx[nm1][nly][nlx];
            E.eyz = W.eyz = N.ezx = S.ezx = Tt.exy = B.exy = (T)0;   // unused by the body
            float ran;
            if constexpr (ran_mode == 2) {
                ran = (float)dppv;   // drawn and stored by the first pass
            } else {
                if constexpr (SMOOTH)
                    ran = (c.rt == 2) ? phase_ran(2, x + 1, y + 1, z + 1, c.it)
                                      : __double2float_rn(ran64(hash63_mix(hin)));
                else
                    ran = __double2float_rn(ran64(hash63_mix(hin)));
                if constexpr (ran_mode == 1) dpp[id] = (T)ran;
            }
            return phase_ppnew<T, true>(nb, E, W, N, S, Tt, B, cpp, ran, c);
        };
        // conc_body.inc at the own cell
        auto solute_cell = [&](T PPc, T cpp) -> T {
            SolNode<T> nP{sm.br[n0][nly][nlx], sm.mu[n0][nly][nlx]};
            SolNode<T> nE{sm.br[n0][nly][nlx + 1], sm.mu[n0][nly][nlx + 1]};
            SolNode<T> nW{sm.br[n0][nly][nlx - 1], sm.mu[n0][nly][nlx - 1]};
            SolNode<T> nN{sm.br[n0][nly + 1][nlx], sm.mu[n0][nly + 1][nlx]};
            SolNode<T> nS{sm.br[n0][nly - 1][nlx], sm.mu[n0][nly - 1][nlx]};
            SolNode<T> nT{sm.br[np1][nly][nlx], sm.mu[np1][nly][nlx]};
            SolNode<T> nB{sm.br[nm1][nly][nlx], sm.mu[nm1][nly][nlx]};
            return conc_new<T, true>(PPc, cpp, nP, nE, nW, nN, nS, nT, nB, c);
        };
        auto heat_cell = [&](T PPc, T dppv) -> T {
            T TE = 0, TW = 0, TN = 0, TS = 0, TT = 0, TB = 0;
            if (c.lap) {
                TE = T_old[id + 1]; TW = T_old[id - 1]; TN = T_old[id + px]; TS = T_old[id - px];
                TT = T_old[id + pl]; TB = T_old[id - pl];
            }
            return heat_new<T>(PPc, dppv, TE, TW, TN, TS, TT, TB, c);
        };

        if (tile_int && z >= 3 && z <= nz - 4) {
            // the whole tile plane is interior and every cell is its own only
            // preimage: no bounds, decoration or scatter (CTA-uniform branch)
            const T PPc = p0[fy][fx];
            if (HEAT) T_new[id] = heat_cell(PPc, dppv);
            const T ppn = phase_cell(PPc, cpp, z);
            if (DPPW) dpp[id] = ppn - PPc;
            phi_out[id] = clamp01(ppn);
            if (SOL) c_out[id] = solute_cell(PPc, cpp);
        } else if (own) {
            const T PPc = p0[fy][fx];
            boundary_cell<T, HEAT, DPPW, SOL>(
                x, y, z, nx, ny, nz, px, pl, id, PPc, cpp, told, xl, xh, yl, yh, phi_out, dpp, c_out, T_new,
                [&]() { return phase_cell(PPc, cpp, z); }, [&]() { return heat_cell(PPc, dppv); },
                [&]() { return solute_cell(PPc, cpp); });
        }
        if (SOL) { cpi = cqi; cpr = cqr; }
        cp_async_wait_prev();   // plane z+3 (needed next) has landed; z+4 may be in flight
        __syncthreads();
        s5 = add6(s5, 1);
        s3 = add3(s3, 1);
    }
    cp_async_wait_all();
    __syncthreads();
}

// single domain: one CTA per tile.  SMOOTH: the kernel may draw the smooth
// noise (compiled only where the pass draws noise and the deck asks for it).
template <typename T, int TY, bool HEAT, bool DPPW, bool SOL, bool SMOOTH>
__global__ void __launch_bounds__(32 * TY, (FusedOcc<T, TY, SMOOTH ? 1 : 0>::v))
    k_fused(DomainDesc d, const KC<T> c, const T* __restrict__ phi_in, const T* __restrict__ c_in,
            T* __restrict__ phi_out, T* __restrict__ dpp, T* __restrict__ c_out, const T* __restrict__ T_old,
            T* __restrict__ T_new, int zchunk)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    fused_tile<T, TY, HEAT, DPPW, SOL, SMOOTH>(d, c, phi_in, c_in, phi_out, dpp, c_out, T_old, T_new, zchunk,
                                               blockIdx.x, blockIdx.y, blockIdx.z, smem_raw);
}

// many domains: a persistent grid walks the work list.  PASS 0 is the first
// pass of a step (temperatura + sweep 1, or the whole step with one sweep),
// PASS 1 the last (sweep 2 + solute).  SMOOTH: some domain of the batch
// draws the smooth noise (the first pass then selects per domain).
template <typename T, int TY, int PASS, bool ONE_SWEEP, bool SMOOTH>
__global__ void __launch_bounds__(32 * TY, (FusedOcc<T, TY, SMOOTH ? 1 : 0>::v))
    k_fused_batch(const BatchDomain* __restrict__ doms, const BatchStep* __restrict__ steps,
                  const BatchItem* __restrict__ items, const int* __restrict__ n_items, int zchunk)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ __align__(16) KC<T> skc;   // the loop constants of the current item
    const int n = *n_items;
    const int tid = threadIdx.x + 32 * threadIdx.y;
    for (int w = blockIdx.x; w < n; w += gridDim.x) {
        const BatchItem it = items[w];
        const BatchStep& st = steps[it.dom];
        if (!st.active) continue;   // uniform across the CTA
        const BatchDomain& D = doms[it.dom];
        const int q = st.q_phi, qc = st.q_c, qt = st.q_T;
        static_assert(sizeof(KC<T>) % 4 == 0, "KC is copied as words");
        if (tid < (int)(sizeof(KC<T>) / 4))
            reinterpret_cast<int*>(&skc)[tid] = reinterpret_cast<const int*>(st.kc)[tid];
        __syncthreads();
        const KC<T>& kc = skc;
        if (PASS == 0) {
            if (ONE_SWEEP)
                fused_tile<T, TY, true, true, true, SMOOTH>(D.d, kc, (const T*)D.phi[q], (const T*)D.c[qc], (T*)D.phi[1 - q],
                                                    (T*)D.dpp, (T*)D.c[1 - qc], (const T*)D.T[qt], (T*)D.T[1 - qt],
                                                    zchunk, it.bx, it.by, it.bz, smem_raw);
            else
                fused_tile<T, TY, true, false, false, SMOOTH>(D.d, kc, (const T*)D.phi[q], (const T*)D.c[qc],
                                                      (T*)D.phi[1 - q], (T*)D.dpp, nullptr, (const T*)D.T[qt],
                                                      (T*)D.T[1 - qt], zchunk, it.bx, it.by, it.bz, smem_raw);
        } else {
            fused_tile<T, TY, false, true, true, false>(D.d, kc, (const T*)D.phi[1 - q], (const T*)D.c[qc], (T*)D.phi[q],
                                                 (T*)D.dpp, (T*)D.c[1 - qc], nullptr, nullptr, zchunk, it.bx, it.by,
                                                 it.bz, smem_raw);
        }
    }
}

template <typename T, int TY>
constexpr size_t fused_smem_bytes()
{
    return sizeof(FusedSmem<T, TY>);
}

template <typename T, int TY, bool HEAT, bool DPPW, bool SOL, bool SMOOTH>
cudaError_t launch_fused_t(const DomainDesc& d, const StepArgs& s, const void* phi_in, const void* c_in,
                           void* phi_out, void* dpp, void* c_out, const void* T_old, void* T_new, int zchunk,
                           cudaStream_t st)
{
    auto kern = k_fused<T, TY, HEAT, DPPW, SOL, SMOOTH>;
    const size_t smem = fused_smem_bytes<T, TY>();
    static bool configured = false;   // one attribute call per instantiation
    if (!configured) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        configured = true;
    }
    if (zchunk <= 0) zchunk = d.nz;
    KC<T> kc;
    kc.load(d, s);
    dim3 grid((d.nx + 31) / 32, (d.ny + TY - 1) / TY, (d.nz + zchunk - 1) / zchunk);
    kern<<<grid, dim3(32, TY), smem, st>>>(d, kc, (const T*)phi_in, (const T*)c_in, (T*)phi_out, (T*)dpp, (T*)c_out,
                                           (const T*)T_old, (T*)T_new, zchunk);
    return cudaGetLastError();
}

template <typename T, bool HEAT, bool DPPW, bool SOL, bool SMOOTH>
cudaError_t launch_fused_ty(const DomainDesc& d, const StepArgs& s, const void* phi_in, const void* c_in,
                            void* phi_out, void* dpp, void* c_out, const void* T_old, void* T_new, int tile_y,
                            int zchunk, cudaStream_t st)
{
#define PF3D_TY_CASE(TYV) \
    launch_fused_t<T, TYV, HEAT, DPPW, SOL, SMOOTH>(d, s, phi_in, c_in, phi_out, dpp, c_out, T_old, T_new, zchunk, st)
    switch (tile_y) {
    case 4: return PF3D_TY_CASE(4);
    case 16: return PF3D_TY_CASE(16);
    default: return PF3D_TY_CASE(8);
    }
#undef PF3D_TY_CASE
}

// first pass of a step: temperatura + sweep 1 (phi_old -> phi_mid); with a
// single sweep it also writes DPP and does the solute step into c_new.
template <typename T>
cudaError_t launch_fused_first(const DomainDesc& d, const StepArgs& s, const Fields& f, bool with_solute, int tile_y,
                               int zchunk, cudaStream_t st)
{
    const bool smooth = d.rt == 2;
    if (with_solute)
        return smooth ? launch_fused_ty<T, true, true, true, true>(d, s, f.phi_old, f.c_old, f.phi_mid, f.dpp, f.c_new,
                                                                   f.T_old, f.T_new, tile_y, zchunk, st)
                      : launch_fused_ty<T, true, true, true, false>(d, s, f.phi_old, f.c_old, f.phi_mid, f.dpp,
                                                                    f.c_new, f.T_old, f.T_new, tile_y, zchunk, st);
    return smooth ? launch_fused_ty<T, true, false, false, true>(d, s, f.phi_old, f.c_old, f.phi_mid, f.dpp, nullptr,
                                                                 f.T_old, f.T_new, tile_y, zchunk, st)
                  : launch_fused_ty<T, true, false, false, false>(d, s, f.phi_old, f.c_old, f.phi_mid, f.dpp, nullptr,
                                                                  f.T_old, f.T_new, tile_y, zchunk, st);
}

// last pass: final sweep (phi_mid -> phi_new) with DPP + solute from phi_mid.
template <typename T>
cudaError_t launch_fused_last(const DomainDesc& d, const StepArgs& s, const Fields& f, int tile_y, int zchunk,
                              cudaStream_t st)
{
    return launch_fused_ty<T, false, true, true, false>(d, s, f.phi_mid, f.c_old, f.phi_new, f.dpp, f.c_new, nullptr,
                                                        nullptr, tile_y, zchunk, st);
}

// The persistent grid is the SM count times the CTAs of this kernel that are
// resident on one SM (each pass has its own register budget).
template <typename T, int TY, int PASS, bool ONE_SWEEP, bool SMOOTH>
cudaError_t launch_batch_t(const BatchDomain* doms, const BatchStep* steps, const BatchItem* items, const int* n_items,
                           int zchunk, int n_sm, cudaStream_t st)
{
    auto kern = k_fused_batch<T, TY, PASS, ONE_SWEEP, SMOOTH>;
    const size_t smem = fused_smem_bytes<T, TY>();
    static int per_sm = 0;   // one attribute and occupancy query per instantiation
    if (per_sm == 0) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        int nb = 0;
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, kern, 32 * TY, smem);
        if (e != cudaSuccess) return e;
        per_sm = nb > 0 ? nb : 1;
    }
    kern<<<n_sm * per_sm, dim3(32, TY), smem, st>>>(doms, steps, items, n_items, zchunk);
    return cudaGetLastError();
}

template <typename T>
cudaError_t launch_fused_batch(const BatchDomain* doms, const BatchStep* steps, const BatchItem* items,
                               const int* n_items, int pass, bool one_sweep, bool smooth, int tile_y, int zchunk,
                               int n_sm, cudaStream_t st)
{
#define PF3D_BATCH_ARGS doms, steps, items, n_items, zchunk, n_sm, st
#define PF3D_BATCH_CASE(TYV)                                                                          \
    if (tile_y == TYV) {                                                                              \
        if (pass == 0) {                                                                              \
            if (one_sweep)                                                                            \
                return smooth ? launch_batch_t<T, TYV, 0, true, true>(PF3D_BATCH_ARGS)                \
                              : launch_batch_t<T, TYV, 0, true, false>(PF3D_BATCH_ARGS);              \
            return smooth ? launch_batch_t<T, TYV, 0, false, true>(PF3D_BATCH_ARGS)                   \
                          : launch_batch_t<T, TYV, 0, false, false>(PF3D_BATCH_ARGS);                 \
        }                                                                                             \
        return launch_batch_t<T, TYV, 1, false, false>(PF3D_BATCH_ARGS);                              \
    }
    PF3D_BATCH_CASE(4)
    PF3D_BATCH_CASE(16)
    PF3D_BATCH_CASE(8)
#undef PF3D_BATCH_CASE
#undef PF3D_BATCH_ARGS
    return cudaErrorInvalidValue;
}

}  // namespace pf3d
