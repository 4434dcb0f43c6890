// pf3d_fused_pair.cuh -- the fused z-marching passes with two cells per
// thread.
//
// Same tile, windows and arithmetic as fused_tile (pf3d_fused.cuh), but a
// 32 x TY tile is marched by 32 x TY/2 threads: thread (tx, ty) owns the
// cells of rows ty and ty + TY/2.  In the interior fast path both cells go
// through the per-cell arithmetic together as a lane pair (pf3d_pair.cuh):
// two independent chains, with the explicit multiply-adds packed (f32x2) in
// FP32.  The
// per-plane work that does not depend on the cell -- window slots, barrier,
// prefetch issue, loop-invariant constants, branches -- is paid once for the
// two cells.  The ring of anisotropy nodes and solute points around the tile
// is paired the same way (top row with bottom row, left column with right
// column).  Boundary tiles and planes run the scalar per-cell code of
// fused_tile once per lane.  Every cell gets the bits it gets from
// fused_tile.  Used for 32 x 8 tiles on decks without the smooth noise and
// without heat diffusion (D = 0, the reference's case); other decks keep the
// one-cell kernels.  Measured on B200 (512 x 512 x 1024, both passes): FP32
// 11.04 -> 10.26 ms per step; FP64 16.0 -> 18.0 ms (a paired FP64 tile has
// the shared memory of a one-cell tile and half its warps, and the FP64
// chains need the warps to hide their latency), so FP64 keeps one cell per
// thread by default.
#pragma once
#include <cstddef>
#include "pf3d_fused.cuh"

namespace pf3d {

// resident CTAs (of TY/2 warps) per SM the register budget is sized for:
// FP64 3 (shared memory allows no more); FP32 5 for the first pass and 4
// for the last (measured best on 512 x 512 x 1024)
template <typename S, bool HEAT>
struct PairOcc {
    static constexpr int v = (sizeof(S) == 8) ? 3 : (HEAT ? 5 : 4);
};

// KC<V> with every scalar constant broadcast to both lanes (host side)
template <typename S>
KC<typename PairOf<S>::type> kc_pair(const KC<S>& k)
{
    using V = typename PairOf<S>::type;
    KC<V> r;
    constexpr int n = (int)(offsetof(KC<S>, hq) / sizeof(S));
    static_assert(offsetof(KC<V>, hq) == n * sizeof(V), "KC layout");
    const S* src = reinterpret_cast<const S*>(&k);
    V* dst = reinterpret_cast<V*>(&r);
    for (int i = 0; i < n; ++i) dst[i] = V::splat(src[i]);
    r.hq = k.hq;
    r.rt = k.rt;
    r.it = k.it;
    r.lap = k.lap;
    return r;
}

template <typename S, int TY, bool HEAT, bool DPPW, bool SOL>
__device__ __forceinline__ void fused_tile_pair(const DomainDesc& d, const KC<S>& c,
                                                const KC<typename PairOf<S>::type>& cv,
                                                const S* __restrict__ phi_in, const S* __restrict__ c_in,
                                                S* __restrict__ phi_out, S* __restrict__ dpp, S* __restrict__ c_out,
                                                const S* __restrict__ T_old, S* __restrict__ T_new, int zchunk,
                                                int bx, int by, int bz, unsigned char* smem_raw)
{
    using V = typename PairOf<S>::type;
    using SM = FusedSmem<S, TY>;
    constexpr int TX = SM::TX, PW = SM::PW, PH = SM::PH, NW = SM::NW, NH = SM::NH;
    constexpr int TYH = TY / 2;                 // thread rows; lane l owns row ty + l*TYH
    constexpr int RPAIRS = NW + TY;             // ring pairs: top/bottom rows, left/right columns
    constexpr int ran_mode = (HEAT && !DPPW) ? 1 : ((!HEAT && DPPW) ? 2 : 0);
    static_assert(TY % 2 == 0, "paired tiles need an even height");
    (void)T_old;   // D = 0 decks only: the heat update reads no neighbour
    SM& sm = *reinterpret_cast<SM*>(smem_raw);

    const int nx = d.nx, ny = d.ny, nz = d.nz;
    const long long px = d.px, pl = d.plane;
    const int x0 = bx * TX, y0 = by * TY;
    const int zb = bz * zchunk;
    const int ze = min(zb + zchunk, nz);
    const int tx = threadIdx.x, ty = threadIdx.y;
    const int tid = tx + TX * ty;
    const int x = x0 + tx;
    int yv[2];
    yv[0] = y0 + ty;
    yv[1] = y0 + ty + TYH;
    bool own[2];
    own[0] = (x < nx) && (yv[0] < ny);
    own[1] = (x < nx) && (yv[1] < ny);

    // ring pair of this thread: (rlx, rly[0]) and (rlx2, rly[1])
    int rlx[2] = {0, 0}, rly[2] = {0, 0};
    const bool rpair = tid < RPAIRS;
    if (rpair) {
        if (tid < NW) {
            rlx[0] = rlx[1] = tid;
            rly[0] = 0;
            rly[1] = NH - 1;
        } else {
            const int r = tid - NW;
            rlx[0] = 0;
            rlx[1] = NW - 1;
            rly[0] = rly[1] = 1 + r;
        }
    }
    bool rg_node[2], rg_pt[2], in_node[2];
    long long rg_col[2], col[2];
    for (int l = 0; l < 2; ++l) {
        const int gx = x0 - 1 + rlx[l], gy = y0 - 1 + rly[l];
        rg_node[l] = rpair && gx >= 1 && gx <= nx - 2 && gy >= 1 && gy <= ny - 2;
        rg_pt[l] = rpair && gx >= 0 && gx <= nx - 1 && gy >= 0 && gy <= ny - 1;
        rg_col[l] = (long long)gx + (long long)gy * px;
        in_node[l] = x >= 1 && x <= nx - 2 && yv[l] >= 1 && yv[l] <= ny - 2;
        col[l] = (long long)x + (long long)yv[l] * px;
    }

    auto load_plane = [&](int z, int sl) {
        if (z < 0 || z >= nz) return;
        S(*dst)[PW] = sm.phi[sl];
        const S* src = phi_in + (long long)z * pl;
        for (int ly = ty; ly < PH; ly += TYH) {
            const int gy = y0 - 2 + ly;
            if (gy < 0 || gy >= ny) continue;
            const S* row = src + (long long)gy * px;
            int gx = x0 - 2 + tx;
            if (gx >= 0 && gx < nx) cp_async_elem(&dst[ly][tx], row + gx, (int)sizeof(S));
            if (tx < 4) {
                gx = x0 + 30 + tx;
                if (gx < nx) cp_async_elem(&dst[ly][32 + tx], row + gx, (int)sizeof(S));
            }
        }
    };

    // anisotropy of a pair of nodes (node-tile coordinates) of plane zn
    auto node_pair = [&](const S (*pm)[PW], const S (*p0)[PW], const S (*pp)[PW], int sl, const int* lx,
                         const int* ly, const bool* ok) {
        const int fx0 = lx[0] + 1, fy0 = ly[0] + 1, fx1 = lx[1] + 1, fy1 = ly[1] + 1;
        const V gx = grad<V, true>(V(p0[fy0][fx0 + 1], p0[fy1][fx1 + 1]), V(p0[fy0][fx0 - 1], p0[fy1][fx1 - 1]),
                                   cv.dx, cv.hx);
        const V gy = grad<V, true>(V(p0[fy0 + 1][fx0], p0[fy1 + 1][fx1]), V(p0[fy0 - 1][fx0], p0[fy1 - 1][fx1]),
                                   cv.dy, cv.hy);
        const V gz = grad<V, true>(V(pp[fy0][fx0], pp[fy1][fx1]), V(pm[fy0][fx0], pm[fy1][fx1]), cv.dz, cv.hz);
        const Node<V> n = aniso_node<V, true>(gx, gy, gz, cv);
        if (ok[0]) {
            sm.eps[sl][ly[0]][lx[0]] = n.eps.x();
            sm.exy[sl][ly[0]][lx[0]] = n.exy.x();
            sm.eyz[sl][ly[0]][lx[0]] = n.eyz.x();
            sm.ezx[sl][ly[0]][lx[0]] = n.ezx.x();
        }
        if (ok[1]) {
            sm.eps[sl][ly[1]][lx[1]] = n.eps.y();
            sm.exy[sl][ly[1]][lx[1]] = n.exy.y();
            sm.eyz[sl][ly[1]][lx[1]] = n.eyz.y();
            sm.ezx[sl][ly[1]][lx[1]] = n.ezx.y();
        }
    };
    auto node_plane = [&](int zn, int sm1, int s0, int sp1, int sl) {
        if (zn < 1 || zn > nz - 2) return;
        const int olx[2] = {tx + 1, tx + 1}, oly[2] = {ty + 1, ty + 1 + TYH};
        if (in_node[0] || in_node[1]) node_pair(sm.phi[sm1], sm.phi[s0], sm.phi[sp1], sl, olx, oly, in_node);
        if (rg_node[0] || rg_node[1]) node_pair(sm.phi[sm1], sm.phi[s0], sm.phi[sp1], sl, rlx, rly, rg_node);
    };

    // solute point quantities of a pair of points of plane zs
    auto sol_pair = [&](const S (*p0)[PW], int sl, const int* lx, const int* ly, const bool* ok, S c0, S c1) {
        const SolNode<V> n = sol_node<V, true>(V(p0[ly[0] + 1][lx[0] + 1], p0[ly[1] + 1][lx[1] + 1]), V(c0, c1), cv);
        if (ok[0]) {
            sm.br[sl][ly[0]][lx[0]] = n.br.x();
            sm.mu[sl][ly[0]][lx[0]] = n.mu.x();
        }
        if (ok[1]) {
            sm.br[sl][ly[1]][lx[1]] = n.br.y();
            sm.mu[sl][ly[1]][lx[1]] = n.mu.y();
        }
    };
    auto sol_plane = [&](int zs, int s0, int sl, const S* ci, const S* cr) {
        if (zs < 0 || zs > nz - 1) return;
        const int olx[2] = {tx + 1, tx + 1}, oly[2] = {ty + 1, ty + 1 + TYH};
        if (own[0] || own[1]) sol_pair(sm.phi[s0], sl, olx, oly, own, ci[0], ci[1]);
        if (rg_pt[0] || rg_pt[1]) sol_pair(sm.phi[s0], sl, rlx, rly, rg_pt, cr[0], cr[1]);
    };
    auto load_c = [&](int zs, S* ci, S* cr) {
        if (!SOL || zs < 0 || zs > nz - 1) return;
        const long long zo = (long long)zs * pl;
        for (int l = 0; l < 2; ++l) {
            if (own[l]) ci[l] = c_in[col[l] + zo];
            if (rg_pt[l]) cr[l] = c_in[rg_col[l] + zo];
        }
    };

    // ---- prologue: planes zb-2 .. zb+3, nodes zb-1 and zb ----
    int s5 = zb % 6, s3 = zb % 3;
    for (int k = -2; k <= 3; ++k) load_plane(zb + k, add6(s5, (k + 6) % 6));
    cp_async_commit();
    S cpi[2] = {0, 0}, cpr[2] = {0, 0}, cqi[2] = {0, 0}, cqr[2] = {0, 0};
    if (SOL) {
        S ai[2] = {0, 0}, ar[2] = {0, 0}, bi[2] = {0, 0}, br_[2] = {0, 0};
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

    const int fx = tx + 2, nlx = tx + 1;
    const int fyv[2] = {ty + 2, ty + 2 + TYH}, nlyv[2] = {ty + 1, ty + 1 + TYH};
    const bool xs_src = x >= 1 && x <= nx - 2;
    const bool tile_int = x0 >= 3 && x0 + TX + 3 <= nx && y0 >= 3 && y0 + TY + 3 <= ny;
    int xl = 0, xh = -1;
    if ((own[0] || own[1]) && xs_src) fpre_range(x, nx, &xl, &xh);
    long long zoff = (long long)zb * pl;
    uint64_t hin[2];
    hin[0] = hash_base(x + 1, yv[0] + 1, c.it, 1) + (uint64_t)(zb + 1) * kHashK;
    hin[1] = hash_base(x + 1, yv[1] + 1, c.it, 1) + (uint64_t)(zb + 1) * kHashK;

    S ncpp[2] = {0, 0}, ndpp[2] = {0, 0}, ntold[2] = {0, 0};
    for (int l = 0; l < 2; ++l)
        if (own[l] && zb < ze) {
            const long long id0 = col[l] + zoff;
            ncpp[l] = c_in[id0];
            if (HEAT) {
                ndpp[l] = dpp[id0];
                ntold[l] = T_old[id0];
            } else if (ran_mode == 2) {
                ndpp[l] = dpp[id0];
            }
        }
    for (int z = zb; z < ze; ++z, zoff += pl, hin[0] += kHashK, hin[1] += kHashK) {
        S cpp[2], dppv[2], told[2];
        for (int l = 0; l < 2; ++l) {
            cpp[l] = ncpp[l];
            dppv[l] = ndpp[l];
            told[l] = ntold[l];
            if (own[l] && z + 1 < ze) {
                const long long idn = col[l] + zoff + pl;
                ncpp[l] = c_in[idn];
                if (HEAT) {
                    ndpp[l] = dpp[idn];
                    ntold[l] = T_old[idn];
                } else if (ran_mode == 2) {
                    ndpp[l] = dpp[idn];
                }
            }
        }
        if (SOL) load_c(z + 2, cqi, cqr);
        node_plane(z + 1, s5, add6(s5, 1), add6(s5, 2), add3(s3, 1));
        if (SOL) sol_plane(z + 1, add6(s5, 1), add3(s3, 1), cpi, cpr);
        __syncthreads();
        load_plane(z + 4, add6(s5, 4));
        cp_async_commit();

        const S(*pm)[PW] = sm.phi[add6(s5, 5)];
        const S(*p0)[PW] = sm.phi[s5];
        const S(*pp)[PW] = sm.phi[add6(s5, 1)];
        const int n0 = s3, np1 = add3(s3, 1), nm1 = add3(s3, 2);

        // the REAL(4) noise of lane l at plane z
        auto ran_of = [&](int l) -> float {
            if constexpr (ran_mode == 2) return (float)dppv[l];
            return __double2float_rn(ran64(hash63_mix(hin[l])));
        };
        // node quantities of the six neighbours, lane l
        auto nodes = [&](int l, Node<S>& E, Node<S>& W, Node<S>& N, Node<S>& So, Node<S>& Tt, Node<S>& B) {
            const int nly = nlyv[l];
            E.eps = sm.eps[n0][nly][nlx + 1]; E.exy = sm.exy[n0][nly][nlx + 1]; E.ezx = sm.ezx[n0][nly][nlx + 1];
            W.eps = sm.eps[n0][nly][nlx - 1]; W.exy = sm.exy[n0][nly][nlx - 1]; W.ezx = sm.ezx[n0][nly][nlx - 1];
            N.eps = sm.eps[n0][nly + 1][nlx]; N.exy = sm.exy[n0][nly + 1][nlx]; N.eyz = sm.eyz[n0][nly + 1][nlx];
            So.eps = sm.eps[n0][nly - 1][nlx]; So.exy = sm.exy[n0][nly - 1][nlx]; So.eyz = sm.eyz[n0][nly - 1][nlx];
            Tt.eps = sm.eps[np1][nly][nlx]; Tt.eyz = sm.eyz[np1][nly][nlx]; Tt.ezx = sm.ezx[np1][nly][nlx];
            B.eps = sm.eps[nm1][nly][nlx]; B.eyz = sm.eyz[nm1][nly][nlx]; B.ezx = sm.ezx[nm1][nly][nlx];
            E.eyz = W.eyz = N.ezx = So.ezx = Tt.exy = B.exy = (S)0;   // unused by the body
        };
        auto nbr = [&](int l, Nbr<S>& nb) {
            const int fy = fyv[l];
            nb.PP = p0[fy][fx];
            nb.PN = p0[fy + 1][fx]; nb.PS = p0[fy - 1][fx];
            nb.PE = p0[fy][fx + 1]; nb.PW = p0[fy][fx - 1];
            nb.PT = pp[fy][fx]; nb.PB = pm[fy][fx];
            nb.PNE = p0[fy + 1][fx + 1]; nb.PSE = p0[fy - 1][fx + 1];
            nb.PNW = p0[fy + 1][fx - 1]; nb.PSW = p0[fy - 1][fx - 1];
            nb.PNT = pp[fy + 1][fx]; nb.PNB = pm[fy + 1][fx];
            nb.PST = pp[fy - 1][fx]; nb.PSB = pm[fy - 1][fx];
            nb.PET = pp[fy][fx + 1]; nb.PEB = pm[fy][fx + 1];
            nb.PWT = pp[fy][fx - 1]; nb.PWB = pm[fy][fx - 1];
        };
        auto solnodes = [&](int l, SolNode<S>* q) {   // P, E, W, N, S, T, B
            const int nly = nlyv[l];
            q[0] = {sm.br[n0][nly][nlx], sm.mu[n0][nly][nlx]};
            q[1] = {sm.br[n0][nly][nlx + 1], sm.mu[n0][nly][nlx + 1]};
            q[2] = {sm.br[n0][nly][nlx - 1], sm.mu[n0][nly][nlx - 1]};
            q[3] = {sm.br[n0][nly + 1][nlx], sm.mu[n0][nly + 1][nlx]};
            q[4] = {sm.br[n0][nly - 1][nlx], sm.mu[n0][nly - 1][nlx]};
            q[5] = {sm.br[np1][nly][nlx], sm.mu[np1][nly][nlx]};
            q[6] = {sm.br[nm1][nly][nlx], sm.mu[nm1][nly][nlx]};
        };
        // scalar per-cell arithmetic of fused_tile for lane l
        auto phase_cell_s = [&](int l, long long id) -> S {
            Nbr<S> nb;
            nbr(l, nb);
            Node<S> E, W, N, So, Tt, B;
            nodes(l, E, W, N, So, Tt, B);
            const float ran = ran_of(l);
            if constexpr (ran_mode == 1) dpp[id] = (S)ran;
            return phase_ppnew<S, true>(nb, E, W, N, So, Tt, B, cpp[l], ran, c);
        };
        // the paired kernels run only on decks with D = 0 (no heat diffusion):
        // TNEW = TP + the latent term, from the centre cell alone
        auto heat_cell_s = [&](int l, long long id, S PPc) -> S {
            (void)id;
            const S z0 = (S)0;
            return heat_new<S, false>(PPc, dppv[l], z0, z0, z0, z0, z0, z0, c);
        };
        auto solute_cell_s = [&](int l, S PPc) -> S {
            SolNode<S> q[7];
            solnodes(l, q);
            return conc_new<S, true>(PPc, cpp[l], q[0], q[1], q[2], q[3], q[4], q[5], q[6], c);
        };

        if (tile_int && z >= 3 && z <= nz - 4) {
            // interior fast path, both lanes together (CTA-uniform branch)
            const long long id0 = col[0] + zoff, id1 = col[1] + zoff;
            Nbr<S> a, b;
            nbr(0, a);
            nbr(1, b);
            Nbr<V> nb;
            nb.PP = V(a.PP, b.PP); nb.PN = V(a.PN, b.PN); nb.PS = V(a.PS, b.PS); nb.PE = V(a.PE, b.PE);
            nb.PW = V(a.PW, b.PW); nb.PT = V(a.PT, b.PT); nb.PB = V(a.PB, b.PB);
            nb.PNE = V(a.PNE, b.PNE); nb.PSE = V(a.PSE, b.PSE); nb.PNW = V(a.PNW, b.PNW); nb.PSW = V(a.PSW, b.PSW);
            nb.PNT = V(a.PNT, b.PNT); nb.PNB = V(a.PNB, b.PNB); nb.PST = V(a.PST, b.PST); nb.PSB = V(a.PSB, b.PSB);
            nb.PET = V(a.PET, b.PET); nb.PEB = V(a.PEB, b.PEB); nb.PWT = V(a.PWT, b.PWT); nb.PWB = V(a.PWB, b.PWB);
            Node<S> e0, w0, n0_, s0_, t0, b0, e1, w1, n1_, s1_, t1, b1;
            nodes(0, e0, w0, n0_, s0_, t0, b0);
            nodes(1, e1, w1, n1_, s1_, t1, b1);
            auto pn = [](const Node<S>& p, const Node<S>& q) {
                Node<V> r;
                r.eps = V(p.eps, q.eps); r.exy = V(p.exy, q.exy); r.eyz = V(p.eyz, q.eyz); r.ezx = V(p.ezx, q.ezx);
                return r;
            };
            const Node<V> E = pn(e0, e1), W = pn(w0, w1), N = pn(n0_, n1_), So = pn(s0_, s1_), Tt = pn(t0, t1),
                          B = pn(b0, b1);
            const float r0 = ran_of(0), r1 = ran_of(1);
            if constexpr (ran_mode == 1) {
                dpp[id0] = (S)r0;
                dpp[id1] = (S)r1;
            }
            const V PPc = nb.PP;
            const V cppv = V(cpp[0], cpp[1]);
            if (HEAT) {
                // pointwise unless D > 0; per lane keeps the neighbour loads short-lived
                T_new[id0] = heat_cell_s(0, id0, a.PP);
                T_new[id1] = heat_cell_s(1, id1, b.PP);
            }
            const V ppn = phase_ppnew<V, true>(nb, E, W, N, So, Tt, B, cppv, V((S)r0, (S)r1), cv);
            if (DPPW) {
                const V dv = ppn - PPc;
                dpp[id0] = dv.x();
                dpp[id1] = dv.y();
            }
            const V u = clamp01(ppn);
            phi_out[id0] = u.x();
            phi_out[id1] = u.y();
            if (SOL) {
                SolNode<S> qa[7], qb[7];
                solnodes(0, qa);
                solnodes(1, qb);
                SolNode<V> q[7];
                for (int i = 0; i < 7; ++i) q[i] = {V(qa[i].br, qb[i].br), V(qa[i].mu, qb[i].mu)};
                const V cn = conc_new<V, true>(PPc, cppv, q[0], q[1], q[2], q[3], q[4], q[5], q[6], cv);
                c_out[id0] = cn.x();
                c_out[id1] = cn.y();
            }
        } else {
            // boundary tiles and planes: fused_tile's scalar path, lane by lane
            for (int l = 0; l < 2; ++l) {
                if (!own[l]) continue;
                const int y = yv[l];
                const long long id = col[l] + zoff;
                const S PPc = p0[fyv[l]][fx];
                int yl_ = 0, yh_ = -1;
                if (y >= 1 && y <= ny - 2) fpre_range(y, ny, &yl_, &yh_);
                boundary_cell<S, HEAT, DPPW, SOL>(
                    x, y, z, nx, ny, nz, px, pl, id, PPc, cpp[l], told[l], xl, xh, yl_, yh_, phi_out, dpp, c_out,
                    T_new, [&]() { return phase_cell_s(l, id); }, [&]() { return heat_cell_s(l, id, PPc); },
                    [&]() { return solute_cell_s(l, PPc); });
            }
        }
        if (SOL) {
            cpi[0] = cqi[0]; cpi[1] = cqi[1];
            cpr[0] = cqr[0]; cpr[1] = cqr[1];
        }
        cp_async_wait_prev();   // plane z+3 (needed next) has landed; z+4 may be in flight
        __syncthreads();
        s5 = add6(s5, 1);
        s3 = add3(s3, 1);
    }
    cp_async_wait_all();
    __syncthreads();
}

template <typename S, int TY, bool HEAT, bool DPPW, bool SOL>
__global__ void __launch_bounds__(16 * TY, (PairOcc<S, HEAT>::v))
    k_fused_pair(DomainDesc d, const KC<S> c, const KC<typename PairOf<S>::type> cv, const S* __restrict__ phi_in,
                 const S* __restrict__ c_in, S* __restrict__ phi_out, S* __restrict__ dpp, S* __restrict__ c_out,
                 const S* __restrict__ T_old, S* __restrict__ T_new, int zchunk)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    fused_tile_pair<S, TY, HEAT, DPPW, SOL>(d, c, cv, phi_in, c_in, phi_out, dpp, c_out, T_old, T_new, zchunk,
                                            blockIdx.x, blockIdx.y, blockIdx.z, smem_raw);
}

template <typename S, int TY, bool HEAT, bool DPPW, bool SOL>
cudaError_t launch_fused_pair_t(const DomainDesc& d, const StepArgs& s, const void* phi_in, const void* c_in,
                                void* phi_out, void* dpp, void* c_out, const void* T_old, void* T_new, int zchunk,
                                cudaStream_t st)
{
    auto kern = k_fused_pair<S, TY, HEAT, DPPW, SOL>;
    const size_t smem = fused_smem_bytes<S, TY>();
    static bool configured = false;
    if (!configured) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        configured = true;
    }
    if (zchunk <= 0) zchunk = d.nz;
    KC<S> kc;
    kc.load(d, s);
    const auto kv = kc_pair<S>(kc);
    dim3 grid((d.nx + 31) / 32, (d.ny + TY - 1) / TY, (d.nz + zchunk - 1) / zchunk);
    kern<<<grid, dim3(32, TY / 2), smem, st>>>(d, kc, kv, (const S*)phi_in, (const S*)c_in, (S*)phi_out, (S*)dpp,
                                                (S*)c_out, (const S*)T_old, (S*)T_new, zchunk);
    return cudaGetLastError();
}

}  // namespace pf3d

namespace pf3d {

// first / last pass of a step with two cells per thread (32 x 8 tiles; decks
// without the smooth noise)
template <typename S>
cudaError_t launch_fused_first_pair(const DomainDesc& d, const StepArgs& s, const Fields& f, bool with_solute,
                                    int zchunk, cudaStream_t st)
{
    if (with_solute)
        return launch_fused_pair_t<S, 8, true, true, true>(d, s, f.phi_old, f.c_old, f.phi_mid, f.dpp, f.c_new,
                                                           f.T_old, f.T_new, zchunk, st);
    return launch_fused_pair_t<S, 8, true, false, false>(d, s, f.phi_old, f.c_old, f.phi_mid, f.dpp, nullptr,
                                                         f.T_old, f.T_new, zchunk, st);
}

template <typename S>
cudaError_t launch_fused_last_pair(const DomainDesc& d, const StepArgs& s, const Fields& f, int zchunk,
                                   cudaStream_t st)
{
    return launch_fused_pair_t<S, 8, false, true, true>(d, s, f.phi_mid, f.c_old, f.phi_new, f.dpp, f.c_new,
                                                        nullptr, nullptr, zchunk, st);
}

}  // namespace pf3d

namespace pf3d {

// many domains, two cells per thread: the persistent work-list kernel of
// k_fused_batch with fused_tile_pair (PASS 0 first pass, 1 last pass)
template <typename S, int TY, int PASS, bool ONE_SWEEP>
__global__ void __launch_bounds__(16 * TY, (PairOcc<S, PASS == 0>::v))
    k_fused_batch_pair(const BatchDomain* __restrict__ doms, const BatchStep* __restrict__ steps,
                       const BatchItem* __restrict__ items, const int* __restrict__ n_items, int zchunk)
{
    using V = typename PairOf<S>::type;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ __align__(16) KC<S> skc;   // the loop constants of the current item
    __shared__ __align__(16) KC<V> skv;   // the same, broadcast to both lanes
    constexpr int nf = (int)(offsetof(KC<S>, hq) / sizeof(S));
    const int n = *n_items;
    const int tid = threadIdx.x + 32 * threadIdx.y;
    for (int w = blockIdx.x; w < n; w += gridDim.x) {
        const BatchItem it = items[w];
        const BatchStep& st = steps[it.dom];
        if (!st.active) continue;   // uniform across the CTA
        const BatchDomain& D = doms[it.dom];
        const int q = st.q_phi, qc = st.q_c, qt = st.q_T;
        static_assert(sizeof(KC<S>) % 4 == 0, "KC is copied as words");
        for (int i = tid; i < (int)(sizeof(KC<S>) / 4); i += 16 * TY)
            reinterpret_cast<int*>(&skc)[i] = reinterpret_cast<const int*>(st.kc)[i];
        __syncthreads();
        for (int i = tid; i < nf; i += 16 * TY) reinterpret_cast<V*>(&skv)[i] = V::splat(reinterpret_cast<const S*>(&skc)[i]);
        if (tid == 0) {
            skv.hq = skc.hq;
            skv.rt = skc.rt;
            skv.it = skc.it;
            skv.lap = skc.lap;
        }
        __syncthreads();
        if (PASS == 0) {
            if (ONE_SWEEP)
                fused_tile_pair<S, TY, true, true, true>(D.d, skc, skv, (const S*)D.phi[q], (const S*)D.c[qc],
                                                         (S*)D.phi[1 - q], (S*)D.dpp, (S*)D.c[1 - qc],
                                                         (const S*)D.T[qt], (S*)D.T[1 - qt], zchunk, it.bx, it.by,
                                                         it.bz, smem_raw);
            else
                fused_tile_pair<S, TY, true, false, false>(D.d, skc, skv, (const S*)D.phi[q], (const S*)D.c[qc],
                                                           (S*)D.phi[1 - q], (S*)D.dpp, nullptr, (const S*)D.T[qt],
                                                           (S*)D.T[1 - qt], zchunk, it.bx, it.by, it.bz, smem_raw);
        } else {
            fused_tile_pair<S, TY, false, true, true>(D.d, skc, skv, (const S*)D.phi[1 - q], (const S*)D.c[qc],
                                                      (S*)D.phi[q], (S*)D.dpp, (S*)D.c[1 - qc], nullptr, nullptr,
                                                      zchunk, it.bx, it.by, it.bz, smem_raw);
        }
    }
}

template <typename S, int PASS, bool ONE_SWEEP>
cudaError_t launch_batch_pair_t(const BatchDomain* doms, const BatchStep* steps, const BatchItem* items,
                                const int* n_items, int zchunk, int n_sm, cudaStream_t st)
{
    auto kern = k_fused_batch_pair<S, 8, PASS, ONE_SWEEP>;
    const size_t smem = fused_smem_bytes<S, 8>();
    static int per_sm = 0;   // one attribute and occupancy query per instantiation
    if (per_sm == 0) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        int nb = 0;
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, kern, 128, smem);
        if (e != cudaSuccess) return e;
        per_sm = nb > 0 ? nb : 1;
    }
    kern<<<n_sm * per_sm, dim3(32, 4), smem, st>>>(doms, steps, items, n_items, zchunk);
    return cudaGetLastError();
}

// a batch pass with two cells per thread (32 x 8 tiles; batches without the
// smooth noise and without heat diffusion)
template <typename S>
cudaError_t launch_fused_batch_pair(const BatchDomain* doms, const BatchStep* steps, const BatchItem* items,
                                    const int* n_items, int pass, bool one_sweep, int zchunk, int n_sm,
                                    cudaStream_t st)
{
    if (pass == 0)
        return one_sweep ? launch_batch_pair_t<S, 0, true>(doms, steps, items, n_items, zchunk, n_sm, st)
                         : launch_batch_pair_t<S, 0, false>(doms, steps, items, n_items, zchunk, n_sm, st);
    return launch_batch_pair_t<S, 1, false>(doms, steps, items, n_items, zchunk, n_sm, st);
}

}  // namespace pf3d
