// pf3d_march.cuh -- the z-marching passes of the coupled step, TMA-staged.
//
// A CTA owns a 32 x TY column tile and a z-chunk and marches along z, like
// the passes of pf3d_fused.cuh, with the same per-cell arithmetic (the fast
// form of pf3d_device.cuh), so every output has the bits of those passes.
// What differs is how data moves and how the boundary is treated:
//
//  * Plane staging.  Each plane of the input phase field (tile + 2-cell halo)
//    is one TMA tiled load (cp.async.bulk.tensor.3d, no multicast) issued by
//    one thread into a 6-slot window and completed on that slot's mbarrier;
//    the loads run two planes ahead of the stencil.  Cells outside the domain
//    read as zero.  Every wait is bounded: a load that does not arrive sets
//    the context's status word and the CTA stops (pf3d_tma.cuh).
//  * Node windows.  The anisotropy quantities (eps^2, exy, eyz, ezx) of every
//    node of the tile and its 1-cell ring, and the solute point quantities
//    (Gamma bracket, mu), are computed once per plane into 3- or 4-plane
//    windows; the window mode (MarchWin) says how many and how many barriers
//    a plane takes, and whether the own column's values roll in registers.
//  * Uniform arithmetic, fan-out stores.  Every cell of every tile -- also
//    the tiles on the domain boundary -- goes through the same arithmetic
//    (two cells per thread as lane pairs when L = 2, packed f32x2 in FP32).
//    The boundary decoration of the reference (plane copies after the sweep,
//    equacao_campo_fase.f90:151-167, concentracao_soluto.f90:116-124) is a
//    per-cell store fan-out: a cell writes its value to every cell whose
//    copy source it is (one store in the interior, up to 27 at a corner).
//    Only the stores diverge; small domains, whose tiles are all boundary
//    tiles, run the paired arithmetic at the interior's cost.
//
// Template switches: HEAT (temperatura), DPPW (write DPP: last sweep), SOL
// (concentracao_soluto from the same input phase field), SMOOTH (the deck
// may draw the smooth noise).  The first pass of a multi-sweep step stores
// the step's REAL(4) noise in the DPP buffer and the last pass reads it back
// (both sweeps use the same it, so the same noise: principal.f90:127-151).
#pragma once
#include <type_traits>
#include "pf3d_launch.h"
#include "pf3d_pair.cuh"
#include "pf3d_tma.cuh"

namespace pf3d {

// L lanes (cells) per thread: the arithmetic type and its packing
template <typename S, int L> struct Lanes;
template <typename S> struct Lanes<S, 1> {
    using V = S;
    static __device__ __forceinline__ V make(const S* a) { return a[0]; }
    static __device__ __forceinline__ S get(const V& v, int) { return v; }
};
template <typename S> struct Lanes<S, 2> {
    using V = typename PairOf<S>::type;
    static __device__ __forceinline__ V make(const S* a) { return V(a[0], a[1]); }
    static __device__ __forceinline__ S get(const V& v, int l) { return l ? v.y() : v.x(); }
};

// Window modes of the march passes (one barrier per plane in each):
//   3: node / solute-point windows of 3 planes.  The cells of plane z read
//      plane z's nodes and points at their neighbours' positions, written
//      by other threads before the previous plane's barrier, and those of
//      planes z-1 and z+1 only at their own position, written by the same
//      thread; so when the nodes of plane z+1 overwrite plane z-2's slot,
//      the last cross-thread reader of that slot (the cells of plane z-2)
//      is behind the previous plane's barrier, and no second barrier is
//      needed;
//   4: windows of 4 planes (a spare slot, same results);
//   5: the own column's values rolled in registers along z -- the phase
//      values of planes z-1, z, z+1 at the cell and its four axis
//      neighbours, the cell's node quantities of planes z-1, z, z+1 and its
//      solute-point quantities of the same planes -- so the stencil reads
//      from shared memory only the in-plane neighbours of plane z (the
//      diagonal phase values and the four neighbour nodes and points),
//      with windows of 3 planes.
template <int WIN> struct MarchWin {
    static_assert(WIN == 3 || WIN == 4 || WIN == 5, "window mode 3, 4 or 5");
    static constexpr int nslot = (WIN == 4) ? 4 : 3;
    static constexpr bool roll = WIN == 5;
};

// Shared-memory layout of one tile (bytes from a 128-byte aligned base).
template <typename S, int TY, bool SOL, int NSLOT>
struct MarchLayout {
    static constexpr int TX = 32;
    // the TMA box starts XOFF cells left of the tile: x * sizeof(S) must be a
    // multiple of 16 bytes (tile origins are multiples of 32 cells)
    static constexpr int XOFF = (sizeof(S) == 8) ? 2 : 4;
    static constexpr int TW = TX + 2 * XOFF;       // phase tile width (box x)
    static constexpr int PH = TY + 4;              // phase tile height (box y)
    static constexpr int NW = TX + 2, NH = TY + 2; // node / point tile (ring 1)
    static constexpr int NQ = NW * NH;
    static constexpr int NPHI = 6;                 // phase planes z-1 .. z+4
    static constexpr int PHI_SLOT = TW * PH;       // elements per phase slot
    static constexpr int PHI_BYTES = PHI_SLOT * (int)sizeof(S);
    static_assert(PHI_BYTES % 128 == 0, "TMA destinations are 128-byte aligned");
    static constexpr int BAR_OFF = NPHI * PHI_BYTES;
    static constexpr int NODE_OFF = (BAR_OFF + NPHI * 8 + 127) / 128 * 128;
    static constexpr int NODE_SLOT = 4 * NQ;       // eps^2, exy, eyz, ezx
    static constexpr int SOL_OFF = NODE_OFF + NSLOT * NODE_SLOT * (int)sizeof(S);
    static constexpr int SOL_SLOT = 2 * NQ;        // Gamma bracket, mu
    static constexpr int BYTES = SOL_OFF + (SOL ? NSLOT * SOL_SLOT * (int)sizeof(S) : 0);
    static constexpr int ALLOC = BYTES + 128;      // slack to align the dynamic base
};

// temperatura at one own cell (temp_body.inc:31-41): the neighbours of TOLD
// are read only when the deck has heat diffusion (D != 0)
template <typename S>
__device__ __forceinline__ S heat_at(const S* __restrict__ T_old, long long id, long long px, long long pl, S PP,
                                     S dppv, const KC<S>& c)
{
    S TE = 0, TW = 0, TN = 0, TS = 0, TT = 0, TB = 0;
    if (c.lap) {
        TE = T_old[id + 1]; TW = T_old[id - 1]; TN = T_old[id + px]; TS = T_old[id - px];
        TT = T_old[id + pl]; TB = T_old[id - pl];
    }
    return heat_new<S>(PP, dppv, TE, TW, TN, TS, TT, TB, c);
}

// (a + k) mod N for a in [0, N) and k in [0, N)
template <int N>
__device__ __forceinline__ int wrap_add(int a, int k)
{
    const int t = a + k;
    return t >= N ? t - N : t;
}

// the dynamic shared-memory base rounded up to 128 bytes.  The offset is
// added to the shared array itself (not computed through an integer cast of
// its address), so the compiler still knows every pointer derived from it
// is a shared-memory pointer and emits shared loads and stores, not generic
// ones with 64-bit address arithmetic.
__device__ __forceinline__ unsigned char* align128(unsigned char* p)
{
    return p + ((128u - (smem_u32(p) & 127u)) & 127u);
}

// Initialises the six plane barriers of a tile's window (one thread), made
// visible to the TMA unit and to every thread of the CTA.
template <typename S, int TY, bool SOL, int NSLOT>
__device__ __forceinline__ void march_init_barriers(unsigned char* smem)
{
    using LY = MarchLayout<S, TY, SOL, NSLOT>;
    if (threadIdx.x == 0 && threadIdx.y == 0) {
        const uint32_t b0 = smem_u32(smem + LY::BAR_OFF);
        for (int s = 0; s < LY::NPHI; ++s) mbar_init(b0 + 8 * s, 1);
        fence_mbar_init();
    }
    __syncthreads();
}

// One 32 x TY x zchunk tile (tile coordinates bx, by, bz) of one domain, read
// from the phase field the tensor map `tm` describes.  `par` carries the
// parity of each plane barrier across the tiles a CTA processes (every load
// issued is waited for).  Returns false if a plane load did not arrive in
// time; the CTA must then stop.  SPLIT: a second copy of the plane body for
// the interior planes, without their z checks (single domains; a batch's
// short items gain less than the larger code costs them, measured).
template <typename S, int L, int TY, int WIN, bool HEAT, bool DPPW, bool SOL, bool SMOOTH, bool SPLIT = true>
__device__ __forceinline__ bool march_tile(const DomainDesc& d, const KC<S>& c, const KC<typename Lanes<S, L>::V>& cv,
                                           const CUtensorMap* tm, const S* __restrict__ c_in,
                                           S* __restrict__ phi_out, S* __restrict__ dpp, S* __restrict__ c_out,
                                           const S* __restrict__ T_old, S* __restrict__ T_new, int zchunk, int bx,
                                           int by, int bz, unsigned char* smem, uint32_t& par)
{
    using LN = Lanes<S, L>;
    using V = typename LN::V;
    constexpr int NSLOT = MarchWin<WIN>::nslot;
    constexpr bool ROLL = MarchWin<WIN>::roll;
    using LY = MarchLayout<S, TY, SOL, NSLOT>;
    constexpr int TX = 32, TW = LY::TW, NW = LY::NW, NH = LY::NH, NQ = LY::NQ, XOFF = LY::XOFF;
    constexpr int TR = TY / L;                                    // thread rows; lane l owns row ty + l*TR
    constexpr int ran_mode = (HEAT && !DPPW) ? 1 : ((!HEAT && DPPW) ? 2 : 0);
    constexpr int NRING = (L == 1) ? 2 * NW + 2 * TY : NW + TY;  // ring items (pairs when L = 2)
    static_assert(TY % L == 0, "tile height must be a multiple of the lanes");

    S* const sphi = reinterpret_cast<S*>(smem);
    const uint32_t bar0 = smem_u32(smem + LY::BAR_OFF);
    S* const snode = reinterpret_cast<S*>(smem + LY::NODE_OFF);
    S* const ssol = reinterpret_cast<S*>(smem + LY::SOL_OFF);

    const int nx = d.nx, ny = d.ny, nz = d.nz;
    const long long px = d.px, pl = d.plane;
    const int x0 = bx * TX, y0 = by * TY;
    const int zb = bz * zchunk;
    const int ze = min(zb + zchunk, nz);
    const int zlast = min(nz - 1, ze + 1);   // the last plane any computation of this tile reads
    const int tx = threadIdx.x, ty = threadIdx.y;
    const int tid = tx + TX * ty;
    const bool lead = tid == 0;
    const int x = x0 + tx;

    // ---- the cells of this thread (lanes) ----
    int yv[L];
    bool own[L];
    long long col[L];
    int phi_off[L], node_off[L];
#pragma unroll
    for (int l = 0; l < L; ++l) {
        yv[l] = y0 + ty + l * TR;
        own[l] = x < nx && yv[l] < ny;
        col[l] = (long long)x + (long long)yv[l] * px;
        phi_off[l] = (ty + l * TR + 2) * TW + (tx + XOFF);
        node_off[l] = (ty + l * TR + 1) * NW + (tx + 1);
    }
    // ---- the ring items of this thread: node-tile positions.  The first
    // NRING threads compute the ring's node quantities, the last NRING its
    // solute points (solute passes), so that no warp carries both ring parts
    // of a plane while the others wait for it at the plane's barrier ----
    constexpr int NT = 32 * TY / L;
    static_assert(2 * NRING <= NT, "the node and solute ring threads are disjoint");
    int rlx[L], rly[L];
    const bool ring = tid < NRING;                      // ring nodes
    const bool ring_s = SOL && tid >= NT - NRING;       // ring solute points
    if (L == 1) {
        int r = ring ? tid : (ring_s ? tid - (NT - NRING) : 0);
        if (r < NW) { rlx[0] = r; rly[0] = 0; }
        else if ((r -= NW) < NW) { rlx[0] = r; rly[0] = NH - 1; }
        else if ((r -= NW) < TY) { rlx[0] = 0; rly[0] = 1 + r; }
        else { r -= TY; rlx[0] = NW - 1; rly[0] = 1 + r; }
    } else {
        const int r = ring ? tid : (ring_s ? tid - (NT - NRING) : 0);
        if (r < NW) { rlx[0] = r; rly[0] = 0; rlx[L - 1] = r; rly[L - 1] = NH - 1; }
        else { rlx[0] = 0; rly[0] = 1 + (r - NW); rlx[L - 1] = NW - 1; rly[L - 1] = 1 + (r - NW); }
    }
    bool rin[L];
    long long rcol[L];
    int rphi_off[L], rnode_off[L];
#pragma unroll
    for (int l = 0; l < L; ++l) {
        const int gx = x0 - 1 + rlx[l], gy = y0 - 1 + rly[l];
        rin[l] = ring_s && gx >= 0 && gx < nx && gy >= 0 && gy < ny;   // a ring point's concentration is read
        rcol[l] = (long long)gx + (long long)gy * px;
        rphi_off[l] = (rly[l] + 1) * TW + (rlx[l] - 1 + XOFF);
        rnode_off[l] = rly[l] * NW + rlx[l];
    }

    // ---- plane loads ----
    uint32_t pend = 0;          // slots with a load issued and not yet seen complete (lead thread)
    auto issue = [&](int p, int s) {   // one thread: plane p into its slot s = p mod 6
        const uint32_t bar = bar0 + 8 * s;
        mbar_arrive_expect_tx(bar, (uint32_t)LY::PHI_BYTES);
        tma_load_3d(smem_u32(sphi + s * LY::PHI_SLOT), tm, x0 - XOFF, y0 - 2, p, bar);
        pend |= 1u << s;
    };
    auto wait_plane = [&](int s) -> bool {   // the load into slot s has landed
        const bool ok = mbar_wait(bar0 + 8 * s, (par >> s) & 1u);
        if (ok) {
            par ^= 1u << s;
            pend &= ~(1u << s);
        }
        return ok;
    };
    // after a failed wait: the lead thread waits (bounded) for the loads
    // still in flight, so that no TMA write lands in shared memory the CTA
    // has left
    auto drain = [&]() {
        if (!lead) return;
        for (int s = 0; s < 6; ++s)
            if ((pend >> s) & 1u) mbar_wait(bar0 + 8 * s, (par >> s) & 1u);
    };

    // the node quantities of one set of items from their gradient; stored
    // into the slot `dst`; the own items' eps^2, eyz, ezx also into `keep`
    auto node_store = [&](S* dst, const int* off_node, V gx, V gy, V gz, S (*keep)[3]) {
        const Node<V> q = aniso_node<V, true>(gx, gy, gz, cv);
        const V eps2 = q.eps * q.eps;   // the stencil reads eps only squared
#pragma unroll
        for (int l = 0; l < L; ++l) {
            S* o = dst + off_node[l];
            o[0] = LN::get(eps2, l);
            o[NQ] = LN::get(q.exy, l);
            o[2 * NQ] = LN::get(q.eyz, l);
            o[3 * NQ] = LN::get(q.ezx, l);
            if (keep) {
                keep[l][0] = LN::get(eps2, l);
                keep[l][1] = LN::get(q.eyz, l);
                keep[l][2] = LN::get(q.ezx, l);
            }
        }
    };
    // node quantities of plane n into its slot, from phase planes n-1, n, n+1
    // in shared memory (own items' values also into `keep` when given)
    auto node_plane = [&](int sl, const S* pm, const S* p0, const S* pp, S (*keep)[3]) {
        S* dst = snode + sl * LY::NODE_SLOT;
        auto one = [&](const int* off_phi, const int* off_node, S (*kp)[3]) {
            S a[L], b[L];
#pragma unroll
            for (int l = 0; l < L; ++l) { a[l] = p0[off_phi[l] + 1]; b[l] = p0[off_phi[l] - 1]; }
            const V gx = grad<V, true>(LN::make(a), LN::make(b), cv.dx, cv.hx);
#pragma unroll
            for (int l = 0; l < L; ++l) { a[l] = p0[off_phi[l] + TW]; b[l] = p0[off_phi[l] - TW]; }
            const V gy = grad<V, true>(LN::make(a), LN::make(b), cv.dy, cv.hy);
#pragma unroll
            for (int l = 0; l < L; ++l) { a[l] = pp[off_phi[l]]; b[l] = pm[off_phi[l]]; }
            const V gz = grad<V, true>(LN::make(a), LN::make(b), cv.dz, cv.hz);
            node_store(dst, off_node, gx, gy, gz, kp);
        };
        one(phi_off, node_off, keep);
        if (ring) one(rphi_off, rnode_off, nullptr);
    };
    // solute point quantities of plane s into its slot, from phase plane s
    // and the concentration of that plane at the own (co) and ring (cr)
    // points; the own points' values also into `keep` when given, and their
    // phase values taken from `ownp` when given
    auto sol_plane = [&](int sl, const S* p0, const S* co, const S* cr, S (*keep)[2], const S* ownp) {
        S* dst = ssol + sl * LY::SOL_SLOT;
        auto one = [&](const int* off_phi, const int* off_node, const S* cc, S (*kp)[2], const S* op) {
            S a[L];
#pragma unroll
            for (int l = 0; l < L; ++l) a[l] = op ? op[l] : p0[off_phi[l]];
            const SolNode<V> q = sol_node<V, true>(LN::make(a), LN::make(cc), cv);
#pragma unroll
            for (int l = 0; l < L; ++l) {
                S* o = dst + off_node[l];
                o[0] = LN::get(q.br, l);
                o[NQ] = LN::get(q.mu, l);
                if (kp) {
                    kp[l][0] = LN::get(q.br, l);
                    kp[l][1] = LN::get(q.mu, l);
                }
            }
        };
        one(phi_off, node_off, co, keep, ownp);
        if (ring_s) one(rphi_off, rnode_off, cr, nullptr, nullptr);
    };
    // concentration of plane s at the own and ring points (a benign value
    // outside the domain, so that no logarithm there leaves the normal range)
    auto load_c = [&](int s, S* co, S* cr) {
        const bool zin = s >= 0 && s < nz;
        const long long zo = (long long)s * pl;
#pragma unroll
        for (int l = 0; l < L; ++l) {
            co[l] = (zin && own[l]) ? c_in[col[l] + zo] : (S)0.02;
            if (SOL) cr[l] = (zin && rin[l]) ? c_in[rcol[l] + zo] : (S)0.02;
        }
    };

    // ---- the cell's flags (x / y parts; z parts are per plane) ----
    const bool xin = x >= 1 && x <= nx - 2;    // T interior, phase source, solute interior
    const bool xph = x >= 2 && x <= nx - 3;    // phase interior
    const bool xone = x >= 3 && x <= nx - 4;   // sole preimage of itself
    bool yin[L], yph[L], yone[L];
    int xl = 0, xh = -1, yl[L], yh[L];
    if (xin) fpre_range(x, nx, &xl, &xh);
#pragma unroll
    for (int l = 0; l < L; ++l) {
        yin[l] = yv[l] >= 1 && yv[l] <= ny - 2;
        yph[l] = yv[l] >= 2 && yv[l] <= ny - 3;
        yone[l] = yv[l] >= 3 && yv[l] <= ny - 4;
        yl[l] = 0;
        yh[l] = -1;
        if (yin[l]) fpre_range(yv[l], ny, &yl[l], &yh[l]);
    }
    // CTA-uniform: every column and row of the tile lies in [3, N-4]
    const bool tile_int = x0 >= 3 && x0 + TX + 3 <= nx && y0 >= 3 && y0 + TY + 3 <= ny;

    // ---- prologue: planes zb-2 .. zb+3 in flight, nodes zb-1, zb ----
    if (lead) {
        fence_proxy_async_smem();   // the slots may hold a previous tile's planes
        for (int p = zb - 2; p <= zb + 3; ++p)
            if (p >= 0 && p <= zlast) issue(p, (p + 6) % 6);
    }
    S co[3][L], cr[2][L];   // concentration: own points of planes z, z+1, z+2; ring points of z+1, z+2
    S nd[L], nt[L];         // centre values of the next plane: DPP (or the noise), TOLD
#pragma unroll
    for (int l = 0; l < L; ++l) { nd[l] = 0; nt[l] = 0; cr[0][l] = cr[1][l] = 0; }
    // DPP / noise and TOLD of the own cells of plane z.  TOLD is read only
    // where the heat equation keeps it (outside 2..N-1): inside, TNEW is TP
    // plus the latent term (and the Laplacian reads its own neighbours)
    auto load_centre = [&](int z) {
        if (!(HEAT || ran_mode == 2) || z >= ze) return;
        const long long zo = (long long)z * pl;
        const bool zi = z >= 1 && z <= nz - 2;
#pragma unroll
        for (int l = 0; l < L; ++l) {
            if (!own[l]) continue;
            nd[l] = dpp[col[l] + zo];
            if (HEAT && !(zi && x >= 1 && x <= nx - 2 && yv[l] >= 1 && yv[l] <= ny - 2)) nt[l] = T_old[col[l] + zo];
        }
    };
    // rolled own-column state (window mode 5): phase values of planes z-1,
    // z, z+1 at the cell and its N, S, E, W neighbours; the cell's node
    // (eps^2, eyz, ezx) and solute-point (bracket, mu) quantities of the same
    // planes.  Index of the five phase values: cell, N, S, E, W.  Unused, and
    // so not allocated, in the other modes.
    S rpm[L][5], rp0[L][5], rpp[L][5];
    S rnB[L][3], rnC[L][3], rnT[L][3];
    S rsB[L][2], rsP[L][2], rsT[L][2];
    auto load5 = [&](S (*dst)[5], const S* pl_) {
        if constexpr (ROLL) {
#pragma unroll
            for (int l = 0; l < L; ++l) {
                const S* q = pl_ + phi_off[l];
                dst[l][0] = q[0]; dst[l][1] = q[TW]; dst[l][2] = q[-TW]; dst[l][3] = q[1]; dst[l][4] = q[-1];
            }
        }
    };
    bool bad = false;
    if (SOL) {
        S ca[L], cra[L];
        load_c(zb - 1, ca, cra);
        load_c(zb, co[0], cr[0]);
        load_c(zb + 1, co[1], cr[1]);
        for (int p = zb - 2; p <= zb + 1; ++p)
            if (p >= 0 && p <= zlast) bad |= !wait_plane((p + 6) % 6);
        if (zb - 1 >= 0)
            sol_plane(wrap_add<NSLOT>(zb % NSLOT, NSLOT - 1), sphi + ((zb + 5) % 6) * LY::PHI_SLOT, ca, cra,
                      ROLL ? rsB : nullptr, nullptr);
        sol_plane(zb % NSLOT, sphi + (zb % 6) * LY::PHI_SLOT, co[0], cr[0], ROLL ? rsP : nullptr, nullptr);
#pragma unroll
        for (int l = 0; l < L; ++l) cr[0][l] = cr[1][l];
    } else {
        load_c(zb, co[0], cr[0]);
        for (int p = zb - 2; p <= zb + 1; ++p)
            if (p >= 0 && p <= zlast) bad |= !wait_plane((p + 6) % 6);
    }
    load_centre(zb);
    if (zb - 1 >= 1 && zb - 1 <= nz - 2)
        node_plane(wrap_add<NSLOT>(zb % NSLOT, NSLOT - 1), sphi + ((zb + 4) % 6) * LY::PHI_SLOT,
                   sphi + ((zb + 5) % 6) * LY::PHI_SLOT,
                   sphi + (zb % 6) * LY::PHI_SLOT, ROLL ? rnB : nullptr);
    if (zb >= 1 && zb <= nz - 2)
        node_plane(zb % NSLOT, sphi + ((zb + 5) % 6) * LY::PHI_SLOT, sphi + (zb % 6) * LY::PHI_SLOT,
                   sphi + ((zb + 1) % 6) * LY::PHI_SLOT, ROLL ? rnC : nullptr);
    load5(rpm, sphi + ((zb + 5) % 6) * LY::PHI_SLOT);
    load5(rp0, sphi + (zb % 6) * LY::PHI_SLOT);

    long long zoff = (long long)zb * pl;
    uint64_t hin[L];   // noise hash input of the own cells, carried along z (k = z + 1)
#pragma unroll
    for (int l = 0; l < L; ++l) hin[l] = hash_base(x + 1, yv[l] + 1, c.it, 1) + (uint64_t)(zb + 1) * kHashK;
    int s6 = zb % 6;       // phase slot of plane z
    int sn = zb % NSLOT;   // node / point slot of plane z

    // One plane of the march.  IN: every z-dependent condition of the plane
    // is known true (z in [3, N-4], the planes it reads and the load it
    // issues all inside the domain and the chunk), so that copy of the body
    // carries none of the checks; the other copy serves the first and last
    // planes.  Returns false when a plane load did not arrive.  Always
    // inlined: an outlined copy would pass every captured value through the
    // stack (measured: 5x slower).
    auto plane = [&](int z, auto in_tag) __attribute__((always_inline)) -> bool {
        constexpr bool IN = decltype(in_tag)::value;
        const int s6p1 = wrap_add<6>(s6, 1), s6p2 = wrap_add<6>(s6, 2);
        const int snm1 = wrap_add<NSLOT>(sn, NSLOT - 1), snp1 = wrap_add<NSLOT>(sn, 1);
        const S* const pm = sphi + wrap_add<6>(s6, 5) * LY::PHI_SLOT;
        const S* const p0 = sphi + s6 * LY::PHI_SLOT;
        const S* const pp = sphi + s6p1 * LY::PHI_SLOT;
        const S* const pq = sphi + s6p2 * LY::PHI_SLOT;
        S dcur[L], tcur[L];
#pragma unroll
        for (int l = 0; l < L; ++l) { dcur[l] = nd[l]; tcur[l] = nt[l]; }
        load_centre(z + 1);
        if (SOL) load_c(z + 2, co[2], cr[1]);
        else load_c(z + 1, co[1], cr[1]);

        // A: plane z+2 has landed
        if (IN || z + 2 <= zlast) bad |= !wait_plane(s6p2);
        // B, C: nodes and solute points of plane z+1
        if constexpr (ROLL) {
            load5(rpp, pp);   // plane z+1 at the own column: the stencil's T values and the node's x/y gradient
            if (IN || (z + 1 >= 1 && z + 1 <= nz - 2)) {
                S a[L], b[L];
#pragma unroll
                for (int l = 0; l < L; ++l) { a[l] = rpp[l][3]; b[l] = rpp[l][4]; }
                const V gx = grad<V, true>(LN::make(a), LN::make(b), cv.dx, cv.hx);
#pragma unroll
                for (int l = 0; l < L; ++l) { a[l] = rpp[l][1]; b[l] = rpp[l][2]; }
                const V gy = grad<V, true>(LN::make(a), LN::make(b), cv.dy, cv.hy);
#pragma unroll
                for (int l = 0; l < L; ++l) { a[l] = pq[phi_off[l]]; b[l] = rp0[l][0]; }
                const V gz = grad<V, true>(LN::make(a), LN::make(b), cv.dz, cv.hz);
                S* const dst = snode + snp1 * LY::NODE_SLOT;
                node_store(dst, node_off, gx, gy, gz, rnT);
                if (ring) {
#pragma unroll
                    for (int l = 0; l < L; ++l) { a[l] = pp[rphi_off[l] + 1]; b[l] = pp[rphi_off[l] - 1]; }
                    const V rx = grad<V, true>(LN::make(a), LN::make(b), cv.dx, cv.hx);
#pragma unroll
                    for (int l = 0; l < L; ++l) { a[l] = pp[rphi_off[l] + TW]; b[l] = pp[rphi_off[l] - TW]; }
                    const V ry = grad<V, true>(LN::make(a), LN::make(b), cv.dy, cv.hy);
#pragma unroll
                    for (int l = 0; l < L; ++l) { a[l] = pq[rphi_off[l]]; b[l] = p0[rphi_off[l]]; }
                    const V rz = grad<V, true>(LN::make(a), LN::make(b), cv.dz, cv.hz);
                    node_store(dst, rnode_off, rx, ry, rz, nullptr);
                }
            }
            if (SOL && (IN || z + 1 <= nz - 1)) {
                S op[L];
#pragma unroll
                for (int l = 0; l < L; ++l) op[l] = rpp[l][0];
                sol_plane(snp1, pp, co[1], cr[0], rsT, op);
            }
        } else {
            if (IN || (z + 1 >= 1 && z + 1 <= nz - 2)) node_plane(snp1, p0, pp, pq, nullptr);
            if (SOL && (IN || z + 1 <= nz - 1)) sol_plane(snp1, pp, co[1], cr[0], nullptr, nullptr);
        }
        // D: one barrier orders the plane; everyone learns of a failed load
        if (__syncthreads_or(bad)) {
            drain();
            return false;
        }
        // E: the load of plane z+4 into the slot plane z-2 has left
        if (lead && (IN || z + 4 <= zlast)) {
            fence_proxy_async_smem();
            issue(z + 4, wrap_add<6>(s6, 4));
        }

        // F: the cells of plane z
        const bool zin = IN || (z >= 1 && z <= nz - 2);   // T interior / phase source / solute interior
        const bool zph = IN || (z >= 2 && z <= nz - 3);   // phase interior
        const S* const nm1 = snode + snm1 * LY::NODE_SLOT;
        const S* const n0 = snode + sn * LY::NODE_SLOT;
        const S* const np1 = snode + snp1 * LY::NODE_SLOT;
        S PPs[L];
#pragma unroll
        for (int l = 0; l < L; ++l) PPs[l] = ROLL ? rp0[l][0] : p0[phi_off[l]];
        const V PP = LN::make(PPs);
        const V CPP = LN::make(co[0]);

        // the REAL(4) noise of the own cells
        float ran[L];
#pragma unroll
        for (int l = 0; l < L; ++l) {
            if constexpr (ran_mode == 2) {
                ran[l] = (float)dcur[l];
            } else if constexpr (SMOOTH) {
                ran[l] = (c.rt == 2) ? phase_ran(2, x + 1, yv[l] + 1, z + 1, c.it)
                                     : __double2float_rn(ran64(hash63_mix(hin[l])));
            } else {
                ran[l] = __double2float_rn(ran64(hash63_mix(hin[l])));
            }
            hin[l] += kHashK;
        }

        V ppn = PP;
        if (zph) {
            Nbr<V> nb;
            S t[L];
#define PF3D_NB(FIELD, PLANE, DELTA)                                         \
    _Pragma("unroll") for (int l = 0; l < L; ++l) t[l] = PLANE[phi_off[l] + (DELTA)]; \
    nb.FIELD = LN::make(t);
#define PF3D_NR(FIELD, ARR, I)                                               \
    _Pragma("unroll") for (int l = 0; l < L; ++l) t[l] = ARR[l][I];          \
    nb.FIELD = LN::make(t);
            nb.PP = PP;
            if constexpr (ROLL) {
                PF3D_NR(PN, rp0, 1) PF3D_NR(PS, rp0, 2) PF3D_NR(PE, rp0, 3) PF3D_NR(PW, rp0, 4)
                PF3D_NR(PT, rpp, 0) PF3D_NR(PB, rpm, 0)
                PF3D_NR(PNT, rpp, 1) PF3D_NR(PNB, rpm, 1) PF3D_NR(PST, rpp, 2) PF3D_NR(PSB, rpm, 2)
                PF3D_NR(PET, rpp, 3) PF3D_NR(PEB, rpm, 3) PF3D_NR(PWT, rpp, 4) PF3D_NR(PWB, rpm, 4)
            } else {
                PF3D_NB(PN, p0, TW) PF3D_NB(PS, p0, -TW) PF3D_NB(PE, p0, 1) PF3D_NB(PW, p0, -1)
                PF3D_NB(PT, pp, 0) PF3D_NB(PB, pm, 0)
                PF3D_NB(PNT, pp, TW) PF3D_NB(PNB, pm, TW) PF3D_NB(PST, pp, -TW) PF3D_NB(PSB, pm, -TW)
                PF3D_NB(PET, pp, 1) PF3D_NB(PEB, pm, 1) PF3D_NB(PWT, pp, -1) PF3D_NB(PWB, pm, -1)
            }
            PF3D_NB(PNE, p0, TW + 1) PF3D_NB(PSE, p0, -TW + 1) PF3D_NB(PNW, p0, TW - 1) PF3D_NB(PSW, p0, -TW - 1)
#undef PF3D_NB
            Node<V> E, W, N, So, Tt, B;
#define PF3D_ND(NODE, Q, PLANE, DELTA, QI)                                   \
    _Pragma("unroll") for (int l = 0; l < L; ++l) t[l] = PLANE[node_off[l] + (DELTA) + (QI) * NQ]; \
    NODE.Q = LN::make(t);
            PF3D_ND(E, eps, n0, 1, 0) PF3D_ND(E, exy, n0, 1, 1) PF3D_ND(E, ezx, n0, 1, 3)
            PF3D_ND(W, eps, n0, -1, 0) PF3D_ND(W, exy, n0, -1, 1) PF3D_ND(W, ezx, n0, -1, 3)
            PF3D_ND(N, eps, n0, NW, 0) PF3D_ND(N, exy, n0, NW, 1) PF3D_ND(N, eyz, n0, NW, 2)
            PF3D_ND(So, eps, n0, -NW, 0) PF3D_ND(So, exy, n0, -NW, 1) PF3D_ND(So, eyz, n0, -NW, 2)
            if constexpr (ROLL) {
#define PF3D_NN(NODE, Q, ARR, I)                                             \
    _Pragma("unroll") for (int l = 0; l < L; ++l) t[l] = ARR[l][I];          \
    NODE.Q = LN::make(t);
                PF3D_NN(Tt, eps, rnT, 0) PF3D_NN(Tt, eyz, rnT, 1) PF3D_NN(Tt, ezx, rnT, 2)
                PF3D_NN(B, eps, rnB, 0) PF3D_NN(B, eyz, rnB, 1) PF3D_NN(B, ezx, rnB, 2)
#undef PF3D_NN
            } else {
                PF3D_ND(Tt, eps, np1, 0, 0) PF3D_ND(Tt, eyz, np1, 0, 2) PF3D_ND(Tt, ezx, np1, 0, 3)
                PF3D_ND(B, eps, nm1, 0, 0) PF3D_ND(B, eyz, nm1, 0, 2) PF3D_ND(B, ezx, nm1, 0, 3)
            }
#undef PF3D_ND
#undef PF3D_NR
            E.eyz = W.eyz = N.ezx = So.ezx = Tt.exy = B.exy = V((S)0);   // unused by the body
            S rs[L];
#pragma unroll
            for (int l = 0; l < L; ++l) rs[l] = (S)ran[l];
            ppn = phase_ppnew<V, true, true>(nb, E, W, N, So, Tt, B, CPP, LN::make(rs), cv);
        }
        V cn = CPP;
        if (SOL && zin) {
            const S* const sm1 = ssol + snm1 * LY::SOL_SLOT;
            const S* const s0 = ssol + sn * LY::SOL_SLOT;
            const S* const sp1 = ssol + snp1 * LY::SOL_SLOT;
            SolNode<V> q[7];   // P, E, W, N, S, T, B
            S a[L], b[L];
#define PF3D_SN(I, PLANE, DELTA)                                                                   \
    _Pragma("unroll") for (int l = 0; l < L; ++l) { a[l] = PLANE[node_off[l] + (DELTA)];          \
                                                     b[l] = PLANE[node_off[l] + (DELTA) + NQ]; }  \
    q[I].br = LN::make(a);                                                                         \
    q[I].mu = LN::make(b);
            PF3D_SN(1, s0, 1) PF3D_SN(2, s0, -1) PF3D_SN(3, s0, NW) PF3D_SN(4, s0, -NW)
            if constexpr (ROLL) {
#define PF3D_SR(I, ARR)                                                                              \
    _Pragma("unroll") for (int l = 0; l < L; ++l) { a[l] = ARR[l][0]; b[l] = ARR[l][1]; }           \
    q[I].br = LN::make(a);                                                                           \
    q[I].mu = LN::make(b);
                PF3D_SR(0, rsP) PF3D_SR(5, rsT) PF3D_SR(6, rsB)
#undef PF3D_SR
            } else {
                PF3D_SN(0, s0, 0) PF3D_SN(5, sp1, 0) PF3D_SN(6, sm1, 0)
            }
#undef PF3D_SN
            cn = conc_new<V, true>(PP, CPP, q[0], q[1], q[2], q[3], q[4], q[5], q[6], cv);
        }
        const V U = clamp01(ppn);
        const V DP = ppn - PP;

        if (tile_int && (IN || (z >= 3 && z <= nz - 4))) {
            // every cell of the tile plane is interior and its own only
            // preimage (CTA-uniform branch)
#pragma unroll
            for (int l = 0; l < L; ++l) {
                const long long id = col[l] + zoff;
                if (HEAT) T_new[id] = heat_at<S>(T_old, id, px, pl, PPs[l], dcur[l], c);
                if (ran_mode == 1) dpp[id] = (S)ran[l];
                if (DPPW) dpp[id] = LN::get(DP, l);
                phi_out[id] = LN::get(U, l);
                if (SOL) c_out[id] = LN::get(cn, l);
            }
        } else {
#pragma unroll
            for (int l = 0; l < L; ++l) {
                if (!own[l]) continue;
                const int y = yv[l];
                const long long id = col[l] + zoff;
                const bool src = xin && yin[l] && zin;   // T interior; phase copy source
                if (HEAT) {
                    S tn = tcur[l];
                    if (src) tn = heat_at<S>(T_old, id, px, pl, PPs[l], dcur[l], c);
                    T_new[id] = tn;
                }
                if (src) {
                    const bool inner = xph && yph[l] && zph;
                    S u = PPs[l];
                    if (inner) {
                        if (ran_mode == 1) dpp[id] = (S)ran[l];
                        if (DPPW) dpp[id] = LN::get(DP, l);
                        u = LN::get(U, l);
                    }
                    if (xone && yone[l] && z >= 3 && z <= nz - 4) {
                        phi_out[id] = u;
                    } else {
                        int zl, zh;
                        fpre_range(z, nz, &zl, &zh);
                        for (int zz = zl; zz <= zh; ++zz)
                            for (int yy = yl[l]; yy <= yh[l]; ++yy)
                                for (int xx = xl; xx <= xh; ++xx)
                                    phi_out[(long long)xx + (long long)yy * px + (long long)zz * pl] = u;
                    }
                }
                if (SOL) {
                    // concentracao_soluto.f90:116-124 as a fan-out: the point
                    // writes its value to the face cells copied from it
                    const S uc = src ? LN::get(cn, l) : co[0][l];
                    if (src) c_out[id] = uc;
                    if (z == 1) c_out[id - pl] = uc;
                    if (z == nz - 2) c_out[id + pl] = uc;
                    if (zin && x == 1) c_out[id - 1] = uc;
                    if (zin && x == nx - 2) c_out[id + 1] = uc;
                    if (zin && xin && y == 1) c_out[id - px] = uc;
                    if (zin && xin && y == ny - 2) c_out[id + px] = uc;
                }
            }
        }

        // rotate the concentration registers and the phase slot
#pragma unroll
        for (int l = 0; l < L; ++l) {
            co[0][l] = co[1][l];
            if (SOL) {
                co[1][l] = co[2][l];
                cr[0][l] = cr[1][l];
            }
        }
        if constexpr (ROLL) {
#pragma unroll
            for (int l = 0; l < L; ++l) {
#pragma unroll
                for (int i = 0; i < 5; ++i) {
                    rpm[l][i] = rp0[l][i];
                    rp0[l][i] = rpp[l][i];
                }
#pragma unroll
                for (int i = 0; i < 3; ++i) {
                    rnB[l][i] = rnC[l][i];
                    rnC[l][i] = rnT[l][i];
                }
#pragma unroll
                for (int i = 0; i < 2; ++i) {
                    rsB[l][i] = rsP[l][i];
                    rsP[l][i] = rsT[l][i];
                }
            }
        }
        s6 = s6p1;
        sn = snp1;
        zoff += pl;
        return true;
    };
    if constexpr (SPLIT) {
        // interior planes [zi0, zi1): z >= 3, z <= nz - 4 and z + 4 <= zlast
        const int zi0 = max(zb, 3), zi1 = min(min(ze, nz - 3), zlast - 3);
        int z = zb;
        for (; z < ze && z < zi0; ++z)
            if (!plane(z, std::false_type{})) return false;
        for (; z < zi1; ++z)
            if (!plane(z, std::true_type{})) return false;
        for (; z < ze; ++z)
            if (!plane(z, std::false_type{})) return false;
    } else {
        for (int z = zb; z < ze; ++z)
            if (!plane(z, std::false_type{})) return false;
    }
    return true;
}

// resident CTAs per SM the register budget is sized for (shared memory
// allows no more): FP64 3, or 2 -- 128 registers a thread -- for the rolled
// window mode (its carried column values), a solute pass with 4-plane
// windows and a pass that may draw the smooth noise (its trilinear blend of
// eight hashes); FP32 pairs 6 (80 registers, no spills), 5 in the rolled
// mode; FP32 single cells 3
template <typename S, int L, int WIN, bool SOL, bool HEAT, bool SMOOTH = false>
struct MarchOcc {
    static constexpr int v = (sizeof(S) == 8) ? ((WIN == 5 || (SOL && WIN == 4) || SMOOTH) ? 2 : 3)
                                              : (L == 2 ? ((WIN != 5) ? 6 : 5) : 3);
};

// single domain: one CTA per tile; the phase field comes through `tm`
template <typename S, int L, int TY, int WIN, bool HEAT, bool DPPW, bool SOL, bool SMOOTH>
__global__ void __launch_bounds__(32 * TY / L, (MarchOcc<S, L, WIN, SOL, HEAT, SMOOTH>::v))
    k_march(const __grid_constant__ CUtensorMap tm, DomainDesc d, const KC<S> c,
            const KC<typename Lanes<S, L>::V> cv, const S* __restrict__ c_in, S* __restrict__ phi_out,
            S* __restrict__ dpp, S* __restrict__ c_out, const S* __restrict__ T_old, S* __restrict__ T_new,
            int zchunk, int* __restrict__ err)
{
    extern __shared__ __align__(128) unsigned char smem_raw[];
    unsigned char* smem = align128(smem_raw);
    march_init_barriers<S, TY, SOL, MarchWin<WIN>::nslot>(smem);
    uint32_t par = 0;
    if (!march_tile<S, L, TY, WIN, HEAT, DPPW, SOL, SMOOTH>(d, c, cv, &tm, c_in, phi_out, dpp, c_out, T_old,
                                                                T_new, zchunk, blockIdx.x, blockIdx.y, blockIdx.z,
                                                                smem, par)) {
        if (threadIdx.x == 0 && threadIdx.y == 0) atomicExch(err, kErrTmaTimeout);
    }
}

// many domains: a persistent grid walks the work list.  PASS 0 is the first
// pass of a step (temperatura + sweep 1, or the whole step with one sweep),
// PASS 1 the last (sweep 2 + solute).  tmaps[2 d + b] describes buffer b of
// domain d's phase field.  Items are handed out dynamically: each CTA starts
// with item blockIdx.x and then takes the next unclaimed item from the
// counter *ctr (zero before the launch), so CTAs that drew short items (thin
// z-chunks, small domains at the end of the largest-first list) keep
// working while others finish long ones.
template <typename S, int L, int TY, int WIN, int PASS, bool ONE_SWEEP, bool SMOOTH>
__global__ void __launch_bounds__(32 * TY / L,
                                  (MarchOcc<S, L, WIN, PASS == 1 || ONE_SWEEP, PASS == 0, SMOOTH>::v))
    k_march_batch(const BatchDomain* __restrict__ doms, const CUtensorMap* __restrict__ tmaps,
                  const BatchStep* __restrict__ steps, const BatchItem* __restrict__ items,
                  const int* __restrict__ n_items, int zchunk, int* __restrict__ ctr, int* __restrict__ err)
{
    using V = typename Lanes<S, L>::V;
    constexpr bool SOL = PASS == 1 || ONE_SWEEP;
    __shared__ int s_next;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    __shared__ __align__(16) KC<S> skc;   // the loop constants of the current item
    __shared__ __align__(16) KC<V> skv;   // the same, broadcast to the lanes (L = 2)
    constexpr int nf = (int)(offsetof(KC<S>, hq) / sizeof(S));
    constexpr int NT = 32 * TY / L;
    unsigned char* smem = align128(smem_raw);
    march_init_barriers<S, TY, SOL, MarchWin<WIN>::nslot>(smem);
    uint32_t par = 0;
    const int n = *n_items;
    const int tid = threadIdx.x + 32 * threadIdx.y;
    for (int w = blockIdx.x; w < n;) {
        const BatchItem it = items[w];
        const BatchStep& st = steps[it.dom];
        // the next item, claimed now so the atomic's latency hides behind this one
        __syncthreads();            // every thread has read the previous claim
        if (tid == 0) s_next = (int)gridDim.x + atomicAdd(ctr, 1);
        if (!st.active) {           // uniform across the CTA
            __syncthreads();
            w = s_next;
            continue;
        }
        const BatchDomain& D = doms[it.dom];
        const int q = st.q_phi, qc = st.q_c, qt = st.q_T;
        __syncthreads();            // the previous item is done with the constants and the windows
        static_assert(sizeof(KC<S>) % 4 == 0, "KC is copied as words");
        for (int i = tid; i < (int)(sizeof(KC<S>) / 4); i += NT)
            reinterpret_cast<int*>(&skc)[i] = reinterpret_cast<const int*>(st.kc)[i];
        if (L == 2) {
            __syncthreads();
            for (int i = tid; i < nf; i += NT)
                reinterpret_cast<V*>(&skv)[i] = V(reinterpret_cast<const S*>(&skc)[i]);
            if (tid == 0) {
                skv.hq = skc.hq;
                skv.rt = skc.rt;
                skv.it = skc.it;
                skv.lap = skc.lap;
            }
        }
        __syncthreads();
        const KC<V>& kv = (L == 2) ? skv : *reinterpret_cast<const KC<V>*>(&skc);
        bool ok;
        if (PASS == 0) {
            const CUtensorMap* tm = tmaps + 2 * it.dom + q;
            if (ONE_SWEEP)
                ok = march_tile<S, L, TY, WIN, true, true, true, SMOOTH, false>(
                    D.d, skc, kv, tm, (const S*)D.c[qc], (S*)D.phi[1 - q], (S*)D.dpp, (S*)D.c[1 - qc],
                    (const S*)D.T[qt], (S*)D.T[1 - qt], zchunk, it.bx, it.by, it.bz, smem, par);
            else
                ok = march_tile<S, L, TY, WIN, true, false, false, SMOOTH, false>(
                    D.d, skc, kv, tm, (const S*)D.c[qc], (S*)D.phi[1 - q], (S*)D.dpp, nullptr, (const S*)D.T[qt],
                    (S*)D.T[1 - qt], zchunk, it.bx, it.by, it.bz, smem, par);
        } else {
            const CUtensorMap* tm = tmaps + 2 * it.dom + (1 - q);
            ok = march_tile<S, L, TY, WIN, false, true, true, false, false>(
                D.d, skc, kv, tm, (const S*)D.c[qc], (S*)D.phi[q], (S*)D.dpp, (S*)D.c[1 - qc], nullptr, nullptr,
                zchunk, it.bx, it.by, it.bz, smem, par);
        }
        if (!ok) {
            if (tid == 0) atomicExch(err, kErrTmaTimeout);
            return;
        }
        __syncthreads();            // the claim is visible (and the tile is done)
        w = s_next;
    }
}

// ---------------------------------------------------------------------------
// host launchers
// ---------------------------------------------------------------------------

// KC with every scalar constant broadcast to the lanes (host side)
template <typename S, int L>
KC<typename Lanes<S, L>::V> kc_lanes(const KC<S>& k)
{
    using V = typename Lanes<S, L>::V;
    if constexpr (L == 1) {
        return k;
    } else {
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
}

template <typename S, int L, int TY, int WIN, bool HEAT, bool DPPW, bool SOL, bool SMOOTH>
cudaError_t launch_march_t(const CUtensorMap& tm, const DomainDesc& d, const StepArgs& s, const void* c_in,
                           void* phi_out, void* dpp, void* c_out, const void* T_old, void* T_new, int zchunk,
                           int* err, cudaStream_t st)
{
    using LY = MarchLayout<S, TY, SOL, MarchWin<WIN>::nslot>;
    auto kern = k_march<S, L, TY, WIN, HEAT, DPPW, SOL, SMOOTH>;
    static bool configured = false;   // one attribute call per instantiation
    if (!configured) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, LY::ALLOC);
        if (e != cudaSuccess) return e;
        configured = true;
    }
    if (zchunk <= 0) zchunk = d.nz;
    KC<S> kc;
    kc.load(d, s);
    const auto kv = kc_lanes<S, L>(kc);
    dim3 grid((d.nx + 31) / 32, (d.ny + TY - 1) / TY, (d.nz + zchunk - 1) / zchunk);
    kern<<<grid, dim3(32, TY / L), LY::ALLOC, st>>>(tm, d, kc, kv, (const S*)c_in, (S*)phi_out, (S*)dpp, (S*)c_out,
                                                     (const S*)T_old, (S*)T_new, zchunk, err);
    return cudaGetLastError();
}

// the passes of a step (32 x 8 tiles).  lanes: cells per thread (1 or 2);
// win: window mode (3, 4 or 5, MarchWin).  The smooth noise runs one cell
// per thread.
template <typename S>
cudaError_t launch_march_first(const CUtensorMap& tm, const DomainDesc& d, const StepArgs& s, const Fields& f,
                               bool with_solute, int lanes, int win, int zchunk, int* err, cudaStream_t st)
{
    const bool smooth = d.rt == 2;
#define PF3D_MF(L, NS, DW, SO, SM)                                                                            \
    launch_march_t<S, L, 8, NS, true, DW, SO, SM>(tm, d, s, f.c_old, f.phi_mid, f.dpp, SO ? f.c_new : nullptr, \
                                                  f.T_old, f.T_new, zchunk, err, st)
#define PF3D_MW(L, DW, SO, SM) \
    (win == 3 ? PF3D_MF(L, 3, DW, SO, SM) : win == 4 ? PF3D_MF(L, 4, DW, SO, SM) : PF3D_MF(L, 5, DW, SO, SM))
    if (smooth) return with_solute ? PF3D_MW(1, true, true, true) : PF3D_MW(1, false, false, true);
    if (with_solute) return lanes == 2 ? PF3D_MW(2, true, true, false) : PF3D_MW(1, true, true, false);
    return lanes == 2 ? PF3D_MW(2, false, false, false) : PF3D_MW(1, false, false, false);
#undef PF3D_MW
#undef PF3D_MF
}

template <typename S>
cudaError_t launch_march_last(const CUtensorMap& tm, const DomainDesc& d, const StepArgs& s, const Fields& f,
                              int lanes, int win, int zchunk, int* err, cudaStream_t st)
{
#define PF3D_ML(L, NS)                                                                                     \
    launch_march_t<S, L, 8, NS, false, true, true, false>(tm, d, s, f.c_old, f.phi_new, f.dpp, f.c_new, nullptr, \
                                                          nullptr, zchunk, err, st)
#define PF3D_MW(L) (win == 3 ? PF3D_ML(L, 3) : win == 4 ? PF3D_ML(L, 4) : PF3D_ML(L, 5))
    return lanes == 2 ? PF3D_MW(2) : PF3D_MW(1);
#undef PF3D_MW
#undef PF3D_ML
}

// The persistent grid is the SM count times the CTAs of this kernel that are
// resident on one SM.
template <typename S, int L, int WIN, int PASS, bool ONE_SWEEP, bool SMOOTH>
cudaError_t launch_march_batch_t(const BatchDomain* doms, const CUtensorMap* tmaps, const BatchStep* steps,
                                 const BatchItem* items, const int* n_items, int zchunk, int n_sm, int* ctr,
                                 int* err, cudaStream_t st)
{
    constexpr bool SOL = PASS == 1 || ONE_SWEEP;
    using LY = MarchLayout<S, 8, SOL, MarchWin<WIN>::nslot>;
    auto kern = k_march_batch<S, L, 8, WIN, PASS, ONE_SWEEP, SMOOTH>;
    static int per_sm = 0;   // one attribute and occupancy query per instantiation
    if (per_sm == 0) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, LY::ALLOC);
        if (e != cudaSuccess) return e;
        int nb = 0;
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, kern, 32 * 8 / L, LY::ALLOC);
        if (e != cudaSuccess) return e;
        per_sm = nb > 0 ? nb : 1;
    }
    kern<<<n_sm * per_sm, dim3(32, 8 / L), LY::ALLOC, st>>>(doms, tmaps, steps, items, n_items, zchunk, ctr, err);
    return cudaGetLastError();
}

template <typename S>
cudaError_t launch_march_batch(const BatchDomain* doms, const CUtensorMap* tmaps, const BatchStep* steps,
                               const BatchItem* items, const int* n_items, int pass, bool one_sweep, bool smooth,
                               int lanes, int win, int zchunk, int n_sm, int* ctr, int* err, cudaStream_t st)
{
#define PF3D_MB(L, NS, P, ONE, SM) \
    launch_march_batch_t<S, L, NS, P, ONE, SM>(doms, tmaps, steps, items, n_items, zchunk, n_sm, ctr, err, st)
#define PF3D_MW(L, P, ONE, SM) \
    (win == 3 ? PF3D_MB(L, 3, P, ONE, SM) : win == 4 ? PF3D_MB(L, 4, P, ONE, SM) : PF3D_MB(L, 5, P, ONE, SM))
    if (pass == 0) {
        if (smooth) return one_sweep ? PF3D_MW(1, 0, true, true) : PF3D_MW(1, 0, false, true);
        if (lanes == 2) return one_sweep ? PF3D_MW(2, 0, true, false) : PF3D_MW(2, 0, false, false);
        return one_sweep ? PF3D_MW(1, 0, true, false) : PF3D_MW(1, 0, false, false);
    }
    return lanes == 2 ? PF3D_MW(2, 1, false, false) : PF3D_MW(1, 1, false, false);
#undef PF3D_MW
#undef PF3D_MB
}

}  // namespace pf3d
