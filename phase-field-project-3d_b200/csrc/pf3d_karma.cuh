// pf3d_karma.cuh -- the quantitative Karma model of the reference
// (karma/karma3d.f90: Karma PRL 87 115701 2001; Echebarria, Folch, Karma &
// Plapp PRE 70 061604 2004) on the z-marching tile scheme of the main model.
//
// State: phi in [-1, 1] and the dimensionless supersaturation U, interior
// cells only, Fortran order with a padded row pitch.  The reference keeps a
// ghost layer refreshed by mirror copies on every face (espelho,
// karma3d.f90:318-339); a mirror ghost equals the interior value at the
// clamped index, so the kernels clamp their neighbour indices instead.
//
// One step = two passes (the U equation needs dphi/dt at the face
// neighbours, karma3d.f90:209):
//   pass A (karma3d.f90:166-207): dphi from phi (19-point stencil: centre,
//           6 faces, 12 edges) and U at the centre;
//   pass B (karma3d.f90:212-287): U_new from phi, U and dphi (anti-trapping
//           current through the 6 faces) and phi_new = clamp(phi + dt dphi).
// Each CTA owns a 32 x TY column tile and marches a z-chunk with rolling
// shared-memory windows of 4 planes (tile + 1-cell ring): 3 in use while the
// next is copied in with cp.async.  Every operation
// is the reference's, in its order, with IEEE division and square root and
// no contraction: the FP64 result is the reference's arithmetic bit for bit
// (checked against the C oracle).
#pragma once
#include <cstdint>
#include "pf3d_launch.h"
#include "pf3d_cpasync.cuh"

namespace pf3d {

struct KarmaDesc {
    int nx, ny, nz;
    long long px, plane;    // row pitch and plane stride (elements)
    int it;                 // step being computed (noise)
};

// loop constants, each computed on the host exactly as the reference's
// expression computes it (same operations, same rounding)
template <typename T>
struct KarmaK {
    T idx;        // 1/dx
    T q;          // 0.25*idx
    T h;          // 0.5*idx
    T om3;        // 1 - 3 eps4
    T e4;         // 4 eps4
    T e16;        // 16 eps4
    T lambda, dt, Fnoise, sqdt;   // sqdt = sqrt(dt)
    T omk;        // 1 - k
    T Ahalf1;     // 0.5*(1+k)
    T Ahalf2;     // 0.5*(1-k)
    T D;          // a2*lambda
    T at;         // 1/(2 sqrt 2)
};

template <typename T>
__device__ __forceinline__ T k_fluxn(T g1, T g2, T g3, const KarmaK<T>& c)
{
    const T g2s = g1 * g1 + g2 * g2 + g3 * g3;
    if (g2s < (T)1.e-20) return (c.om3 * c.om3) * g1;
    const T a = g1 * g1, b = g2 * g2, d = g3 * g3;
    const T s4 = a * a + b * b + d * d;
    const T as = c.om3 + c.e4 * s4 / (g2s * g2s);
    return as * (as * g1 + c.e16 * ((g1 * g1) * g1 - g1 * s4 / g2s) / g2s);
}

// karma3d.f90:52-67 in [-1, 1)
__device__ __forceinline__ double k_ruido(int i, int j, int k, int it)
{
    uint64_t h = (uint64_t)(int64_t)i * 2654435761ull + (uint64_t)(int64_t)j * 2246822519ull +
                 (uint64_t)(int64_t)k * 3266489917ull + (uint64_t)(int64_t)it * 668265263ull + 1ull;
    h ^= h >> 33;
    h *= 0xff51afd7ed558ccdull;
    h ^= h >> 33;
    h *= 0xc4ceb9fe1a85ec53ull;
    h ^= h >> 33;
    const double m = (double)(long long)(h & 0x7fffffffffffffffull);
    return __dsub_rn(__ddiv_rn(__dmul_rn(2.0, m), 9223372036854775808.0), 1.0);
}

template <typename T, int TY>
struct KarmaSmem {
    static constexpr int W = 34, H = TY + 2;
    T a[4][H][W];
};

__device__ __forceinline__ int kclamp(int v, int n) { return v < 0 ? 0 : (v >= n ? n - 1 : v); }

// issues the asynchronous copy of plane z (clamped) of f with the 1-cell
// ring (clamped) into dst; the caller commits and waits
template <typename T, int TY>
__device__ __forceinline__ void k_load_plane(const KarmaDesc& d, const T* __restrict__ f, int z, int x0, int y0,
                                             T (*dst)[34])
{
    const int zc = kclamp(z, d.nz);
    const T* src = f + (long long)zc * d.plane;
    const int tx = threadIdx.x, ty = threadIdx.y;
    for (int ly = ty; ly < TY + 2; ly += TY) {
        const T* row = src + (long long)kclamp(y0 - 1 + ly, d.ny) * d.px;
        cp_async_elem(&dst[ly][tx], row + kclamp(x0 - 1 + tx, d.nx), (int)sizeof(T));
        if (tx < 2) cp_async_elem(&dst[ly][32 + tx], row + kclamp(x0 + 31 + tx, d.nx), (int)sizeof(T));
    }
}

// pass A: dphi of karma3d.f90:166-207
template <typename T, int TY>
__global__ void __launch_bounds__(32 * TY) k_karma_phase(KarmaDesc d, const KarmaK<T> c, const T* __restrict__ phi,
                                                        const T* __restrict__ U, T* __restrict__ dphi, int zchunk)
{
    __shared__ KarmaSmem<T, TY> sm;
    const int x0 = blockIdx.x * 32, y0 = blockIdx.y * TY;
    const int zb = blockIdx.z * zchunk, ze = min(zb + zchunk, d.nz);
    const int tx = threadIdx.x, ty = threadIdx.y;
    const int x = x0 + tx, y = y0 + ty;
    const bool own = x < d.nx && y < d.ny;
    const int fx = tx + 1, fy = ty + 1;
    const long long col = (long long)x + (long long)y * d.px;
    int sm1 = 0, s0 = 1, sp1 = 2, sfree = 3;
    k_load_plane<T, TY>(d, phi, zb - 1, x0, y0, sm.a[sm1]);
    k_load_plane<T, TY>(d, phi, zb, x0, y0, sm.a[s0]);
    k_load_plane<T, TY>(d, phi, zb + 1, x0, y0, sm.a[sp1]);
    cp_async_commit();
    T u_next = (own && zb < ze) ? U[col + (long long)zb * d.plane] : (T)0;
    cp_async_wait_all();
    __syncthreads();
    for (int z = zb; z < ze; ++z) {
        // plane z+2 lands in the free slot while plane z is computed
        if (z + 1 < ze) k_load_plane<T, TY>(d, phi, z + 2, x0, y0, sm.a[sfree]);
        cp_async_commit();
        const T uc = u_next;
        if (own && z + 1 < ze) u_next = U[col + (long long)(z + 1) * d.plane];
        if (own) {
            const T(*B)[34] = sm.a[sm1];
            const T(*P)[34] = sm.a[s0];
            const T(*Tp)[34] = sm.a[sp1];
            const T pp = P[fy][fx];
            const T q = c.q, idx = c.idx;
            const T Jxp = k_fluxn<T>((P[fy][fx + 1] - pp) * idx,
                                     q * (P[fy + 1][fx] + P[fy + 1][fx + 1] - P[fy - 1][fx] - P[fy - 1][fx + 1]),
                                     q * (Tp[fy][fx] + Tp[fy][fx + 1] - B[fy][fx] - B[fy][fx + 1]), c);
            const T Jxm = k_fluxn<T>((pp - P[fy][fx - 1]) * idx,
                                     q * (P[fy + 1][fx] + P[fy + 1][fx - 1] - P[fy - 1][fx] - P[fy - 1][fx - 1]),
                                     q * (Tp[fy][fx] + Tp[fy][fx - 1] - B[fy][fx] - B[fy][fx - 1]), c);
            const T Jyp = k_fluxn<T>((P[fy + 1][fx] - pp) * idx,
                                     q * (P[fy][fx + 1] + P[fy + 1][fx + 1] - P[fy][fx - 1] - P[fy + 1][fx - 1]),
                                     q * (Tp[fy][fx] + Tp[fy + 1][fx] - B[fy][fx] - B[fy + 1][fx]), c);
            const T Jym = k_fluxn<T>((pp - P[fy - 1][fx]) * idx,
                                     q * (P[fy][fx + 1] + P[fy - 1][fx + 1] - P[fy][fx - 1] - P[fy - 1][fx - 1]),
                                     q * (Tp[fy][fx] + Tp[fy - 1][fx] - B[fy][fx] - B[fy - 1][fx]), c);
            const T Jzp = k_fluxn<T>((Tp[fy][fx] - pp) * idx,
                                     q * (P[fy][fx + 1] + Tp[fy][fx + 1] - P[fy][fx - 1] - Tp[fy][fx - 1]),
                                     q * (P[fy + 1][fx] + Tp[fy + 1][fx] - P[fy - 1][fx] - Tp[fy - 1][fx]), c);
            const T Jzm = k_fluxn<T>((pp - B[fy][fx]) * idx,
                                     q * (P[fy][fx + 1] + B[fy][fx + 1] - P[fy][fx - 1] - B[fy][fx - 1]),
                                     q * (P[fy + 1][fx] + B[fy + 1][fx] - P[fy - 1][fx] - B[fy - 1][fx]), c);
            const T divJ = (Jxp - Jxm + Jyp - Jym + Jzp - Jzm) * idx;
            const T g1 = c.h * (P[fy][fx + 1] - P[fy][fx - 1]);
            const T g2 = c.h * (P[fy + 1][fx] - P[fy - 1][fx]);
            const T g3 = c.h * (Tp[fy][fx] - B[fy][fx]);
            const T gm = g1 * g1 + g2 * g2 + g3 * g3;
            T as2;
            if (gm > (T)1.e-20) {
                const T a = g1 * g1, b = g2 * g2, e = g3 * g3;
                const T s4 = (a * a + b * b + e * e) / (gm * gm);
                const T t = c.om3 + c.e4 * s4;
                as2 = t * t;
            } else {
                as2 = c.om3 * c.om3;
            }
            const long long id = col + (long long)z * d.plane;
            const T om = (T)1 - pp * pp;
            const T r = (T)k_ruido(x + 1, y + 1, z + 1, d.it);
            dphi[id] = (divJ + pp - (pp * pp) * pp - c.lambda * (om * om) * uc) / as2 +
                       c.Fnoise * r * ((T)1 - pp * pp) / c.sqdt;
        }
        cp_async_wait_all();
        __syncthreads();
        const int t = sm1;
        sm1 = s0;
        s0 = sp1;
        sp1 = sfree;
        sfree = t;
    }
}

// flux of U through one face of the own cell (karma3d.f90:219-264): g = the
// face gradient (gn its normal component), nb = phi across the face, du =
// the U difference in the face's orientation, un / dn = U and dphi across
template <typename T>
__device__ __forceinline__ T k_uflux(T g1, T g2, T g3, T gn, T pp, T nb, T du, T cl, T un, T dn, const KarmaK<T>& c)
{
    const T gm = sqrt(g1 * g1 + g2 * g2 + g3 * g3);
    const T qf = (T)0.25 * ((T)2 - pp - nb);
    const T cf = (T)0.5 * (cl + ((T)1 + c.omk * un) * dn);
    T F = c.D * qf * du * c.idx;
    if (gm > (T)1.e-10) F = F + c.at * cf * gn / gm;
    return F;
}

template <typename T, int TY>
struct KarmaSmemB {
    T p[4][TY + 2][34];
    T u[4][TY + 2][34];
    T dp[4][TY + 2][34];
};

// pass B: U_new and phi_new of karma3d.f90:212-287
template <typename T, int TY>
__global__ void __launch_bounds__(32 * TY) k_karma_solute(KarmaDesc d, const KarmaK<T> c, const T* __restrict__ phi,
                                                         const T* __restrict__ U, const T* __restrict__ dphi,
                                                         T* __restrict__ phi_out, T* __restrict__ U_out, int zchunk)
{
    __shared__ KarmaSmemB<T, TY> sm;
    const int x0 = blockIdx.x * 32, y0 = blockIdx.y * TY;
    const int zb = blockIdx.z * zchunk, ze = min(zb + zchunk, d.nz);
    const int tx = threadIdx.x, ty = threadIdx.y;
    const int x = x0 + tx, y = y0 + ty;
    const bool own = x < d.nx && y < d.ny;
    const int fx = tx + 1, fy = ty + 1;
    const long long col = (long long)x + (long long)y * d.px;
    int sm1 = 0, s0 = 1, sp1 = 2, sfree = 3;
    for (int k = -1; k <= 1; ++k) {
        const int sl = k + 1;
        k_load_plane<T, TY>(d, phi, zb + k, x0, y0, sm.p[sl]);
        k_load_plane<T, TY>(d, U, zb + k, x0, y0, sm.u[sl]);
        k_load_plane<T, TY>(d, dphi, zb + k, x0, y0, sm.dp[sl]);
    }
    cp_async_commit();
    cp_async_wait_all();
    __syncthreads();
    for (int z = zb; z < ze; ++z) {
        // plane z+2 lands in the free slots while plane z is computed
        if (z + 1 < ze) {
            k_load_plane<T, TY>(d, phi, z + 2, x0, y0, sm.p[sfree]);
            k_load_plane<T, TY>(d, U, z + 2, x0, y0, sm.u[sfree]);
            k_load_plane<T, TY>(d, dphi, z + 2, x0, y0, sm.dp[sfree]);
        }
        cp_async_commit();
        if (own) {
            const T(*B)[34] = sm.p[sm1];
            const T(*P)[34] = sm.p[s0];
            const T(*Tp)[34] = sm.p[sp1];
            const T(*UB)[34] = sm.u[sm1];
            const T(*UP)[34] = sm.u[s0];
            const T(*UT)[34] = sm.u[sp1];
            const T(*DB)[34] = sm.dp[sm1];
            const T(*DP)[34] = sm.dp[s0];
            const T(*DT)[34] = sm.dp[sp1];
            const T pp = P[fy][fx], uc = UP[fy][fx], dc = DP[fy][fx];
            const T q = c.q, idx = c.idx;
            const T cl = ((T)1 + c.omk * uc) * dc;   // the own cell's term of cf
            T g1, g2, g3;
            // x+
            g1 = (P[fy][fx + 1] - pp) * idx;
            g2 = q * (P[fy + 1][fx] + P[fy + 1][fx + 1] - P[fy - 1][fx] - P[fy - 1][fx + 1]);
            g3 = q * (Tp[fy][fx] + Tp[fy][fx + 1] - B[fy][fx] - B[fy][fx + 1]);
            const T Fxp = k_uflux<T>(g1, g2, g3, g1, pp, P[fy][fx + 1], UP[fy][fx + 1] - uc, cl, UP[fy][fx + 1],
                                     DP[fy][fx + 1], c);
            // x-
            g1 = (pp - P[fy][fx - 1]) * idx;
            g2 = q * (P[fy + 1][fx] + P[fy + 1][fx - 1] - P[fy - 1][fx] - P[fy - 1][fx - 1]);
            g3 = q * (Tp[fy][fx] + Tp[fy][fx - 1] - B[fy][fx] - B[fy][fx - 1]);
            const T Fxm = k_uflux<T>(g1, g2, g3, g1, pp, P[fy][fx - 1], uc - UP[fy][fx - 1], cl, UP[fy][fx - 1],
                                     DP[fy][fx - 1], c);
            // y+
            g2 = (P[fy + 1][fx] - pp) * idx;
            g1 = q * (P[fy][fx + 1] + P[fy + 1][fx + 1] - P[fy][fx - 1] - P[fy + 1][fx - 1]);
            g3 = q * (Tp[fy][fx] + Tp[fy + 1][fx] - B[fy][fx] - B[fy + 1][fx]);
            const T Fyp = k_uflux<T>(g1, g2, g3, g2, pp, P[fy + 1][fx], UP[fy + 1][fx] - uc, cl, UP[fy + 1][fx],
                                     DP[fy + 1][fx], c);
            // y-
            g2 = (pp - P[fy - 1][fx]) * idx;
            g1 = q * (P[fy][fx + 1] + P[fy - 1][fx + 1] - P[fy][fx - 1] - P[fy - 1][fx - 1]);
            g3 = q * (Tp[fy][fx] + Tp[fy - 1][fx] - B[fy][fx] - B[fy - 1][fx]);
            const T Fym = k_uflux<T>(g1, g2, g3, g2, pp, P[fy - 1][fx], uc - UP[fy - 1][fx], cl, UP[fy - 1][fx],
                                     DP[fy - 1][fx], c);
            // z+
            g3 = (Tp[fy][fx] - pp) * idx;
            g1 = q * (P[fy][fx + 1] + Tp[fy][fx + 1] - P[fy][fx - 1] - Tp[fy][fx - 1]);
            g2 = q * (P[fy + 1][fx] + Tp[fy + 1][fx] - P[fy - 1][fx] - Tp[fy - 1][fx]);
            const T Fzp = k_uflux<T>(g1, g2, g3, g3, pp, Tp[fy][fx], UT[fy][fx] - uc, cl, UT[fy][fx], DT[fy][fx], c);
            // z-
            g3 = (pp - B[fy][fx]) * idx;
            g1 = q * (P[fy][fx + 1] + B[fy][fx + 1] - P[fy][fx - 1] - B[fy][fx - 1]);
            g2 = q * (P[fy + 1][fx] + B[fy + 1][fx] - P[fy - 1][fx] - B[fy - 1][fx]);
            const T Fzm = k_uflux<T>(g1, g2, g3, g3, pp, B[fy][fx], uc - UB[fy][fx], cl, UB[fy][fx], DB[fy][fx], c);

            const T Au = c.Ahalf1 - c.Ahalf2 * pp;
            const T rhsU = (Fxp - Fxm + Fyp - Fym + Fzp - Fzm) * idx + (T)0.5 * ((T)1 + c.omk * uc) * dc;
            const long long id = col + (long long)z * d.plane;
            U_out[id] = uc + c.dt * rhsU / Au;
            const T pn = pp + c.dt * dc;
            phi_out[id] = fmax((T)-1, fmin((T)1, pn));
        }
        cp_async_wait_all();
        __syncthreads();
        const int t = sm1;
        sm1 = s0;
        s0 = sp1;
        sp1 = sfree;
        sfree = t;
    }
}

// karma3d.f90:290-296 on the device: largest 1-based i with phi(i,1,1) > 0
// and with phi(i,i,i) > 0 (i up to the smallest extent); out[2] ints
template <typename T>
__global__ void k_karma_tip(KarmaDesc d, const T* __restrict__ phi, int* __restrict__ out)
{
    const int nd = min(d.nx, min(d.ny, d.nz));
    int tx = 0, td = 0;
    for (int i = threadIdx.x; i < d.nx; i += blockDim.x)
        if (phi[i] > (T)0) tx = max(tx, i + 1);
    for (int i = threadIdx.x; i < nd; i += blockDim.x)
        if (phi[(long long)i + (long long)i * d.px + (long long)i * d.plane] > (T)0) td = max(td, i + 1);
    for (int o = 16; o > 0; o >>= 1) {
        tx = max(tx, __shfl_xor_sync(0xffffffffu, tx, o));
        td = max(td, __shfl_xor_sync(0xffffffffu, td, o));
    }
    __shared__ int s[2][32];
    const int w = threadIdx.x / 32, l = threadIdx.x % 32;
    if (l == 0) {
        s[0][w] = tx;
        s[1][w] = td;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        int a = 0, b = 0;
        for (int q = 0; q < (int)(blockDim.x / 32); ++q) {
            a = max(a, s[0][q]);
            b = max(b, s[1][q]);
        }
        out[0] = a;
        out[1] = b;
    }
}

}  // namespace pf3d
