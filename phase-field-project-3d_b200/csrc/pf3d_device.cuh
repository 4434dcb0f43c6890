// pf3d_device.cuh -- device-side data model and per-cell arithmetic of the
// coupled explicit phase-field step (ileaof/phase-field-project-3D).
//
// Two arithmetic forms share this header:
//   double : the plain form.  Every operation follows the reference's Fortran
//            statement order (left-to-right association, x**2 = x*x,
//            x**4 = (x*x)*(x*x), divisions kept as IEEE divisions).  The
//            translation unit that instantiates it is compiled with
//            --fmad=false so no multiply-add is contracted, matching gfortran
//            on x86-64.
//   float  : storage and stencil arithmetic in FP32; the divisions by grid
//            constants become multiplications by host-rounded reciprocals,
//            the others products with the hardware's approximate
//            reciprocal, and log uses the hardware's approximate log2.
//            Its error is stated against the FP64 form, not bit parity.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>
#include "pf3d_pair.cuh"

namespace pf3d {

// ---------------------------------------------------------------------------
// Per-domain constants (set once) and per-step scalars.  All host-computed in
// FP64 with the reference's expressions, so FP64 kernels see the same bits the
// reference's loop-invariant scalars have.
// ---------------------------------------------------------------------------
struct DomainDesc {
    int nx, ny, nz;      // cells
    int px;              // row pitch in elements (>= nx)
    long long plane;     // px * ny
    double dx, dy, dz;
    double E0, W0, DE, K_aniso;   // K_aniso = 16*E0*DELTA_EPSLON (phase_body.inc:49)
    double AAA;                   // effective noise amplitude
    double Ke, D_liq, D_sol, dt;
    double dH_cp;                 // delta_H / cp_s (temp_body.inc:36)
    double Ddt;                   // D*DELTA_T of temp_body.inc:41 (D = 0 in the reference)
    double cxy, cyz, czx;         // 0.25/(dx*dy), 0.25/(dy*dz), 0.25/(dz*dx)
    double dx2, dy2, dz2;         // dx**2 ...
    double InvDX, InvDY, InvDZ;   // 1/(DX*DX) ... (concentracao_soluto.f90:9-11)
    double hx, hy, hz;            // 0.5/dx, 0.5/dy, 0.5/dz (fast-form gradients)
    double rdx2, rdy2, rdz2;      // 1/dx^2 ... (fast form)
    double AAA16;                 // AAA*16 (fast form)
    double omKe;                  // 1 - Ke (fast form)
    double dtIX, dtIY, dtIZ;      // DELTA_T*InvDX ... (fast form)
    int hq;                       // h_quintico
    int rt;                       // ruido_tipo
    int do_heat_lap;              // D != 0
    int pad_;
};

struct StepArgs {
    int it;              // noise step index (1-based step number)
    int pad_;
    double TP_heat;      // TP seen by temperatura (the previous step's TP)
    double TP;           // TP of this step's sweeps
    double M0dt;         // M0*DELTA_T (phase_body.inc:194)
    double RTV;          // R*TP/Vm (phase_body.inc:174)
    double omCs, omCl;   // 1-Cs_eq, 1-Cl_eq
    double Lc;           // log((1-Cs_eq)/(1-Cl_eq)) (fast form of phase_body.inc:174)
};

// ---------------------------------------------------------------------------
// Noise: variaveis.f90:73-111.  Integer hash of 1-based (i,j,k,it,salt).
// ---------------------------------------------------------------------------
__host__ __device__ __forceinline__ uint64_t hash63(int i, int j, int k, int it, int salt)
{
    uint64_t h = (uint64_t)(int64_t)i * 2654435761ull + (uint64_t)(int64_t)j * 2246822519ull +
                 (uint64_t)(int64_t)k * 3266489917ull + (uint64_t)(int64_t)it * 668265263ull +
                 (uint64_t)(int64_t)salt * 374761393ull + 1ull;
    h ^= h >> 33;
    h *= 0xff51afd7ed558ccdull;
    h ^= h >> 33;
    h *= 0xc4ceb9fe1a85ec53ull;
    h ^= h >> 33;
    return h & 0x7fffffffffffffffull;
}

// pseudo_random as FP64: the 63-bit integer rounded to double, then divided
// by real(MASK63,8) = 2^63 (exact).
__host__ __device__ __forceinline__ double ran64(uint64_t m)
{
    return (double)(long long)m * 0x1p-63;
}

__device__ __forceinline__ double ruido_suave64(int i, int j, int k, int it)
{
    const int LR = 6, TR = 20;
    int i0 = i / LR, j0 = j / LR, k0 = k / LR, tb = it / TR;
    double fx = (double)(i % LR) / (double)LR;
    double fy = (double)(j % LR) / (double)LR;
    double fz = (double)(k % LR) / (double)LR;
    double p000 = ran64(hash63(i0, j0, k0, tb, 3)), p100 = ran64(hash63(i0 + 1, j0, k0, tb, 3));
    double p010 = ran64(hash63(i0, j0 + 1, k0, tb, 3)), p110 = ran64(hash63(i0 + 1, j0 + 1, k0, tb, 3));
    double p001 = ran64(hash63(i0, j0, k0 + 1, tb, 3)), p101 = ran64(hash63(i0 + 1, j0, k0 + 1, tb, 3));
    double p011 = ran64(hash63(i0, j0 + 1, k0 + 1, tb, 3)), p111 = ran64(hash63(i0 + 1, j0 + 1, k0 + 1, tb, 3));
    double a = __dadd_rn(__dmul_rn(1.0 - fx, p000), __dmul_rn(fx, p100));
    double b = __dadd_rn(__dmul_rn(1.0 - fx, p010), __dmul_rn(fx, p110));
    double c = __dadd_rn(__dmul_rn(1.0 - fx, p001), __dmul_rn(fx, p101));
    double d = __dadd_rn(__dmul_rn(1.0 - fx, p011), __dmul_rn(fx, p111));
    double lo = __dadd_rn(__dmul_rn(1.0 - fy, a), __dmul_rn(fy, b));
    double hi = __dadd_rn(__dmul_rn(1.0 - fy, c), __dmul_rn(fy, d));
    return __dadd_rn(__dmul_rn(1.0 - fz, lo), __dmul_rn(fz, hi));
}

// The hash input of variaveis.f90:82-83 without the k term; adding k*C for
// each plane gives the input of cell (i, j, k) (wrapping 64-bit arithmetic).
__host__ __device__ __forceinline__ uint64_t hash_base(int i, int j, int it, int salt)
{
    return (uint64_t)(int64_t)i * 2654435761ull + (uint64_t)(int64_t)j * 2246822519ull +
           (uint64_t)(int64_t)it * 668265263ull + (uint64_t)(int64_t)salt * 374761393ull + 1ull;
}
constexpr uint64_t kHashK = 3266489917ull;

// fmix64 rounds of variaveis.f90:84-88 on a precomputed input
__host__ __device__ __forceinline__ uint64_t hash63_mix(uint64_t h)
{
    h ^= h >> 33;
    h *= 0xff51afd7ed558ccdull;
    h ^= h >> 33;
    h *= 0xc4ceb9fe1a85ec53ull;
    h ^= h >> 33;
    return h & 0x7fffffffffffffffull;
}

// The REAL(4) `ran` of phase_body.inc:181-185 (identical for both precisions).
__device__ __forceinline__ float phase_ran(int rt, int i, int j, int k, int it)
{
    double r = (rt == 2) ? ruido_suave64(i, j, k, it) : ran64(hash63(i, j, k, it, 1));
    return __double2float_rn(r);
}

// ---------------------------------------------------------------------------
// ---------------------------------------------------------------------------
// FP64 reciprocal of the fast form: the hardware approximation y0 refined in
// one step of third order.  With e = 1 - b y0 (exact in an fma),
// 1/b = y0/(1 - e) = y0 (1 + e + e^2 + e^3 + ...), so y = y0 + y0 (e + e^2)
// leaves out y0 e^3: |e| stays below 2^-19.9 (measured on B200 over 4 M
// operands from 1e-260 to 1e260), so that is below 2^-59 relative and the
// result is within one ulp of the correctly rounded 1/b (equal to it on
// 99.97 % of those operands; two Newton-Raphson steps y <- y + y (1 - b y),
// Markstein, IBM J. Res. Dev. 34(1), 1990, were equal on all of them but take
// four fmas instead of three).  Tests hold the fused FP64 form to 1e-12 of
// the IEEE-division reference form.
__device__ __forceinline__ double rcp_nr(double b)
{
    double y;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(b));
    const double e = __fma_rn(-b, y, 1.0);
    return __fma_rn(y, __fma_rn(e, e, e), y);
}

// Natural logarithm in FP64 for the fast form -- this library's own, written
// from the mathematics, not the CUDA library's: x = 2^k m with m in
// [sqrt(1/2), sqrt(2)), f = m - 1 (exact, Sterbenz), and
//     log x = k ln2 + 2 atanh(s) = k ln2 + 2s + 2s z P(z),
//     s = f/(2 + f),  |s| <= 0.17158,  z = s^2 <= 0.029438,
// where P(z) = (atanh(sqrt z)/sqrt z - 1)/z = 1/3 + z/5 + z^2/7 + ... (the
// Taylor series of atanh) is replaced by its degree-6 Chebyshev interpolant
// on [0, 0.029441] (Lanczos economization; coefficients and their error from
// log_coeffs.py: |P6 - P| <= 1.6e-16, i.e. below 5e-18 of log x after the
// factor 2s z).  The reduction works on the high word: adding
// 0x3ff00000 - 0x3fe6a09e (0x3fe6a09e = high word of sqrt(1/2)) carries into
// the exponent field exactly when the mantissa is at or above sqrt(2)'s, so k
// and m come out of integer operations with no compare.  s is carried as
// s + sl: the rounding error of 2 + f (Fast2Sum, Dekker 1971) and the residual
// of the quotient (one Newton correction, Markstein 1990) go into sl, which
// joins the low-order sum.  ln2 is split into a head with the low 32 mantissa
// bits zero, so k ln2_hi is exact, and a tail.  Within 1 ulp of log x
// (pf_math_log, tests).  Zero, negative, subnormal, infinite and NaN
// arguments (one unsigned compare on the high word) call the CUDA library's
// log out of line, so nothing of it is evaluated on the common path.
static __device__ __noinline__ double log_special(double x) { return log(x); }
__device__ __forceinline__ double pf_log(double x)
{
    int hi = __double2hiint(x);
    const int lo = __double2loint(x);
    if ((unsigned)(hi - 0x00100000) >= 0x7fe00000u) return log_special(x);
    hi += 0x3ff00000 - 0x3fe6a09e;
    const int k = (hi >> 20) - 0x3ff;
    const double m = __hiloint2double((hi & 0x000fffff) + 0x3fe6a09e, lo);   // [sqrt(1/2), sqrt(2))
    const double f = m - 1.0;                      // exact
    const double d = 2.0 + f;
    const double derr = f - (d - 2.0);             // 2 + f = d + derr exactly
    const double rc = rcp_nr(d);
    const double s = f * rc;
    const double e = __fma_rn(-s, derr, __fma_rn(-s, d, f));   // f - s (d + derr)
    const double sl = e * rc;                      // f/(2 + f) = s + sl
    const double z = s * s;
    double p = 0.07308292712444311;
    p = __fma_rn(p, z, 0.07665855309105386);
    p = __fma_rn(p, z, 0.09091444727837474);
    p = __fma_rn(p, z, 0.11111105565129939);
    p = __fma_rn(p, z, 0.14285714313001635);
    p = __fma_rn(p, z, 0.19999999999949722);
    p = __fma_rn(p, z, 0.3333333333333335);
    const double t = 2.0 * s;                      // exact
    const double lo_sum = __fma_rn(t * z, p, sl + sl);   // 2 atanh(s) - t
    const double kd = (double)k;
    const double ln2_hi = 0.6931467056274414;      // 0x3fe62e4200000000
    const double ln2_lo = 4.7493250390316726e-07;  // ln2 - ln2_hi
    return __fma_rn(kd, ln2_hi, __fma_rn(kd, ln2_lo, lo_sum) + t);
}

// Arithmetic of the fast form (the reference form uses plain / and log).
template <typename T> struct Ar;
template <> struct Ar<double> {
    static __device__ __forceinline__ double rcp(double x) { return rcp_nr(x); }
    static __device__ __forceinline__ double div(double a, double b) { return a * rcp_nr(b); }
    static __device__ __forceinline__ double lg(double x) { return pf_log(x); }
};
// FP32 fast form: the hardware's approximate reciprocal and base-2
// logarithm (PTX rcp.approx.ftz.f32, lg2.approx.ftz.f32), a quotient as the
// product with the reciprocal and ln x = log2(x) ln 2.  The lane pairs take
// the same scalar steps lane by lane, so every lane of a pair gets the bits
// of the one-cell form.
__device__ __forceinline__ float rcp_ap(float x)
{
    float y;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
__device__ __forceinline__ float lg2_ap(float x)
{
    float y;
    asm("lg2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
constexpr float kLn2f = 0.693147180559945309f;   // ln 2 rounded to float
template <> struct Ar<float> {
    static __device__ __forceinline__ float rcp(float x) { return rcp_ap(x); }
    static __device__ __forceinline__ float div(float a, float b) { return __fmul_rn(a, rcp_ap(b)); }
    static __device__ __forceinline__ float lg(float x) { return __fmul_rn(lg2_ap(x), kLn2f); }
};

// ---- lane-generic helpers: scalar float / double, and the lane pairs F2 / D2
// (two cells per thread, pf3d_pair.cuh) with the same per-lane operations ----
template <typename T> struct IsF64 { static constexpr bool value = false; };
template <> struct IsF64<double> { static constexpr bool value = true; };
template <> struct IsF64<D2> { static constexpr bool value = true; };

__device__ __forceinline__ float vabs(float x) { return fabsf(x); }
__device__ __forceinline__ double vabs(double x) { return fabs(x); }
__device__ __forceinline__ F2 vabs(F2 x) { F2 r; r.v = x.v & 0x7fffffff7fffffffull; return r; }
__device__ __forceinline__ D2 vabs(D2 x) { return D2(fabs(x.a), fabs(x.b)); }
__device__ __forceinline__ float vmax(float a, float b) { return fmaxf(a, b); }
__device__ __forceinline__ double vmax(double a, double b) { return fmax(a, b); }
__device__ __forceinline__ F2 vmax(F2 a, F2 b) { return F2(fmaxf(a.x(), b.x()), fmaxf(a.y(), b.y())); }
__device__ __forceinline__ D2 vmax(D2 a, D2 b) { return D2(fmax(a.a, b.a), fmax(a.b, b.b)); }
// (a < b) ? x : y, (a > b) ? x : y and (a <= b) ? x : y, lane by lane
template <typename T> __device__ __forceinline__ T sel_lt(T a, T b, T x, T y) { return (a < b) ? x : y; }
template <typename T> __device__ __forceinline__ T sel_gt(T a, T b, T x, T y) { return (a > b) ? x : y; }
template <typename T> __device__ __forceinline__ T sel_le(T a, T b, T x, T y) { return (a <= b) ? x : y; }
#define PF3D_PAIR_SEL(NAME, OP)                                                                          \
    template <> __device__ __forceinline__ F2 NAME<F2>(F2 a, F2 b, F2 x, F2 y)                          \
    {                                                                                                    \
        return F2((a.x() OP b.x()) ? x.x() : y.x(), (a.y() OP b.y()) ? x.y() : y.y());                  \
    }                                                                                                    \
    template <> __device__ __forceinline__ D2 NAME<D2>(D2 a, D2 b, D2 x, D2 y)                          \
    {                                                                                                    \
        return D2((a.a OP b.a) ? x.a : y.a, (a.b OP b.b) ? x.b : y.b);                                  \
    }
PF3D_PAIR_SEL(sel_lt, <)
PF3D_PAIR_SEL(sel_gt, >)
PF3D_PAIR_SEL(sel_le, <=)
#undef PF3D_PAIR_SEL

template <> struct Ar<F2> {
    static __device__ __forceinline__ F2 rcp(F2 x) { return F2(rcp_ap(x.x()), rcp_ap(x.y())); }
    static __device__ __forceinline__ F2 div(F2 a, F2 b)
    {
        return F2(Ar<float>::div(a.x(), b.x()), Ar<float>::div(a.y(), b.y()));
    }
    static __device__ __forceinline__ F2 lg(F2 x) { return F2(Ar<float>::lg(x.x()), Ar<float>::lg(x.y())); }
};
template <> struct Ar<D2> {
    static __device__ __forceinline__ D2 rcp(D2 x) { return D2(rcp_nr(x.a), rcp_nr(x.b)); }
    static __device__ __forceinline__ D2 div(D2 a, D2 b) { return D2(a.a * rcp_nr(b.a), a.b * rcp_nr(b.b)); }
    static __device__ __forceinline__ D2 lg(D2 x) { return D2(pf_log(x.a), pf_log(x.b)); }
};

// Explicit multiply-add.  Every translation unit is built without automatic
// contraction, so the same source gives the same bits in every kernel that
// inlines it (single domain, batch, any tile shape); the fast form asks for
// its multiply-adds here.
__device__ __forceinline__ double fmadd(double a, double b, double c) { return __fma_rn(a, b, c); }
__device__ __forceinline__ float fmadd(float a, float b, float c) { return __fmaf_rn(a, b, c); }

// Loop-invariant constants in the stencil type.  The fused passes receive
// them built on the host, by value, so they are constant-bank operands.
template <typename T>
struct KC {
    T dx, dy, dz, E0, W0, DE, K, AAA, Ke, D_liq, D_sol, dt, dH_cp, Ddt;
    T cxy, cyz, czx, dx2, dy2, dz2, InvDX, InvDY, InvDZ;
    T hx, hy, hz, rdx2, rdy2, rdz2;
    T TP, TP_heat, M0dt, RTV, omCs, omCl;
    T AAA16, omKe, dtIX, dtIY, dtIZ, Lc;
    int hq, rt, it, lap;
    __host__ __device__ __forceinline__ void load(const DomainDesc& d, const StepArgs& s)
    {
        dx = (T)d.dx; dy = (T)d.dy; dz = (T)d.dz;
        E0 = (T)d.E0; W0 = (T)d.W0; DE = (T)d.DE; K = (T)d.K_aniso; AAA = (T)d.AAA;
        Ke = (T)d.Ke; D_liq = (T)d.D_liq; D_sol = (T)d.D_sol; dt = (T)d.dt;
        dH_cp = (T)d.dH_cp; Ddt = (T)d.Ddt;
        cxy = (T)d.cxy; cyz = (T)d.cyz; czx = (T)d.czx;
        dx2 = (T)d.dx2; dy2 = (T)d.dy2; dz2 = (T)d.dz2;
        InvDX = (T)d.InvDX; InvDY = (T)d.InvDY; InvDZ = (T)d.InvDZ;
        hx = (T)d.hx; hy = (T)d.hy; hz = (T)d.hz;
        rdx2 = (T)d.rdx2; rdy2 = (T)d.rdy2; rdz2 = (T)d.rdz2;
        TP = (T)s.TP; TP_heat = (T)s.TP_heat; M0dt = (T)s.M0dt; RTV = (T)s.RTV;
        omCs = (T)s.omCs; omCl = (T)s.omCl;
        AAA16 = (T)d.AAA16; omKe = (T)d.omKe; dtIX = (T)d.dtIX; dtIY = (T)d.dtIY; dtIZ = (T)d.dtIZ;
        Lc = (T)s.Lc;
        hq = d.hq; rt = d.rt; it = s.it; lap = d.do_heat_lap;
    }
};

// ---------------------------------------------------------------------------
// Per-cell arithmetic.  FAST = false is the reference form (statement order of
// the Fortran, IEEE divisions; FP64 kernels built without contraction).
// FAST = true is the fast form used by the fused passes: the same equations,
// divisions by grid constants replaced by products with host-rounded
// reciprocals, one reciprocal per shared denominator, the cross terms grouped
// by node, and the log argument of phase_body.inc:174 reduced to
// (den - c)/(den - Ke c) plus a per-step constant.  In FP64 it stays within
// 1e-12 of the reference form after thousands of steps (tests).
// ---------------------------------------------------------------------------

// node-centred central gradient component: (a-b)*0.5d0/dx (phase_body.inc:55-122)
template <typename T, bool FAST>
__device__ __forceinline__ T grad(T a, T b, T d, T half_inv)
{
    if constexpr (!FAST) return (a - b) * (T)0.5 / d;
    else return (a - b) * half_inv;
}

// Anisotropy quantities at one node from its gradient (phase_body.inc:59-64):
// eps and the three cross coefficients exy, eyz, ezx.
template <typename T>
struct Node { T eps, exy, eyz, ezx; };

template <typename T, bool FAST>
__device__ __forceinline__ Node<T> aniso_node(T gx, T gy, T gz, const KC<T>& c)
{
    Node<T> n;
    T gx2 = gx * gx, gy2 = gy * gy, gz2 = gz * gz;
    if constexpr (!FAST) {
        T Q = gx2 + gy2 + gz2 + (T)1e-23;
        T S4 = gx2 * gx2 + gy2 * gy2 + gz2 * gz2;
        T Q2 = Q * Q;
        n.eps = c.E0 * ((T)1 + c.DE * ((T)4 * S4 / Q2 - (T)3));
        T Ke_ = c.K * n.eps;
        n.exy = Ke_ * gx * gy * (gx2 - gy2) / Q2;
        n.eyz = Ke_ * gy * gz * (gy2 - gz2) / Q2;
        n.ezx = Ke_ * gz * gx * (gz2 - gx2) / Q2;
    } else if constexpr (IsF64<T>::value) {
        T Q = fmadd(gx, gx, fmadd(gy, gy, fmadd(gz, gz, (T)1e-23)));
        T S4 = fmadd(gx2, gx2, fmadd(gy2, gy2, gz2 * gz2));
        T rq = Ar<T>::rcp(Q * Q);
        n.eps = c.E0 * fmadd(c.DE, fmadd((T)4 * S4, rq, (T)-3), (T)1);
        T f = c.K * n.eps * rq;
        n.exy = f * gx * gy * (gx2 - gy2);
        n.eyz = f * gy * gz * (gy2 - gz2);
        n.ezx = f * gz * gx * (gz2 - gx2);
    } else {
        // FP32: Q^2 >= 1e-46 is below the FP32 range, so evaluate the
        // scale-invariant form with g normalised by its largest component m:
        // 4 S4/Q^2 and e_ab are unchanged, and `small` becomes 1e-23/m^2.
        // Clamping m at 1e-15 keeps it branch-free: for smaller gradients the
        // normalised components stay <= 1e-0 and small/m^2 >= 1e7, so the
        // ratio and the cross terms vanish as in the reference.
        const T m = vmax(vmax(vabs(gx), vabs(gy)), vmax(vabs(gz), (T)1e-15));
        const T im = Ar<T>::rcp(m);
        const T ux = gx * im, uy = gy * im, uz = gz * im;
        const T ux2 = ux * ux, uy2 = uy * uy, uz2 = uz * uz;
        const T Q = fmadd(ux, ux, fmadd(uy, uy, fmadd(uz, uz, (T)1e-23 * im * im)));
        const T S4 = fmadd(ux2, ux2, fmadd(uy2, uy2, uz2 * uz2));
        const T rq = Ar<T>::rcp(Q * Q);
        n.eps = c.E0 * fmadd(c.DE, fmadd((T)4 * S4, rq, (T)-3), (T)1);
        const T f = c.K * n.eps * rq;
        // every product that feeds a sum is an explicit multiply-add in the
        // FP32 form: nothing is left for a compiler to contract, so the lane
        // pairs may issue packed f32x2 products and sums (pf3d_pair.cuh)
        n.exy = f * ux * uy * fmadd(ux, ux, -uy2);
        n.eyz = f * uy * uz * fmadd(uy, uy, -uz2);
        n.ezx = f * uz * ux * fmadd(uz, uz, -ux2);
    }
    (void)gx2; (void)gy2; (void)gz2;
    return n;
}

// The 19 phase values of phase_body.inc:14-41.
template <typename T>
struct Nbr {
    T PP, PN, PS, PE, PW, PT, PB;
    T PNE, PSE, PNW, PSW, PNT, PNB, PST, PSB, PET, PEB, PWT, PWB;
};

// phase_body.inc:133-198 given the stencil values and the six node
// quantities.  Returns PPNEW (unclamped).  SQ (fast form only): the nodes'
// eps member already holds eps*eps, squared once per node instead of once
// per use (the same product, so the same bits).
template <typename T, bool FAST, bool SQ = false>
__device__ __forceinline__ T phase_ppnew(const Nbr<T>& p, const Node<T>& E, const Node<T>& W, const Node<T>& N,
                                          const Node<T>& S, const Node<T>& Tt, const Node<T>& B, T CPP,
                                          T ran, const KC<T>& c)
{
    static_assert(FAST || !SQ, "squared node values are a fast-form input");
    auto e2 = [](const Node<T>& n) -> T {
        if constexpr (SQ) return n.eps;
        else return n.eps * n.eps;
    };
    const T PP = p.PP;
    const T one = (T)1, two = (T)2;
    if constexpr (!FAST) {
        T AA = (E.eps * E.eps * (p.PE - PP) + W.eps * W.eps * (p.PW - PP)) / c.dx2 +
               (N.eps * N.eps * (p.PN - PP) + S.eps * S.eps * (p.PS - PP)) / c.dy2 +
               (Tt.eps * Tt.eps * (p.PT - PP) + B.eps * B.eps * (p.PB - PP)) / c.dz2;
        T Cxy = c.cxy * (p.PNE * (-N.exy - (-E.exy)) + p.PSE * (-E.exy - (-S.exy)) + p.PNW * (-W.exy - (-N.exy)) +
                         p.PSW * (-S.exy - (-W.exy))) +
                p.PN * c.cxy * (-W.exy - (-E.exy)) + p.PS * c.cxy * (-E.exy - (-W.exy)) +
                p.PE * c.cxy * (-N.exy - (-S.exy)) + p.PW * c.cxy * (-S.exy - (-N.exy));
        T Cyz = c.cyz * (p.PNT * (-Tt.eyz - (-N.eyz)) + p.PNB * (-N.eyz - (-B.eyz)) + p.PST * (-S.eyz - (-Tt.eyz)) +
                         p.PSB * (-B.eyz - (-S.eyz))) +
                p.PT * c.cyz * (-S.eyz - (-N.eyz)) + p.PB * c.cyz * (-N.eyz - (-S.eyz)) +
                p.PN * c.cyz * (-Tt.eyz - (-B.eyz)) + p.PS * c.cyz * (-B.eyz - (-Tt.eyz));
        T Czx = c.czx * (p.PET * (-E.ezx - (-Tt.ezx)) + p.PWT * (-Tt.ezx - (-W.ezx)) + p.PEB * (-B.ezx - (-E.ezx)) +
                         p.PWB * (-W.ezx - (-B.ezx))) +
                p.PE * c.czx * (-B.ezx - (-Tt.ezx)) + p.PW * c.czx * (-Tt.ezx - (-B.ezx)) +
                p.PT * c.czx * (-E.ezx - (-W.ezx)) + p.PB * c.czx * (-W.ezx - (-E.ezx));
        AA = AA + Cxy + Cyz + Czx;
        T g_linha = two * PP * (one - PP) * (one - PP) - two * PP * PP * (one - PP);
        T h_linha, h;
        if (c.hq == 1) {
            h_linha = (T)30 * PP * PP * (one - PP) * (one - PP);
            h = PP * PP * PP * ((T)10 - (T)15 * PP + (T)6 * PP * PP);
        } else {
            h_linha = two * PP * ((T)3 - two * PP) - two * PP * PP;
            h = PP * PP * ((T)3 - two * PP);
        }
        T den = c.Ke * h + (one - h);
        T CLP = CPP / den;
        T CSP = c.Ke * CPP / den;
        T GG = (-(c.W0 * g_linha)) + c.RTV * h_linha * log(fabs(c.omCs * (one - CLP) / (c.omCl * (one - CSP))));
        T pp2 = PP * PP, q = one - PP;
        T ruidos;
        if (c.rt == 0)
            ruidos = (T)ran * c.AAA * (T)16 * pp2 * (q * q);
        else
            ruidos = (two * (T)ran - one) * c.AAA * (T)16 * pp2 * (q * q);
        return PP + c.M0dt * (AA + GG) + ruidos;
    } else {
        T ax = fmadd(e2(E), p.PE - PP, e2(W) * (p.PW - PP));
        T ay = fmadd(e2(N), p.PN - PP, e2(S) * (p.PS - PP));
        T az = fmadd(e2(Tt), p.PT - PP, e2(B) * (p.PB - PP));
        T AA = fmadd(ax, c.rdx2, fmadd(ay, c.rdy2, az * c.rdz2));
        // cross terms of phase_body.inc:137-147 grouped by node.  The axis
        // differences occur with both signs; b - a is exactly -(a - b), so
        // each is formed once and a + (b - c) is written a - (c - b): the
        // same values, three subtractions instead of twelve.
        const T dNS = p.PN - p.PS, dEW = p.PE - p.PW, dTB = p.PT - p.PB;
        T Cxy = fmadd(E.exy, (p.PNE - p.PSE) + dNS,
                      fmadd(N.exy, (p.PNW - p.PNE) - dEW,
                            fmadd(W.exy, (p.PSW - p.PNW) - dNS, S.exy * ((p.PSE - p.PSW) + dEW))));
        T Cyz = fmadd(N.eyz, (p.PNT - p.PNB) + dTB,
                      fmadd(Tt.eyz, (p.PST - p.PNT) - dNS,
                            fmadd(S.eyz, (p.PSB - p.PST) - dTB, B.eyz * ((p.PNB - p.PSB) + dNS))));
        T Czx = fmadd(Tt.ezx, (p.PET - p.PWT) + dEW,
                      fmadd(W.ezx, (p.PWT - p.PWB) + dTB,
                            fmadd(B.ezx, (p.PWB - p.PEB) - dEW, E.ezx * ((p.PEB - p.PET) - dTB))));
        AA = fmadd(c.cxy, Cxy, fmadd(c.cyz, Cyz, fmadd(c.czx, Czx, AA)));
        const T q = one - PP;
        T g_linha, h_linha, h;
        if constexpr (IsF64<T>::value) {
            g_linha = two * PP * q * (one - two * PP);
            if (c.hq == 1) {
                h_linha = (T)30 * PP * PP * q * q;
                h = PP * PP * PP * ((T)10 - (T)15 * PP + (T)6 * PP * PP);
            } else {
                h_linha = (T)6 * PP * q;
                h = PP * PP * ((T)3 - two * PP);
            }
        } else {
            // FP32: products feeding sums as explicit multiply-adds
            g_linha = two * PP * q * fmadd(-two, PP, one);
            if (c.hq == 1) {
                h_linha = (T)30 * PP * PP * q * q;
                h = PP * PP * PP * fmadd((T)6 * PP, PP, fmadd((T)-15, PP, (T)10));
            } else {
                h_linha = (T)6 * PP * q;
                h = PP * PP * fmadd(-two, PP, (T)3);
            }
        }
        T den = fmadd(-c.omKe, h, one);
        // (1-CLP)/(1-CSP) = (den - c)/(den - Ke c); the constant factor is in Lc
        T lg = Ar<T>::lg(vabs(Ar<T>::div(den - CPP, fmadd(-c.Ke, CPP, den)))) + c.Lc;
        T GG = fmadd(c.RTV * h_linha, lg, -(c.W0 * g_linha));
        T pp2q2 = PP * PP * q * q * c.AAA16;
        if constexpr (IsF64<T>::value) {
            T ruidos = (c.rt == 0) ? (T)ran * pp2q2 : fmadd(two, (T)ran, -one) * pp2q2;
            return fmadd(c.M0dt, AA + GG, PP + ruidos);
        } else {
            const T r = (c.rt == 0) ? (T)ran : fmadd(two, (T)ran, -one);
            return fmadd(c.M0dt, AA + GG, fmadd(r, pp2q2, PP));
        }
    }
}

// dmax1(0, dmin1(1, x)) (phase_body.inc:198)
template <typename T>
__device__ __forceinline__ T clamp01(T x)
{
    const T one = (T)1, zero = (T)0;
    T t = sel_lt(x, one, x, one);
    return sel_gt(t, zero, t, zero);
}

// h(phi) as written in conc_body.inc:42-58 (note the quintic form differs
// from phase_body.inc:161 in its association).
template <typename T>
__device__ __forceinline__ T h_conc(T P, int hq)
{
    if (hq == 1) return (P * P * P) * ((T)10 - ((T)15 * P) + ((T)6 * (P * P)));
    return P * P * ((T)3 - (T)2 * P);
}

// Per-point solute quantities of conc_body.inc: the Gamma bracket
// (1-h)CL(1-CL)+h CS(1-CS) and mu = log(CL/(1-CL)).
template <typename T>
struct SolNode { T br, mu; };

template <typename T, bool FAST>
__device__ __forceinline__ SolNode<T> sol_node(T P, T C, const KC<T>& c)
{
    const T one = (T)1;
    T h = h_conc(P, c.hq);
    SolNode<T> n;
    if constexpr (!FAST) {
        T den = (c.Ke * h) + (one - h);
        T CS = (c.Ke * C) / den;
        T CL = C / den;
        n.br = (one - h) * CL * (one - CL) + h * CS * (one - CS);
        n.mu = log(CL / (one - CL));
    } else if constexpr (IsF64<T>::value) {
        T den = fmadd(-c.omKe, h, one);
        T CL = C * Ar<T>::rcp(den);
        T CS = c.Ke * CL;
        n.br = fmadd((one - h) * CL, one - CL, h * CS * (one - CS));
        n.mu = Ar<T>::lg(Ar<T>::div(C, den - C));   // CL/(1-CL) = C/(den-C)
    } else {
        // FP32: h = a*b with 1-h, 1-CL and 1-CS as explicit multiply-adds
        T a, b;
        if (c.hq == 1) {
            a = P * P * P;
            b = fmadd((T)6 * P, P, fmadd((T)-15, P, (T)10));
        } else {
            a = P * P;
            b = fmadd((T)-2, P, (T)3);
        }
        const T hf = a * b, omh = fmadd(-a, b, one);
        const T den = fmadd(-c.omKe, hf, one);
        const T rd = Ar<T>::rcp(den);
        const T CL = C * rd, CS = c.Ke * CL;
        n.br = fmadd(omh * CL, fmadd(-C, rd, one), hf * CS * fmadd(-c.Ke, CL, one));
        n.mu = Ar<T>::lg(Ar<T>::div(C, den - C));
        (void)h;
    }
    return n;
}

// conc_body.inc:92-149 given the seven per-point quantities.
template <typename T, bool FAST>
__device__ __forceinline__ T conc_new(T PP, T CPP, const SolNode<T>& P, const SolNode<T>& E, const SolNode<T>& W,
                                      const SolNode<T>& N, const SolNode<T>& S, const SolNode<T>& Tt,
                                      const SolNode<T>& B, const KC<T>& c)
{
    const T Dc = sel_le(PP, (T)0.95, c.D_liq, c.D_sol);
    const T two = (T)2;
    if constexpr (!FAST) {
        T GP = Dc * P.br, GS = Dc * S.br, GN = Dc * N.br, GW = Dc * W.br, GE = Dc * E.br, GT = Dc * Tt.br,
          GB = Dc * B.br;
        T iP = (T)1 / GP;
        T Gs = two / (iP + (T)1 / GS);
        T Gn = two / ((T)1 / GN + iP);
        T Gw = two / (iP + (T)1 / GW);
        T Ge = two / ((T)1 / GE + iP);
        T Gt = two / ((T)1 / GT + iP);
        T Gb = two / (iP + (T)1 / GB);
        return (Ge * c.InvDX * (E.mu - P.mu) - Gw * c.InvDX * (P.mu - W.mu) + Gn * c.InvDY * (N.mu - P.mu) -
                Gs * c.InvDY * (P.mu - S.mu) + Gt * c.InvDZ * (Tt.mu - P.mu) - Gb * c.InvDZ * (P.mu - B.mu)) *
                   c.dt +
               CPP;
    } else {
        // 2/(1/(Dc a) + 1/(Dc b)) = 2 Dc a b / (a + b)
        const T Dab = two * Dc * P.br;
        auto hm = [&](T b) -> T {
            T sum = P.br + b;
            return sel_gt(sum, (T)0, Dab * b * Ar<T>::rcp(sum), (T)0);
        };
        T fx = fmadd(hm(E.br), E.mu - P.mu, -(hm(W.br) * (P.mu - W.mu)));
        T fy = fmadd(hm(N.br), N.mu - P.mu, -(hm(S.br) * (P.mu - S.mu)));
        T fz = fmadd(hm(Tt.br), Tt.mu - P.mu, -(hm(B.br) * (P.mu - B.mu)));
        return CPP + fmadd(c.dtIX, fx, fmadd(c.dtIY, fy, c.dtIZ * fz));
    }
}

// temp_body.inc:31-41 at an interior cell.  LAP = false compiles only the
// D = 0 form (for kernels that run on decks without heat diffusion).
template <typename T, bool LAP = true>
__device__ __forceinline__ T heat_new(T PP, T dpp, T TE, T TW, T TN, T TS, T TT, T TB, const KC<T>& c)
{
    T h_linha;
    if (c.hq == 1)
        h_linha = (T)30 * PP * PP * ((T)1 - PP) * ((T)1 - PP);
    else
        h_linha = (T)2 * PP * ((T)3 - (T)2 * PP) - (T)2 * PP * PP;
    T FONTE = c.dH_cp * h_linha * dpp;
    if (LAP && c.lap) {
        T TP = c.TP_heat;
        T lap = ((TE - (T)2 * TP + TW) / c.dx2) + ((TN - (T)2 * TP + TS) / c.dy2) + ((TT - (T)2 * TP + TB) / c.dz2);
        return c.Ddt * lap + FONTE + TP;
    }
    // D = 0: D*DELTA_T*(finite) is a signed zero and drops out exactly.
    return FONTE + c.TP_heat;
}

// ---------------------------------------------------------------------------
// Boundary decoration in closed form (0-based indices).
//   phase (equacao_campo_fase.f90:151-167, sequential in-place plane copies
//   y, x, z): phi_new(x,y,z) = U(f(x), f(y), f(z)) with f(0)=1, f(1)=2,
//   f(N-1)=N-2, f(N-2)=N-3, identity elsewhere (valid for N >= 5).
//   A source cell therefore writes its value to every x' with f(x') = x.
// ---------------------------------------------------------------------------
__host__ __device__ __forceinline__ int fmap(int x, int n)
{
    if (x == 0) return 1;
    if (x == 1) return 2;
    if (x == n - 1) return n - 2;
    if (x == n - 2) return n - 3;
    return x;
}

// Preimages of a source coordinate a in [1, N-2] under fmap: the contiguous
// range [*lo, *hi] (one to three cells).
__host__ __device__ __forceinline__ void fpre_range(int a, int n, int* lo, int* hi)
{
    *lo = (a == 1) ? 0 : (a == 2) ? 1 : (a == n - 2) ? n - 1 : a;
    *hi = (a == n - 2) ? n - 1 : (a == n - 3) ? n - 2 : (a == 1) ? 0 : a;
}

}  // namespace pf3d
