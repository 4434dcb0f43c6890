// pf3d_pair.cuh -- lane-pair arithmetic: two cells per thread.
//
// F2 holds two floats in one 64-bit register pair and maps add, sub, mul and
// fma onto Blackwell's packed FP32 instructions (add/sub/mul/fma.rn.f32x2,
// sm_100a): one instruction, the same IEEE operation on both cells.  ptxas
// contracts a packed mul.rn.f32x2 that feeds a packed add.rn.f32x2 into a
// packed fma even under --fmad=false (measured on B200: 15 % of random
// operands then round differently), so the FP32 fast form that runs on F2
// writes every product that feeds a sum as an explicit fmadd: nothing is left
// to contract, and the packed and the scalar kernels agree bit for bit
// (tests/test_paired_gpu.py).  D2 holds two doubles and does each operation
// once per lane.
#pragma once
#include <cstdint>
#include <cstring>

namespace pf3d {

struct F2 {
    unsigned long long v;
    __host__ __device__ __forceinline__ F2() {}
    // both lanes = a (host or device)
    static __host__ __device__ __forceinline__ F2 splat(float a)
    {
        unsigned u;
        memcpy(&u, &a, 4);
        F2 r;
        r.v = ((unsigned long long)u << 32) | u;
        return r;
    }
    __device__ __forceinline__ explicit F2(float a) { asm("mov.b64 %0, {%1, %1};" : "=l"(v) : "f"(a)); }
    __device__ __forceinline__ F2(float a, float b) { asm("mov.b64 %0, {%1, %2};" : "=l"(v) : "f"(a), "f"(b)); }
    __device__ __forceinline__ float x() const { float a; asm("{ .reg .f32 t; mov.b64 {%0, t}, %1; }" : "=f"(a) : "l"(v)); return a; }
    __device__ __forceinline__ float y() const { float b; asm("{ .reg .f32 t; mov.b64 {t, %0}, %1; }" : "=f"(b) : "l"(v)); return b; }
    __device__ __forceinline__ float lane(int i) const { return i ? y() : x(); }
};
__device__ __forceinline__ F2 operator+(F2 a, F2 b) { F2 r; asm("add.rn.f32x2 %0, %1, %2;" : "=l"(r.v) : "l"(a.v), "l"(b.v)); return r; }
__device__ __forceinline__ F2 operator-(F2 a, F2 b) { F2 r; asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(r.v) : "l"(a.v), "l"(b.v)); return r; }
__device__ __forceinline__ F2 operator*(F2 a, F2 b) { F2 r; asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(r.v) : "l"(a.v), "l"(b.v)); return r; }
// exact negation: flip both sign bits
__device__ __forceinline__ F2 operator-(F2 a) { F2 r; r.v = a.v ^ 0x8000000080000000ull; return r; }
__device__ __forceinline__ F2 fmadd(F2 a, F2 b, F2 c) { F2 r; asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(r.v) : "l"(a.v), "l"(b.v), "l"(c.v)); return r; }
__device__ __forceinline__ F2 operator/(F2 a, F2 b) { return F2(a.x() / b.x(), a.y() / b.y()); }

struct D2 {
    double a, b;
    __host__ __device__ __forceinline__ D2() {}
    static __host__ __device__ __forceinline__ D2 splat(double s)
    {
        D2 r;
        r.a = s;
        r.b = s;
        return r;
    }
    __device__ __forceinline__ explicit D2(double s) : a(s), b(s) {}
    __device__ __forceinline__ D2(double p, double q) : a(p), b(q) {}
    __device__ __forceinline__ double x() const { return a; }
    __device__ __forceinline__ double y() const { return b; }
    __device__ __forceinline__ double lane(int i) const { return i ? b : a; }
};
__device__ __forceinline__ D2 operator+(D2 p, D2 q) { return D2(__dadd_rn(p.a, q.a), __dadd_rn(p.b, q.b)); }
__device__ __forceinline__ D2 operator-(D2 p, D2 q) { return D2(__dsub_rn(p.a, q.a), __dsub_rn(p.b, q.b)); }
__device__ __forceinline__ D2 operator*(D2 p, D2 q) { return D2(__dmul_rn(p.a, q.a), __dmul_rn(p.b, q.b)); }
__device__ __forceinline__ D2 operator-(D2 p) { return D2(-p.a, -p.b); }
__device__ __forceinline__ D2 fmadd(D2 p, D2 q, D2 r) { return D2(__fma_rn(p.a, q.a, r.a), __fma_rn(p.b, q.b, r.b)); }
__device__ __forceinline__ D2 operator/(D2 p, D2 q) { return D2(__ddiv_rn(p.a, q.a), __ddiv_rn(p.b, q.b)); }

// scalar type of a lane pair
template <typename V> struct LaneOf;
template <> struct LaneOf<F2> { using type = float; };
template <> struct LaneOf<D2> { using type = double; };
// lane-pair type of a scalar
template <typename S> struct PairOf;
template <> struct PairOf<float> { using type = F2; };
template <> struct PairOf<double> { using type = D2; };

template <typename V, typename F>
__device__ __forceinline__ V lanewise(V a, F f)
{
    return V(f(a.x()), f(a.y()));
}
template <typename V, typename F>
__device__ __forceinline__ V lanewise2(V a, V b, F f)
{
    return V(f(a.x(), b.x()), f(a.y(), b.y()));
}

}  // namespace pf3d
