// Packed FP32 pairs for the z-pair marching kernels.
//
// sm_100 executes two FP32 additions, multiplications or fused multiply-adds in
// one instruction (FADD2 / FMUL2 / FFMA2; __fadd2_rn, __fmul2_rn, __ffma2_rn).
// A thread that computes two adjacent z-sites holds every stencil value, field
// value and intermediate of its point arithmetic as such a pair, so each FP32
// operation of the two sites issues once.
//
// P2 is a float2 with arithmetic operators.  A product is kept unevaluated (Mul2)
// until it is added to or subtracted from something, so that `a * b + c` becomes
// one FFMA2 (as nvcc contracts the scalar expression into one FFMA) and `a * b`
// alone one FMUL2.  The theories' per-site functions, templated on the arithmetic
// type, therefore compile unchanged for P2.
#pragma once

#include <cuda_runtime.h>

namespace sky {

struct P2 {
    float2 v;
    P2() = default;
    __device__ __forceinline__ constexpr P2(float2 w) : v(w) {}
    __device__ __forceinline__ P2(float a, float b) : v(make_float2(a, b)) {}
    // broadcast of a scalar (stencil coefficients, couplings, literals)
    __device__ __forceinline__ explicit P2(double s) : v(make_float2(float(s), float(s))) {}
    __device__ __forceinline__ explicit P2(float s) : v(make_float2(s, s)) {}
    __device__ __forceinline__ explicit P2(int s) : v(make_float2(float(s), float(s))) {}
};

__device__ __forceinline__ P2 p2_fma(P2 a, P2 b, P2 c) { return P2(__ffma2_rn(a.v, b.v, c.v)); }
__device__ __forceinline__ P2 p2_add(P2 a, P2 b) { return P2(__fadd2_rn(a.v, b.v)); }
__device__ __forceinline__ P2 p2_mul(P2 a, P2 b) { return P2(__fmul2_rn(a.v, b.v)); }
__device__ __forceinline__ P2 p2_neg(P2 a) { return P2(make_float2(-a.v.x, -a.v.y)); }
// a - b as one FFMA2 (b * -1 is exact, so the result is the rounded difference)
__device__ __forceinline__ P2 p2_sub(P2 a, P2 b) { return P2(__ffma2_rn(b.v, make_float2(-1.0f, -1.0f), a.v)); }

struct Mul2 {
    P2 a, b;
    __device__ __forceinline__ operator P2() const { return p2_mul(a, b); }
};

__device__ __forceinline__ Mul2 operator*(P2 a, P2 b) { return Mul2{a, b}; }
__device__ __forceinline__ Mul2 operator*(Mul2 a, P2 b) { return Mul2{P2(a), b}; }
__device__ __forceinline__ Mul2 operator*(P2 a, Mul2 b) { return Mul2{a, P2(b)}; }
__device__ __forceinline__ Mul2 operator*(Mul2 a, Mul2 b) { return Mul2{P2(a), P2(b)}; }

__device__ __forceinline__ P2 operator+(P2 a, P2 b) { return p2_add(a, b); }
__device__ __forceinline__ P2 operator-(P2 a, P2 b) { return p2_sub(a, b); }
__device__ __forceinline__ P2 operator-(P2 a) { return p2_neg(a); }
__device__ __forceinline__ P2 operator-(Mul2 m) { return p2_mul(p2_neg(m.a), m.b); }

__device__ __forceinline__ P2 operator+(Mul2 m, P2 c) { return p2_fma(m.a, m.b, c); }
__device__ __forceinline__ P2 operator+(P2 c, Mul2 m) { return p2_fma(m.a, m.b, c); }
__device__ __forceinline__ P2 operator-(P2 c, Mul2 m) { return p2_fma(p2_neg(m.a), m.b, c); }
__device__ __forceinline__ P2 operator-(Mul2 m, P2 c) { return p2_fma(m.a, m.b, p2_neg(c)); }
__device__ __forceinline__ P2 operator+(Mul2 m, Mul2 n) { return p2_fma(m.a, m.b, P2(n)); }
__device__ __forceinline__ P2 operator-(Mul2 m, Mul2 n) { return p2_fma(m.a, m.b, p2_neg(P2(n))); }

__device__ __forceinline__ P2& operator+=(P2& a, P2 b) { return a = a + b; }
__device__ __forceinline__ P2& operator-=(P2& a, P2 b) { return a = a - b; }
__device__ __forceinline__ P2& operator+=(P2& a, Mul2 m) { return a = a + m; }
__device__ __forceinline__ P2& operator-=(P2& a, Mul2 m) { return a = a - m; }
__device__ __forceinline__ P2& operator*=(P2& a, P2 b) { return a = p2_mul(a, b); }

// lane-wise division (IEEE, as the scalar path divides)
__device__ __forceinline__ P2 operator/(P2 a, P2 b) { return P2(make_float2(a.v.x / b.v.x, a.v.y / b.v.y)); }
__device__ __forceinline__ P2 operator/(Mul2 a, P2 b) { return P2(a) / b; }

// lane-wise select: lane k of the result is a's when mk[k], else 0
__device__ __forceinline__ P2 p2_mask(P2 a, bool m0, bool m1) {
    return P2(make_float2(m0 ? a.v.x : 0.0f, m1 ? a.v.y : 0.0f));
}
__device__ __forceinline__ P2 p2_mask(Mul2 a, bool m0, bool m1) { return p2_mask(P2(a), m0, m1); }

// shared-memory pair at an even offset (8-byte aligned)
__device__ __forceinline__ P2 p2_load(const float* p) { return P2(*reinterpret_cast<const float2*>(p)); }

}  // namespace sky
