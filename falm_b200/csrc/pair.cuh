// Arithmetic on pairs of adjacent cells (x, x+1).  FP32 pairs go through the
// packed FP32 pipe of sm_100 (fma/add/mul.rn.f32x2); each lane rounds exactly
// as the scalar operation.  FP64 pairs are two scalar operations.
#pragma once
#include <cuda_runtime.h>

namespace fb {

template <typename V> struct Pair;
template <> struct Pair<float> { using type = float2; };
template <> struct Pair<double> { using type = double2; };
template <typename V> using P2 = typename Pair<V>::type;

__device__ __forceinline__ float2 mk2(float a, float b) { return make_float2(a, b); }
__device__ __forceinline__ double2 mk2(double a, double b) { return make_double2(a, b); }

__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ double2 fma2(double2 a, double2 b, double2 c) { return make_double2(fma(a.x, b.x, c.x), fma(a.y, b.y, c.y)); }
__device__ __forceinline__ double2 mul2(double2 a, double2 b) { return make_double2(a.x * b.x, a.y * b.y); }
__device__ __forceinline__ double2 add2(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
// a - b, one rounding per lane
template <typename V2> __device__ __forceinline__ V2 sub2(V2 a, V2 b) { return add2(a, mk2(-b.x, -b.y)); }
__device__ __forceinline__ float2 fabs2(float2 a) { return make_float2(fabsf(a.x), fabsf(a.y)); }

// lane-wise conversion of a pair
template <typename V, typename T> __device__ __forceinline__ P2<V> cvt2(P2<T> a) { return mk2((V)a.x, (V)a.y); }

// aligned pair loads and stores (the first cell's index is even)
template <typename T> __device__ __forceinline__ P2<T> ld2(const T *p) { return *reinterpret_cast<const P2<T> *>(p); }
template <typename T> __device__ __forceinline__ void st2(T *p, P2<T> v) { *reinterpret_cast<P2<T> *>(p) = v; }

// ac*xc + ae*xe + aw*xw + an*xn + as*xs + at*xt + ab*xb, accumulated in this
// order with fused multiply-adds, on both lanes
template <typename V2>
__device__ __forceinline__ V2 dot7p(V2 ac, V2 ae, V2 aw, V2 an, V2 as, V2 at, V2 ab, V2 xc, V2 xe, V2 xw, V2 xn, V2 xs, V2 xt, V2 xb) {
    V2 r = mul2(ac, xc);
    r = fma2(ae, xe, r);
    r = fma2(aw, xw, r);
    r = fma2(an, xn, r);
    r = fma2(as, xs, r);
    r = fma2(at, xt, r);
    return fma2(ab, xb, r);
}

}  // namespace fb
