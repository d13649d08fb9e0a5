// Two-lane arithmetic for the matrix-free element kernels.
//
// Each thread of the matrix-free product evaluates a pair of elements with the
// same instruction stream.  In FP32 a lane pair lives in one float2 and every
// add, multiply and fused multiply-add issues as one sm_100 packed instruction
// (FADD2 / FMUL2 / FFMA2 through __fadd2_rn / __fmul2_rn / __ffma2_rn, and PTX
// sub.f32x2 for differences), which halves the instruction count of the
// element arithmetic.  Products are kept
// unevaluated (F2Mul) until they meet an addition, so that a*b + c becomes one
// FFMA2 as the scalar compiler would contract it.  In FP64 (D2) the pair is two
// scalars and the compiler contracts as usual.
#pragma once
#include <cuda_runtime.h>

namespace exfem {

struct F2Mul {
  float2 a, b;
};

struct F2 {
  float2 v;
  F2() = default;
  __device__ __forceinline__ F2(float2 x) : v(x) {}
  __device__ __forceinline__ F2(float x, float y) : v(make_float2(x, y)) {}
  __device__ __forceinline__ F2(double s) : v(make_float2((float)s, (float)s)) {}
  __device__ __forceinline__ F2(int s) : v(make_float2((float)s, (float)s)) {}
  __device__ __forceinline__ F2(F2Mul m) : v(__fmul2_rn(m.a, m.b)) {}
  __device__ __forceinline__ float lo() const { return v.x; }
  __device__ __forceinline__ float hi() const { return v.y; }
};

// a - b as one packed instruction (PTX sub.f32x2, sm_100)
__device__ __forceinline__ float2 fsub2(float2 a, float2 b) {
  unsigned long long r;
  asm("sub.rn.f32x2 %0, %1, %2;"
      : "=l"(r)
      : "l"(*reinterpret_cast<const unsigned long long*>(&a)), "l"(*reinterpret_cast<const unsigned long long*>(&b)));
  return *reinterpret_cast<const float2*>(&r);
}
__device__ __forceinline__ float2 neg2(float2 a) { return __fmul2_rn(a, make_float2(-1.0f, -1.0f)); }

__device__ __forceinline__ F2Mul operator*(F2 a, F2 b) { return {a.v, b.v}; }
__device__ __forceinline__ F2Mul operator*(F2Mul m, F2 c) { return {__fmul2_rn(m.a, m.b), c.v}; }
__device__ __forceinline__ F2Mul operator*(F2 c, F2Mul m) { return {c.v, __fmul2_rn(m.a, m.b)}; }
__device__ __forceinline__ F2Mul operator*(F2Mul m, F2Mul n) { return {__fmul2_rn(m.a, m.b), __fmul2_rn(n.a, n.b)}; }
__device__ __forceinline__ F2 operator+(F2 a, F2 b) { return __fadd2_rn(a.v, b.v); }
__device__ __forceinline__ F2 operator-(F2 a, F2 b) { return fsub2(a.v, b.v); }
__device__ __forceinline__ F2 operator-(F2 a) { return neg2(a.v); }
__device__ __forceinline__ F2Mul operator-(F2Mul m) { return {neg2(m.a), m.b}; }
__device__ __forceinline__ F2 operator+(F2Mul m, F2 c) { return __ffma2_rn(m.a, m.b, c.v); }
__device__ __forceinline__ F2 operator+(F2 c, F2Mul m) { return __ffma2_rn(m.a, m.b, c.v); }
__device__ __forceinline__ F2 operator-(F2Mul m, F2 c) { return fsub2(__fmul2_rn(m.a, m.b), c.v); }
__device__ __forceinline__ F2 operator-(F2 c, F2Mul m) { return fsub2(c.v, __fmul2_rn(m.a, m.b)); }
__device__ __forceinline__ F2 operator+(F2Mul m, F2Mul n) { return __ffma2_rn(m.a, m.b, __fmul2_rn(n.a, n.b)); }
__device__ __forceinline__ F2 operator-(F2Mul m, F2Mul n) { return fsub2(__fmul2_rn(m.a, m.b), __fmul2_rn(n.a, n.b)); }
__device__ __forceinline__ F2 operator/(F2 a, F2 b) { return F2(a.v.x / b.v.x, a.v.y / b.v.y); }
__device__ __forceinline__ F2& operator+=(F2& a, F2 b) { return a = a + b; }
__device__ __forceinline__ F2& operator+=(F2& a, F2Mul m) { return a = m + a; }
__device__ __forceinline__ F2& operator-=(F2& a, F2 b) { return a = a - b; }
__device__ __forceinline__ F2& operator-=(F2& a, F2Mul m) { return a = a - m; }
__device__ __forceinline__ F2& operator*=(F2& a, F2 b) { return a = F2(a * b); }

struct alignas(16) D2 {
  double x, y;
  D2() = default;
  __device__ __forceinline__ D2(double a, double b) : x(a), y(b) {}
  __device__ __forceinline__ D2(double s) : x(s), y(s) {}
  __device__ __forceinline__ D2(int s) : x(s), y(s) {}
  __device__ __forceinline__ double lo() const { return x; }
  __device__ __forceinline__ double hi() const { return y; }
};
__device__ __forceinline__ D2 operator*(D2 a, D2 b) { return {a.x * b.x, a.y * b.y}; }
__device__ __forceinline__ D2 operator+(D2 a, D2 b) { return {a.x + b.x, a.y + b.y}; }
__device__ __forceinline__ D2 operator-(D2 a, D2 b) { return {a.x - b.x, a.y - b.y}; }
__device__ __forceinline__ D2 operator-(D2 a) { return {-a.x, -a.y}; }
__device__ __forceinline__ D2 operator/(D2 a, D2 b) { return {a.x / b.x, a.y / b.y}; }
__device__ __forceinline__ D2& operator+=(D2& a, D2 b) { return a = a + b; }
__device__ __forceinline__ D2& operator-=(D2& a, D2 b) { return a = a - b; }
__device__ __forceinline__ D2& operator*=(D2& a, D2 b) { return a = a * b; }

template <class T> struct PairOf;
template <> struct PairOf<float> { using type = F2; };
template <> struct PairOf<double> { using type = D2; };

// a node value or a slot of the matrix-free kernels: (x, y, z) padded to 4
template <class T>
struct alignas(4 * sizeof(T)) Node4 {
  T x, y, z, w;
};

}  // namespace exfem
