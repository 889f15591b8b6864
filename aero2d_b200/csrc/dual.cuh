// Forward-mode dual numbers for the hand-written linearisations of the Euler
// residual: the Jacobian-vector product (one tangent) and the 4x4 face
// Jacobian blocks (several tangents per pass).
//
// Semantics follow JAX's forward-mode rules that aero2d/implicit.py relies on
// through jax.jvp and jax.jacfwd: selections by the primal value carry the
// tangent of the chosen branch, and maximum/minimum split the tangent 0.5/0.5
// at an exact tie of the primal values.
#pragma once
#include <cuda_runtime.h>
#include <math.h>

namespace a2d {

template <typename T, int N>
struct Dual {
  T v;
  T d[N];
};

template <typename S> struct ScalarTraits { using real = S; static constexpr int n = 0; };
template <typename T, int N> struct ScalarTraits<Dual<T, N>> { using real = T; static constexpr int n = N; };

template <typename T> __device__ __forceinline__ T val(T x) { return x; }
template <typename T, int N> __device__ __forceinline__ T val(const Dual<T, N>& x) { return x.v; }

template <typename S> __device__ __forceinline__ S lift(typename ScalarTraits<S>::real x);
template <> __device__ __forceinline__ double lift<double>(double x) { return x; }
template <> __device__ __forceinline__ float lift<float>(float x) { return x; }

template <typename T, int N>
__device__ __forceinline__ Dual<T, N> make_const(T x) {
  Dual<T, N> r;
  r.v = x;
#pragma unroll
  for (int k = 0; k < N; ++k) r.d[k] = T(0);
  return r;
}

// ---- arithmetic -----------------------------------------------------------
#define A2D_DUAL_BINOP(OP, VEXPR, DEXPR)                                         \
  template <typename T, int N>                                                   \
  __device__ __forceinline__ Dual<T, N> operator OP(const Dual<T, N>& a,         \
                                                    const Dual<T, N>& b) {       \
    Dual<T, N> r;                                                                \
    r.v = VEXPR;                                                                 \
    _Pragma("unroll") for (int k = 0; k < N; ++k) r.d[k] = DEXPR;                \
    return r;                                                                    \
  }

A2D_DUAL_BINOP(+, a.v + b.v, a.d[k] + b.d[k])
A2D_DUAL_BINOP(-, a.v - b.v, a.d[k] - b.d[k])
A2D_DUAL_BINOP(*, a.v * b.v, a.d[k] * b.v + a.v * b.d[k])
#undef A2D_DUAL_BINOP

template <typename T, int N>
__device__ __forceinline__ Dual<T, N> operator/(const Dual<T, N>& a, const Dual<T, N>& b) {
  Dual<T, N> r;
  r.v = a.v / b.v;
  const T ib = T(1) / b.v;
#pragma unroll
  for (int k = 0; k < N; ++k) r.d[k] = (a.d[k] - r.v * b.d[k]) * ib;
  return r;
}

template <typename T, int N>
__device__ __forceinline__ Dual<T, N> operator-(const Dual<T, N>& a) {
  Dual<T, N> r;
  r.v = -a.v;
#pragma unroll
  for (int k = 0; k < N; ++k) r.d[k] = -a.d[k];
  return r;
}

// mixed with a plain real
template <typename T, int N>
__device__ __forceinline__ Dual<T, N> operator+(const Dual<T, N>& a, T b) {
  Dual<T, N> r = a;
  r.v = a.v + b;
  return r;
}
template <typename T, int N>
__device__ __forceinline__ Dual<T, N> operator+(T a, const Dual<T, N>& b) {
  Dual<T, N> r = b;
  r.v = a + b.v;
  return r;
}
template <typename T, int N>
__device__ __forceinline__ Dual<T, N> operator-(const Dual<T, N>& a, T b) {
  Dual<T, N> r = a;
  r.v = a.v - b;
  return r;
}
template <typename T, int N>
__device__ __forceinline__ Dual<T, N> operator-(T a, const Dual<T, N>& b) {
  Dual<T, N> r;
  r.v = a - b.v;
#pragma unroll
  for (int k = 0; k < N; ++k) r.d[k] = -b.d[k];
  return r;
}
template <typename T, int N>
__device__ __forceinline__ Dual<T, N> operator*(const Dual<T, N>& a, T b) {
  Dual<T, N> r;
  r.v = a.v * b;
#pragma unroll
  for (int k = 0; k < N; ++k) r.d[k] = a.d[k] * b;
  return r;
}
template <typename T, int N>
__device__ __forceinline__ Dual<T, N> operator*(T a, const Dual<T, N>& b) {
  Dual<T, N> r;
  r.v = a * b.v;
#pragma unroll
  for (int k = 0; k < N; ++k) r.d[k] = a * b.d[k];
  return r;
}
template <typename T, int N>
__device__ __forceinline__ Dual<T, N> operator/(const Dual<T, N>& a, T b) {
  Dual<T, N> r;
  r.v = a.v / b;
#pragma unroll
  for (int k = 0; k < N; ++k) r.d[k] = a.d[k] / b;
  return r;
}
template <typename T, int N>
__device__ __forceinline__ Dual<T, N> operator/(T a, const Dual<T, N>& b) {
  Dual<T, N> r;
  r.v = a / b.v;
  const T s = -r.v / b.v;
#pragma unroll
  for (int k = 0; k < N; ++k) r.d[k] = s * b.d[k];
  return r;
}

// ---- elementary functions ---------------------------------------------------
__device__ __forceinline__ double dsqrt(double x) { return sqrt(x); }
__device__ __forceinline__ float dsqrt(float x) { return sqrtf(x); }
template <typename T, int N>
__device__ __forceinline__ Dual<T, N> dsqrt(const Dual<T, N>& a) {
  Dual<T, N> r;
  r.v = dsqrt(a.v);
  const T s = T(0.5) / r.v;
#pragma unroll
  for (int k = 0; k < N; ++k) r.d[k] = a.d[k] * s;
  return r;
}

__device__ __forceinline__ double dpow(double x, double e) { return pow(x, e); }
__device__ __forceinline__ float dpow(float x, float e) { return powf(x, e); }
template <typename T, int N>
__device__ __forceinline__ Dual<T, N> dpow(const Dual<T, N>& a, T e) {
  Dual<T, N> r;
  r.v = dpow(a.v, e);
  const T s = e * dpow(a.v, e - T(1));
#pragma unroll
  for (int k = 0; k < N; ++k) r.d[k] = a.d[k] * s;
  return r;
}

// maximum / minimum: NaN propagates (as jnp.maximum does), balanced tangent at a tie
template <typename T>
__device__ __forceinline__ T vmax(T a, T b) {
  return a > b ? a : (a < b ? b : T(0.5) * (a + b));
}
template <typename T>
__device__ __forceinline__ T vmin(T a, T b) {
  return a < b ? a : (a > b ? b : T(0.5) * (a + b));
}
template <typename T, int N>
__device__ __forceinline__ Dual<T, N> vmax(const Dual<T, N>& a, const Dual<T, N>& b) {
  if (a.v > b.v) return a;
  if (a.v < b.v) return b;
  return T(0.5) * (a + b);
}
template <typename T, int N>
__device__ __forceinline__ Dual<T, N> vmin(const Dual<T, N>& a, const Dual<T, N>& b) {
  if (a.v < b.v) return a;
  if (a.v > b.v) return b;
  return T(0.5) * (a + b);
}
template <typename T, int N>
__device__ __forceinline__ Dual<T, N> vmax(const Dual<T, N>& a, T b) {
  if (a.v > b) return a;
  if (a.v < b) return make_const<T, N>(b);
  Dual<T, N> r = T(0.5) * a;
  r.v = T(0.5) * (a.v + b);
  return r;
}

template <typename S>
__device__ __forceinline__ S sel(bool c, const S& a, const S& b) { return c ? a : b; }

}  // namespace a2d
