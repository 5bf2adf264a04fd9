// Multi-lane forward dual numbers: value v and N directional derivatives d[N]
// (one seeded direction per lane).  Branches compare values, so a kernel run
// on DN<N> differentiates the branch it takes.  Used for face Jacobians and
// the local Jacobians of the adjoint kernels.
#pragma once
#include <cuda_runtime.h>

namespace fcfd {

template <int N>
struct DN {
  double v, d[N];
  __host__ __device__ DN() : v(0) { for (int i = 0; i < N; ++i) d[i] = 0; }
  __host__ __device__ DN(double x) : v(x) { for (int i = 0; i < N; ++i) d[i] = 0; }
};
template <int N> __device__ __forceinline__ DN<N> operator+(const DN<N> &a, const DN<N> &b) { DN<N> r; r.v = a.v + b.v; for (int i = 0; i < N; ++i) r.d[i] = a.d[i] + b.d[i]; return r; }
template <int N> __device__ __forceinline__ DN<N> operator-(const DN<N> &a, const DN<N> &b) { DN<N> r; r.v = a.v - b.v; for (int i = 0; i < N; ++i) r.d[i] = a.d[i] - b.d[i]; return r; }
template <int N> __device__ __forceinline__ DN<N> operator-(const DN<N> &a) { DN<N> r; r.v = -a.v; for (int i = 0; i < N; ++i) r.d[i] = -a.d[i]; return r; }
template <int N> __device__ __forceinline__ DN<N> operator*(const DN<N> &a, const DN<N> &b) { DN<N> r; r.v = a.v * b.v; for (int i = 0; i < N; ++i) r.d[i] = a.d[i] * b.v + a.v * b.d[i]; return r; }
template <int N> __device__ __forceinline__ DN<N> operator/(const DN<N> &a, const DN<N> &b) { DN<N> r; r.v = a.v / b.v; for (int i = 0; i < N; ++i) r.d[i] = (a.d[i] - r.v * b.d[i]) / b.v; return r; }
template <int N> __device__ __forceinline__ DN<N> operator+(const DN<N> &a, double b) { DN<N> r = a; r.v += b; return r; }
template <int N> __device__ __forceinline__ DN<N> operator+(double a, const DN<N> &b) { DN<N> r = b; r.v += a; return r; }
template <int N> __device__ __forceinline__ DN<N> operator-(const DN<N> &a, double b) { DN<N> r = a; r.v -= b; return r; }
template <int N> __device__ __forceinline__ DN<N> operator-(double a, const DN<N> &b) { DN<N> r = -b; r.v += a; return r; }
template <int N> __device__ __forceinline__ DN<N> operator*(const DN<N> &a, double b) { DN<N> r; r.v = a.v * b; for (int i = 0; i < N; ++i) r.d[i] = a.d[i] * b; return r; }
template <int N> __device__ __forceinline__ DN<N> operator*(double a, const DN<N> &b) { return b * a; }
template <int N> __device__ __forceinline__ DN<N> operator/(const DN<N> &a, double b) { DN<N> r; r.v = a.v / b; for (int i = 0; i < N; ++i) r.d[i] = a.d[i] / b; return r; }
template <int N> __device__ __forceinline__ DN<N> operator/(double a, const DN<N> &b) { DN<N> r; r.v = a / b.v; for (int i = 0; i < N; ++i) r.d[i] = -r.v * b.d[i] / b.v; return r; }
#define FCFD_DN_CMP(op)                                                                                                      \
  template <int N> __device__ __forceinline__ bool operator op(const DN<N> &a, const DN<N> &b) { return a.v op b.v; }      \
  template <int N> __device__ __forceinline__ bool operator op(const DN<N> &a, double b) { return a.v op b; }              \
  template <int N> __device__ __forceinline__ bool operator op(double a, const DN<N> &b) { return a op b.v; }
FCFD_DN_CMP(<)
FCFD_DN_CMP(>)
FCFD_DN_CMP(<=)
FCFD_DN_CMP(>=)
FCFD_DN_CMP(==)
FCFD_DN_CMP(!=)
#undef FCFD_DN_CMP
template <int N> __device__ __forceinline__ DN<N> sqrt(const DN<N> &a) { DN<N> r; r.v = ::sqrt(a.v); for (int i = 0; i < N; ++i) r.d[i] = a.d[i] / (2. * r.v); return r; }
template <int N> __device__ __forceinline__ DN<N> fabs(const DN<N> &a) { return a.v < 0. ? -a : a; }
template <int N> __device__ __forceinline__ DN<N> pow(const DN<N> &a, double e) {
  DN<N> r; r.v = ::pow(a.v, e);
  const double s = (a.v == 0.) ? 0. : e * r.v / a.v;
  for (int i = 0; i < N; ++i) r.d[i] = s * a.d[i];
  return r;
}


}  // namespace fcfd
