// Forward-mode dual numbers with N tangent directions (host and device), for the derivatives of the
// O(N) per-triangle geometry in the adjoint (self blocks, incenters, areas, normals).  Each
// operation carries the chain rule of the operation it mirrors; the values are those of the plain
// double expression.
#pragma once

#include <cmath>

namespace bgpu {

// the plain double functions stay visible beside the Dual overloads below
using ::acos;
using ::cos;
using ::log;
using ::sin;
using ::sqrt;

template <int N>
struct Dual {
  double v;
  double d[N];
  __host__ __device__ Dual() : v(0.0) {
    for (int i = 0; i < N; ++i) d[i] = 0.0;
  }
  __host__ __device__ Dual(double x) : v(x) {  // NOLINT: constants promote implicitly
    for (int i = 0; i < N; ++i) d[i] = 0.0;
  }
  // the k-th independent variable with value x
  __host__ __device__ static Dual var(double x, int k) {
    Dual r(x);
    r.d[k] = 1.0;
    return r;
  }
};

template <int N>
__host__ __device__ inline Dual<N> operator+(const Dual<N>& a, const Dual<N>& b) {
  Dual<N> r;
  r.v = a.v + b.v;
  for (int i = 0; i < N; ++i) r.d[i] = a.d[i] + b.d[i];
  return r;
}
template <int N>
__host__ __device__ inline Dual<N> operator-(const Dual<N>& a, const Dual<N>& b) {
  Dual<N> r;
  r.v = a.v - b.v;
  for (int i = 0; i < N; ++i) r.d[i] = a.d[i] - b.d[i];
  return r;
}
template <int N>
__host__ __device__ inline Dual<N> operator-(const Dual<N>& a) {
  Dual<N> r;
  r.v = -a.v;
  for (int i = 0; i < N; ++i) r.d[i] = -a.d[i];
  return r;
}
template <int N>
__host__ __device__ inline Dual<N> operator*(const Dual<N>& a, const Dual<N>& b) {
  Dual<N> r;
  r.v = a.v * b.v;
  for (int i = 0; i < N; ++i) r.d[i] = a.d[i] * b.v + a.v * b.d[i];
  return r;
}
template <int N>
__host__ __device__ inline Dual<N> operator/(const Dual<N>& a, const Dual<N>& b) {
  Dual<N> r;
  r.v = a.v / b.v;
  const double ib = 1.0 / b.v;
  for (int i = 0; i < N; ++i) r.d[i] = (a.d[i] - r.v * b.d[i]) * ib;
  return r;
}
template <int N>
__host__ __device__ inline Dual<N> operator+(const Dual<N>& a, double b) { return a + Dual<N>(b); }
template <int N>
__host__ __device__ inline Dual<N> operator+(double a, const Dual<N>& b) { return Dual<N>(a) + b; }
template <int N>
__host__ __device__ inline Dual<N> operator-(const Dual<N>& a, double b) { return a - Dual<N>(b); }
template <int N>
__host__ __device__ inline Dual<N> operator-(double a, const Dual<N>& b) { return Dual<N>(a) - b; }
template <int N>
__host__ __device__ inline Dual<N> operator*(const Dual<N>& a, double b) {
  Dual<N> r;
  r.v = a.v * b;
  for (int i = 0; i < N; ++i) r.d[i] = a.d[i] * b;
  return r;
}
template <int N>
__host__ __device__ inline Dual<N> operator*(double a, const Dual<N>& b) { return b * a; }
template <int N>
__host__ __device__ inline Dual<N> operator/(const Dual<N>& a, double b) { return a * (1.0 / b); }
template <int N>
__host__ __device__ inline Dual<N> operator/(double a, const Dual<N>& b) { return Dual<N>(a) / b; }

// f(a) with f' given: value fv, derivative df
template <int N>
__host__ __device__ inline Dual<N> chain(const Dual<N>& a, double fv, double df) {
  Dual<N> r;
  r.v = fv;
  for (int i = 0; i < N; ++i) r.d[i] = df * a.d[i];
  return r;
}
template <int N>
__host__ __device__ inline Dual<N> sqrt(const Dual<N>& a) {
  const double s = ::sqrt(a.v);
  return chain(a, s, 0.5 / s);
}
template <int N>
__host__ __device__ inline Dual<N> log(const Dual<N>& a) {
  return chain(a, ::log(a.v), 1.0 / a.v);
}
template <int N>
__host__ __device__ inline Dual<N> sin(const Dual<N>& a) {
  return chain(a, ::sin(a.v), ::cos(a.v));
}
template <int N>
__host__ __device__ inline Dual<N> cos(const Dual<N>& a) {
  return chain(a, ::cos(a.v), -::sin(a.v));
}
template <int N>
__host__ __device__ inline Dual<N> acos(const Dual<N>& a) {
  return chain(a, ::acos(a.v), -1.0 / ::sqrt(1.0 - a.v * a.v));
}

}  // namespace bgpu
