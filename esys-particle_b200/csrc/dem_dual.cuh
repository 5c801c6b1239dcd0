// Forward-mode dual numbers with N tangent components, FP64.  Evaluating a law
// on Dual<N> inputs seeded with unit tangents yields its N input derivatives
// alongside the value; the adjoint contracts them with the output adjoints.
// Branches follow the primal values, so the derivative is the one of the branch
// taken by the forward pass.
#pragma once
#include <math.h>

namespace dem {

// keep the FP64 overloads visible beside the dual ones inside this namespace
using ::acos;
using ::sqrt;

template <int N>
struct Dual {
  double v;
  double d[N];
  __host__ __device__ __forceinline__ Dual() : v(0.0) {
#pragma unroll
    for (int k = 0; k < N; ++k) d[k] = 0.0;
  }
  __host__ __device__ __forceinline__ Dual(double x) : v(x) {
#pragma unroll
    for (int k = 0; k < N; ++k) d[k] = 0.0;
  }
  __host__ __device__ __forceinline__ static Dual seed(double x, int k) {
    Dual r(x);
    r.d[k] = 1.0;
    return r;
  }
};

#define DEM_DUAL_BIN(OP, VAL, DER)                                                                        \
  template <int N>                                                                                        \
  __host__ __device__ __forceinline__ Dual<N> operator OP(const Dual<N>& a, const Dual<N>& b) {          \
    Dual<N> r;                                                                                            \
    r.v = VAL;                                                                                            \
    _Pragma("unroll") for (int k = 0; k < N; ++k) r.d[k] = DER;                                           \
    return r;                                                                                             \
  }
DEM_DUAL_BIN(+, a.v + b.v, a.d[k] + b.d[k])
DEM_DUAL_BIN(-, a.v - b.v, a.d[k] - b.d[k])
DEM_DUAL_BIN(*, a.v * b.v, a.d[k] * b.v + a.v * b.d[k])
#undef DEM_DUAL_BIN

template <int N>
__host__ __device__ __forceinline__ Dual<N> operator/(const Dual<N>& a, const Dual<N>& b) {
  Dual<N> r;
  r.v = a.v / b.v;
  const double ib = 1.0 / b.v;
#pragma unroll
  for (int k = 0; k < N; ++k) r.d[k] = (a.d[k] - r.v * b.d[k]) * ib;
  return r;
}
template <int N>
__host__ __device__ __forceinline__ Dual<N> operator-(const Dual<N>& a) {
  Dual<N> r;
  r.v = -a.v;
#pragma unroll
  for (int k = 0; k < N; ++k) r.d[k] = -a.d[k];
  return r;
}
template <int N>
__host__ __device__ __forceinline__ Dual<N> operator*(const Dual<N>& a, double s) {
  Dual<N> r;
  r.v = a.v * s;
#pragma unroll
  for (int k = 0; k < N; ++k) r.d[k] = a.d[k] * s;
  return r;
}
template <int N>
__host__ __device__ __forceinline__ Dual<N> operator*(double s, const Dual<N>& a) { return a * s; }
template <int N>
__host__ __device__ __forceinline__ Dual<N> operator/(const Dual<N>& a, double s) {
  Dual<N> r;
  r.v = a.v / s;  // the primal is the IEEE quotient of the FP64 law
#pragma unroll
  for (int k = 0; k < N; ++k) r.d[k] = a.d[k] / s;
  return r;
}
template <int N>
__host__ __device__ __forceinline__ Dual<N> operator/(double s, const Dual<N>& a) { return Dual<N>(s) / a; }
template <int N>
__host__ __device__ __forceinline__ Dual<N> operator+(const Dual<N>& a, double s) {
  Dual<N> r = a;
  r.v += s;
  return r;
}
template <int N>
__host__ __device__ __forceinline__ Dual<N> operator+(double s, const Dual<N>& a) { return a + s; }
template <int N>
__host__ __device__ __forceinline__ Dual<N> operator-(const Dual<N>& a, double s) { return a + (-s); }
template <int N>
__host__ __device__ __forceinline__ Dual<N> operator-(double s, const Dual<N>& a) { return (-a) + s; }
template <int N>
__host__ __device__ __forceinline__ Dual<N>& operator+=(Dual<N>& a, const Dual<N>& b) { a = a + b; return a; }
template <int N>
__host__ __device__ __forceinline__ Dual<N>& operator-=(Dual<N>& a, const Dual<N>& b) { a = a - b; return a; }

template <int N>
__host__ __device__ __forceinline__ Dual<N> sqrt(const Dual<N>& a) {
  Dual<N> r;
  r.v = ::sqrt(a.v);
  const double g = r.v > 0.0 ? 0.5 / r.v : 0.0;
#pragma unroll
  for (int k = 0; k < N; ++k) r.d[k] = a.d[k] * g;
  return r;
}
template <int N>
__host__ __device__ __forceinline__ Dual<N> acos(const Dual<N>& a) {
  Dual<N> r;
  r.v = ::acos(a.v);
  const double g = -1.0 / ::sqrt(1.0 - a.v * a.v);
#pragma unroll
  for (int k = 0; k < N; ++k) r.d[k] = a.d[k] * g;
  return r;
}

#define DEM_DUAL_CMP(OP)                                                                                  \
  template <int N>                                                                                        \
  __host__ __device__ __forceinline__ bool operator OP(const Dual<N>& a, double b) { return a.v OP b; }  \
  template <int N>                                                                                        \
  __host__ __device__ __forceinline__ bool operator OP(const Dual<N>& a, const Dual<N>& b) { return a.v OP b.v; }
DEM_DUAL_CMP(<)
DEM_DUAL_CMP(>)
DEM_DUAL_CMP(<=)
DEM_DUAL_CMP(>=)
DEM_DUAL_CMP(==)
DEM_DUAL_CMP(!=)
#undef DEM_DUAL_CMP

}  // namespace dem
