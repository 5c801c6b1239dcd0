// Device vector / quaternion / matrix algebra for the DEM step.
//
// Operation order follows ESyS-Particle's Foundation/vec3.hpp,
// Foundation/Quaternion.hpp and Foundation/Matrix3.hpp term by term, so that
// the FP64 kernels (built with --fmad=false) reproduce the reference's IEEE
// double arithmetic for every + - * / sqrt.  The scalar type is a template
// parameter so the same code serves the FP32 force form.
#pragma once
#include <cuda_runtime.h>
#include <math.h>

#include <type_traits>

namespace dem {

template <class S>
struct V3 {
  S x, y, z;
};
template <class S>
__host__ __device__ __forceinline__ V3<S> mk(S x, S y, S z) { return V3<S>{x, y, z}; }
template <class S>
__host__ __device__ __forceinline__ V3<S> operator+(const V3<S>& a, const V3<S>& b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
template <class S>
__host__ __device__ __forceinline__ V3<S> operator-(const V3<S>& a, const V3<S>& b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
template <class S>
__host__ __device__ __forceinline__ V3<S> operator-(const V3<S>& a) { return {-a.x, -a.y, -a.z}; }
// Vec3 * double (vec3.hpp:117) and double * Vec3 (vec3.hpp:219): both multiply
// componentwise; kept as two functions because the operand order is part of
// the reference expression.
template <class S>
__host__ __device__ __forceinline__ V3<S> operator*(const V3<S>& a, S s) { return {a.x * s, a.y * s, a.z * s}; }
template <class S>
__host__ __device__ __forceinline__ V3<S> operator*(S f, const V3<S>& a) { return {f * a.x, f * a.y, f * a.z}; }
template <class S>
__host__ __device__ __forceinline__ V3<S> operator/(const V3<S>& a, S s) { return {a.x / s, a.y / s, a.z / s}; }
// Mixed forms for non-double scalars (the adjoint's dual numbers): vector of S times a double.
template <class S, typename std::enable_if<!std::is_same<S, double>::value, int>::type = 0>
__host__ __device__ __forceinline__ V3<S> operator*(const V3<S>& a, double s) { return {a.x * s, a.y * s, a.z * s}; }
template <class S, typename std::enable_if<!std::is_same<S, double>::value, int>::type = 0>
__host__ __device__ __forceinline__ V3<S> operator*(double f, const V3<S>& a) { return {f * a.x, f * a.y, f * a.z}; }
template <class S>
__host__ __device__ __forceinline__ S dot(const V3<S>& a, const V3<S>& b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
template <class S>
__host__ __device__ __forceinline__ V3<S>& operator+=(V3<S>& a, const V3<S>& b) { a.x += b.x; a.y += b.y; a.z += b.z; return a; }
template <class S>
__host__ __device__ __forceinline__ V3<S>& operator-=(V3<S>& a, const V3<S>& b) { a.x -= b.x; a.y -= b.y; a.z -= b.z; return a; }
template <class S>  // vec3.hpp:203
__host__ __device__ __forceinline__ V3<S> cross(const V3<S>& l, const V3<S>& r) {
  return {l.y * r.z - l.z * r.y, l.z * r.x - l.x * r.z, l.x * r.y - l.y * r.x};
}
template <class S>  // vec3.hpp:234
__host__ __device__ __forceinline__ S norm2(const V3<S>& a) { return a.x * a.x + a.y * a.y + a.z * a.z; }
template <class S>  // vec3.hpp:227
__host__ __device__ __forceinline__ S norm(const V3<S>& a) { return sqrt(a.x * a.x + a.y * a.y + a.z * a.z); }
template <class T, class S>
__host__ __device__ __forceinline__ V3<T> cvt(const V3<S>& a) { return {T(a.x), T(a.y), T(a.z)}; }

template <class S>
struct Quat {
  S s;
  V3<S> v;
};
template <class S>  // Quaternion::operator*(const Quaternion&)
__host__ __device__ __forceinline__ Quat<S> qmul(const Quat<S>& a, const Quat<S>& b) {
  return {a.s * b.s - dot(a.v, b.v), a.s * b.v + b.s * a.v + cross(a.v, b.v)};
}
template <class S>
__host__ __device__ __forceinline__ Quat<S> qinv(const Quat<S>& a) { return {a.s, -a.v}; }

template <class S>
struct M3 {
  S m[3][3];
};
template <class S>  // Quaternion::to_matrix
__host__ __device__ __forceinline__ M3<S> to_matrix(const Quat<S>& q) {
  M3<S> r;
  const S s = q.s, x = q.v.x, y = q.v.y, z = q.v.z;
  r.m[0][0] = s * s + x * x - y * y - z * z;
  r.m[0][1] = S(2) * (x * y + s * z);
  r.m[0][2] = S(2) * (x * z - s * y);
  r.m[1][0] = S(2) * (x * y - s * z);
  r.m[1][1] = s * s - x * x + y * y - z * z;
  r.m[1][2] = S(2) * (y * z + s * x);
  r.m[2][0] = S(2) * (x * z + s * y);
  r.m[2][1] = S(2) * (y * z - s * x);
  r.m[2][2] = s * s - x * x - y * y + z * z;
  return r;
}
template <class S>  // Matrix3 * Vec3 (Matrix3.hpp:126)
__host__ __device__ __forceinline__ V3<S> mul(const M3<S>& a, const V3<S>& v) {
  return {a.m[0][0] * v.x + a.m[0][1] * v.y + a.m[0][2] * v.z, a.m[1][0] * v.x + a.m[1][1] * v.y + a.m[1][2] * v.z,
          a.m[2][0] * v.x + a.m[2][1] * v.y + a.m[2][2] * v.z};
}
template <class S>  // Matrix3::trans() * Vec3, without forming the transpose
__host__ __device__ __forceinline__ V3<S> mulT(const M3<S>& a, const V3<S>& v) {
  return {a.m[0][0] * v.x + a.m[1][0] * v.y + a.m[2][0] * v.z, a.m[0][1] * v.x + a.m[1][1] * v.y + a.m[2][1] * v.z,
          a.m[0][2] * v.x + a.m[1][2] * v.y + a.m[2][2] * v.z};
}

__device__ __forceinline__ V3<double> xyz(const double4& a) { return {a.x, a.y, a.z}; }
__device__ __forceinline__ double4 d4(const V3<double>& a, double w) { return make_double4(a.x, a.y, a.z, w); }

}  // namespace dem
