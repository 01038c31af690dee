// Minimal complex arithmetic for device code (interleaved re, im).
#pragma once
#include <cuda_runtime.h>

namespace ss {

template <class T>
struct cplx {
  T x, y;
};
using cd = cplx<double>;
using cf = cplx<float>;

template <class T>
__host__ __device__ inline cplx<T> operator+(cplx<T> a, cplx<T> b) { return {a.x + b.x, a.y + b.y}; }
template <class T>
__host__ __device__ inline cplx<T> operator-(cplx<T> a, cplx<T> b) { return {a.x - b.x, a.y - b.y}; }
template <class T>
__host__ __device__ inline cplx<T> operator*(cplx<T> a, T s) { return {a.x * s, a.y * s}; }
template <class T>
__host__ __device__ inline cplx<T> cmul(cplx<T> a, cplx<T> b) {
  return {a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x};
}
template <class T>
__host__ __device__ inline cplx<T> operator*(cplx<T> a, cplx<T> b) { return cmul(a, b); }
// a - b*c with the two real products of each part fused
template <class T>
__host__ __device__ inline cplx<T> cfms(cplx<T> a, cplx<T> b, cplx<T> c) {
  return {a.x - b.x * c.x + b.y * c.y, a.y - b.x * c.y - b.y * c.x};
}
template <class T>
__host__ __device__ inline cplx<T> cdiv(cplx<T> a, cplx<T> b) {
  // Smith's algorithm
  if (fabs(b.x) >= fabs(b.y)) {
    T r = b.y / b.x, d = b.x + b.y * r;
    return {(a.x + a.y * r) / d, (a.y - a.x * r) / d};
  }
  T r = b.x / b.y, d = b.x * r + b.y;
  return {(a.x * r + a.y) / d, (a.y * r - a.x) / d};
}
template <class T>
__host__ __device__ inline T cabs1(cplx<T> a) { return fabs(a.x) + fabs(a.y); }
template <class T>
__host__ __device__ inline T cabs2(cplx<T> a) { return a.x * a.x + a.y * a.y; }

}  // namespace ss
