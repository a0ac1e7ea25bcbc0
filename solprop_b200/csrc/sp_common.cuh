// Shared definitions of the B200 propagation library: complex helpers, error plumbing
// and launch constants.  Complex numbers are double2 (x = re, y = im), the memory layout
// of NumPy's complex128, or float2 (complex64) in the mixed-precision form.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace sp {

__host__ __device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__host__ __device__ __forceinline__ double2 cadd(double2 a, double2 b) {
  return make_double2(a.x + b.x, a.y + b.y);
}
__host__ __device__ __forceinline__ double2 csub(double2 a, double2 b) {
  return make_double2(a.x - b.x, a.y - b.y);
}
__host__ __device__ __forceinline__ double2 cscale(double s, double2 a) {
  return make_double2(s * a.x, s * a.y);
}
__host__ __device__ __forceinline__ double2 cconj(double2 a) { return make_double2(a.x, -a.y); }
// multiply by -i (forward) or +i (inverse): exact
__host__ __device__ __forceinline__ double2 mul_mi(double2 a) { return make_double2(a.y, -a.x); }
__host__ __device__ __forceinline__ double2 mul_pi(double2 a) { return make_double2(-a.y, a.x); }
// complex division a / b, Smith's algorithm (one scaling, robust to overflow)
__host__ __device__ __forceinline__ double2 cdiv(double2 a, double2 b) {
  if (fabs(b.x) >= fabs(b.y)) {
    double r = b.y / b.x, d = b.x + b.y * r;
    return make_double2((a.x + a.y * r) / d, (a.y - a.x * r) / d);
  }
  double r = b.x / b.y, d = b.x * r + b.y;
  return make_double2((a.x * r + a.y) / d, (a.y * r - a.x) / d);
}
// the same operations on complex64
__host__ __device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__host__ __device__ __forceinline__ float2 cadd(float2 a, float2 b) {
  return make_float2(a.x + b.x, a.y + b.y);
}
__host__ __device__ __forceinline__ float2 csub(float2 a, float2 b) {
  return make_float2(a.x - b.x, a.y - b.y);
}
__host__ __device__ __forceinline__ float2 cscale(float s, float2 a) {
  return make_float2(s * a.x, s * a.y);
}
__host__ __device__ __forceinline__ float2 cconj(float2 a) { return make_float2(a.x, -a.y); }
__host__ __device__ __forceinline__ float2 mul_mi(float2 a) { return make_float2(a.y, -a.x); }
__host__ __device__ __forceinline__ float2 mul_pi(float2 a) { return make_float2(-a.y, a.x); }

// the complex type of a real type, and conversions between the two precisions
template <class R> struct complex_of;
template <> struct complex_of<double> { using type = double2; };
template <> struct complex_of<float> { using type = float2; };
template <class R> using cplx = typename complex_of<R>::type;

template <class C> __host__ __device__ __forceinline__ C to_c(double2 v);
template <> __host__ __device__ __forceinline__ double2 to_c<double2>(double2 v) { return v; }
template <> __host__ __device__ __forceinline__ float2 to_c<float2>(double2 v) {
  return make_float2((float)v.x, (float)v.y);
}
__host__ __device__ __forceinline__ double2 to_d2(double2 v) { return v; }
__host__ __device__ __forceinline__ double2 to_d2(float2 v) { return make_double2(v.x, v.y); }

// exp of a complex number
__device__ __forceinline__ double2 cexp(double2 z) {
  double e = exp(z.x), s, c;
  sincos(z.y, &s, &c);
  return make_double2(e * c, e * s);
}

// Largest fine-grid length one response-column CTA holds; longer rows use a cluster.
constexpr int kColumnSpan = 4096;
constexpr int kColumnThreads = 512;
constexpr int kMaxModes = 8;   // modal route columns handled by the projection kernel
constexpr int kMaxTaps = 16;   // band-rule half-width K + 1

}  // namespace sp
