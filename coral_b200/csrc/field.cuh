// Element arithmetic shared by the double / complex level-2 kernels: one
// struct per element type (double, float2 = complex64, double2 = complex128)
// with the operations the kernels need, so a kernel template reads the same
// for real and complex data.
#pragma once

#include <cuda_runtime.h>

namespace coral {

template <typename T> struct Fld;

template <> struct Fld<double> {
  static constexpr bool kComplex = false;
  static __host__ __device__ __forceinline__ double zero() { return 0.0; }
  static __host__ __device__ __forceinline__ double one() { return 1.0; }
  static __device__ __forceinline__ double mul(double a, double b) { return a * b; }
  static __device__ __forceinline__ void mac(double& c, double a, double b) { c = fma(a, b, c); }
  static __device__ __forceinline__ double add(double a, double b) { return a + b; }
  static __device__ __forceinline__ double sub(double a, double b) { return a - b; }
  static __device__ __forceinline__ double conj(double a) { return a; }
  static __device__ __forceinline__ double re(double a) { return a; }
  static __device__ __forceinline__ double scale_re(double a, double s) { return a * s; }
  static __device__ __forceinline__ double div(double a, double b) { return a / b; }
  static __device__ __forceinline__ double shfl_xor(double v, int o) {
    return __shfl_xor_sync(0xffffffffu, v, o);
  }
  static __device__ __forceinline__ double shfl(double v, int src) { return __shfl_sync(0xffffffffu, v, src); }
  static __device__ __forceinline__ double neg(double a) { return -a; }
};

template <> struct Fld<float2> {
  static constexpr bool kComplex = true;
  static __host__ __device__ __forceinline__ float2 zero() { return make_float2(0.f, 0.f); }
  static __host__ __device__ __forceinline__ float2 one() { return make_float2(1.f, 0.f); }
  static __device__ __forceinline__ float2 mul(float2 a, float2 b) {
    return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
  }
  static __device__ __forceinline__ void mac(float2& c, float2 a, float2 b) {
    c.x = fmaf(a.x, b.x, c.x);
    c.x = fmaf(-a.y, b.y, c.x);
    c.y = fmaf(a.x, b.y, c.y);
    c.y = fmaf(a.y, b.x, c.y);
  }
  static __device__ __forceinline__ float2 add(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
  static __device__ __forceinline__ float2 sub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
  static __device__ __forceinline__ float2 conj(float2 a) { return make_float2(a.x, -a.y); }
  static __device__ __forceinline__ float2 re(float2 a) { return make_float2(a.x, 0.f); }
  static __device__ __forceinline__ float2 scale_re(float2 a, float s) { return make_float2(a.x * s, a.y * s); }
  // a / b by Smith's method (scaling by the larger component of b)
  static __device__ __forceinline__ float2 div(float2 a, float2 b) {
    if (fabsf(b.x) >= fabsf(b.y)) {
      const float r = b.y / b.x, d = b.x + b.y * r;
      return make_float2((a.x + a.y * r) / d, (a.y - a.x * r) / d);
    }
    const float r = b.x / b.y, d = b.x * r + b.y;
    return make_float2((a.x * r + a.y) / d, (a.y * r - a.x) / d);
  }
  static __device__ __forceinline__ float2 shfl_xor(float2 v, int o) {
    return make_float2(__shfl_xor_sync(0xffffffffu, v.x, o), __shfl_xor_sync(0xffffffffu, v.y, o));
  }
  static __device__ __forceinline__ float2 shfl(float2 v, int src) {
    return make_float2(__shfl_sync(0xffffffffu, v.x, src), __shfl_sync(0xffffffffu, v.y, src));
  }
  static __device__ __forceinline__ float2 neg(float2 a) { return make_float2(-a.x, -a.y); }
};

template <> struct Fld<double2> {
  static constexpr bool kComplex = true;
  static __host__ __device__ __forceinline__ double2 zero() { return make_double2(0.0, 0.0); }
  static __host__ __device__ __forceinline__ double2 one() { return make_double2(1.0, 0.0); }
  static __device__ __forceinline__ double2 mul(double2 a, double2 b) {
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
  }
  static __device__ __forceinline__ void mac(double2& c, double2 a, double2 b) {
    c.x = fma(a.x, b.x, c.x);
    c.x = fma(-a.y, b.y, c.x);
    c.y = fma(a.x, b.y, c.y);
    c.y = fma(a.y, b.x, c.y);
  }
  static __device__ __forceinline__ double2 add(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
  static __device__ __forceinline__ double2 sub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
  static __device__ __forceinline__ double2 conj(double2 a) { return make_double2(a.x, -a.y); }
  static __device__ __forceinline__ double2 re(double2 a) { return make_double2(a.x, 0.0); }
  static __device__ __forceinline__ double2 scale_re(double2 a, double s) { return make_double2(a.x * s, a.y * s); }
  static __device__ __forceinline__ double2 div(double2 a, double2 b) {
    if (fabs(b.x) >= fabs(b.y)) {
      const double r = b.y / b.x, d = b.x + b.y * r;
      return make_double2((a.x + a.y * r) / d, (a.y - a.x * r) / d);
    }
    const double r = b.x / b.y, d = b.x * r + b.y;
    return make_double2((a.x * r + a.y) / d, (a.y * r - a.x) / d);
  }
  static __device__ __forceinline__ double2 shfl_xor(double2 v, int o) {
    return make_double2(__shfl_xor_sync(0xffffffffu, v.x, o), __shfl_xor_sync(0xffffffffu, v.y, o));
  }
  static __device__ __forceinline__ double2 shfl(double2 v, int src) {
    return make_double2(__shfl_sync(0xffffffffu, v.x, src), __shfl_sync(0xffffffffu, v.y, src));
  }
  static __device__ __forceinline__ double2 neg(double2 a) { return make_double2(-a.x, -a.y); }
};

// y <- beta * y the way the reference's scal routines do it: mode 0 leaves y
// (beta == 1), mode 1 multiplies by a real beta (dscal, and csscal/zdscal
// when Im(beta) == 0: both parts scaled, so Inf/NaN in one part stays there),
// mode 2 is the full complex product (cscal/zscal).  Always a multiplication:
// beta == 0 keeps NaN, as the reference's scal does.
template <typename T>
__device__ __forceinline__ T beta_scale(T y, T beta, int mode);
template <> __device__ __forceinline__ double beta_scale(double y, double beta, int mode) {
  return mode == 0 ? y : beta * y;
}
template <> __device__ __forceinline__ float2 beta_scale(float2 y, float2 beta, int mode) {
  return mode == 0 ? y : (mode == 1 ? Fld<float2>::scale_re(y, beta.x) : Fld<float2>::mul(beta, y));
}
template <> __device__ __forceinline__ double2 beta_scale(double2 y, double2 beta, int mode) {
  return mode == 0 ? y : (mode == 1 ? Fld<double2>::scale_re(y, beta.x) : Fld<double2>::mul(beta, y));
}

}  // namespace coral
