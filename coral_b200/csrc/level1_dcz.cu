// The rest of level 1 (coral-aarch64/src/level1): d/c/z dot (u / c), asum
// (s, d, sc, dz), nrm2 (d, sc, dz), i?amax (d, c, z), axpy, scal (incl.
// csscal / zdscal), copy, swap (d, c, z), the rotations srot / drot / csrot
// / zdrot and srotm / drotm, and the rotation constructors srotg / drotg /
// srotmg / drotmg.  Complex data is interleaved (re, im); increments count
// complex elements.
//
// Reductions are single launches with per-block partials that the last block
// to arrive adds in a fixed order (deterministic).  Sums of fp32 data are
// accumulated in fp64 (each product of two fp32 values is exact in fp64),
// sums of fp64 data in fp64.  dnrm2 / dznrm2 take the fp64 sum of squares in
// one pass and rescale by the largest component in a second pass only when
// that sum overflowed or underflowed (the reference keeps a running
// (scale, ssq) pair instead, nrm2_helpers.rs:15-38); NaN propagates.
// i?amax returns the first index of the largest |x| (|re| + |im| for complex,
// icamax.rs), NaN never wins, nothing valid -> 0.  The rotation constructors
// run as one device thread on the handle's stream, reading and writing their
// scalars through the handle's pointer mode.
#include "common.cuh"

#include <cfloat>
#include <mutex>
#include <unordered_map>

namespace coral {
namespace {

constexpr int kL1 = 256;

__device__ bool last_block_l1(unsigned* counter) {
  __shared__ bool is_last;
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    is_last = atomicAdd(counter, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  return is_last;
}

__device__ double bsum(double v, double* sh) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if (lane == 0) sh[warp] = v;
  __syncthreads();
  double r = 0.0;
  if (warp == 0) {
    r = lane < (int)(blockDim.x >> 5) ? sh[lane] : 0.0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) r += __shfl_xor_sync(0xffffffffu, r, o);
  }
  __syncthreads();
  return r;  // valid in thread 0
}

__device__ double bmax(double v, double* sh) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  if (lane == 0) sh[warp] = v;
  __syncthreads();
  double r = 0.0;
  if (warp == 0) {
    r = lane < (int)(blockDim.x >> 5) ? sh[lane] : 0.0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) r = fmax(r, __shfl_xor_sync(0xffffffffu, r, o));
  }
  __syncthreads();
  return r;
}

// Real and imaginary parts of an element as double (imag 0 for real data).
__device__ __forceinline__ double re_of(double v) { return v; }
__device__ __forceinline__ double im_of(double) { return 0.0; }
__device__ __forceinline__ double re_of(float v) { return v; }
__device__ __forceinline__ double im_of(float) { return 0.0; }
__device__ __forceinline__ double re_of(float2 v) { return v.x; }
__device__ __forceinline__ double im_of(float2 v) { return v.y; }
__device__ __forceinline__ double re_of(double2 v) { return v.x; }
__device__ __forceinline__ double im_of(double2 v) { return v.y; }

template <typename T> struct IsCx { static constexpr bool v = false; };
template <> struct IsCx<float2> { static constexpr bool v = true; };
template <> struct IsCx<double2> { static constexpr bool v = true; };

template <typename T> __device__ __forceinline__ T from2(double r, double i);
template <> __device__ __forceinline__ double from2(double r, double) { return r; }
template <> __device__ __forceinline__ float2 from2(double r, double i) { return make_float2((float)r, (float)i); }
template <> __device__ __forceinline__ double2 from2(double r, double i) { return make_double2(r, i); }


// ---- unit-stride access in 16-byte vectors ---------------------------------
// Unit-stride, 16-byte-aligned operands are read (and written) as 16-byte
// vectors, kUnroll of them in flight per thread; the last n % V elements and
// every strided operand go element by element.
constexpr int kUnroll = 4;

template <typename T> struct V16;
template <> struct V16<float> {
  using L = float4;
  static constexpr int kN = 4;
  __device__ static float get(const L& v, int e) { return e == 0 ? v.x : e == 1 ? v.y : e == 2 ? v.z : v.w; }
  __device__ static void set(L& v, int e, float a) {
    if (e == 0) v.x = a; else if (e == 1) v.y = a; else if (e == 2) v.z = a; else v.w = a;
  }
};
template <> struct V16<double> {
  using L = double2;
  static constexpr int kN = 2;
  __device__ static double get(const L& v, int e) { return e == 0 ? v.x : v.y; }
  __device__ static void set(L& v, int e, double a) { if (e == 0) v.x = a; else v.y = a; }
};
template <> struct V16<float2> {
  using L = float4;
  static constexpr int kN = 2;
  __device__ static float2 get(const L& v, int e) { return e == 0 ? make_float2(v.x, v.y) : make_float2(v.z, v.w); }
  __device__ static void set(L& v, int e, float2 a) {
    if (e == 0) { v.x = a.x; v.y = a.y; } else { v.z = a.x; v.w = a.y; }
  }
};
template <> struct V16<double2> {
  using L = double2;
  static constexpr int kN = 1;
  __device__ static double2 get(const L& v, int) { return v; }
  __device__ static void set(L& v, int, double2 a) { v = a; }
};

__device__ __forceinline__ size_t gtid() { return (size_t)blockIdx.x * blockDim.x + threadIdx.x; }
__device__ __forceinline__ size_t gstride() { return (size_t)gridDim.x * blockDim.x; }

// f(x_i, y_i, i) over i in [0, n); y may be null (f then gets x_i twice).
template <typename T, bool kUnit, typename F>
__device__ __forceinline__ void visit(size_t n, const T* __restrict__ x, size_t incx, const T* __restrict__ y,
                                      size_t incy, F f) {
  const size_t tid = gtid(), stride = gstride();
  if constexpr (!kUnit) {
    for (size_t i = tid; i < n; i += stride) {
      const T a = x[i * incx];
      f(a, y ? y[i * incy] : a, i);
    }
  } else {
    using W = V16<T>;
    using L = typename W::L;
    constexpr int V = W::kN;
    const size_t nv = n / V;
    const L* xv = reinterpret_cast<const L*>(x);
    const L* yv = reinterpret_cast<const L*>(y);
    size_t j = tid;
    for (; j + (size_t)(kUnroll - 1) * stride < nv; j += (size_t)kUnroll * stride) {
      L a[kUnroll], b[kUnroll];
#pragma unroll
      for (int u = 0; u < kUnroll; ++u) a[u] = __ldcs(xv + j + u * stride);
      if (y) {
#pragma unroll
        for (int u = 0; u < kUnroll; ++u) b[u] = __ldcs(yv + j + u * stride);
      }
#pragma unroll
      for (int u = 0; u < kUnroll; ++u)
#pragma unroll
        for (int e = 0; e < V; ++e) f(W::get(a[u], e), W::get(y ? b[u] : a[u], e), (j + u * stride) * V + e);
    }
    for (; j < nv; j += stride) {
      const L a = __ldcs(xv + j), b = y ? __ldcs(yv + j) : a;
#pragma unroll
      for (int e = 0; e < V; ++e) f(W::get(a, e), W::get(b, e), j * V + e);
    }
    for (size_t i = nv * V + tid; i < n; i += stride) {
      const T a = x[i];
      f(a, y ? y[i] : a, i);
    }
  }
}

// f(a, b, i) updates a (x_i) and b (y_i) in place; kRX / kWX / kRY / kWY say
// which of x and y are read and written.
template <typename T, bool kUnit, bool kRX, bool kWX, bool kRY, bool kWY, typename F>
__device__ __forceinline__ void update(size_t n, T* __restrict__ x, size_t incx, T* __restrict__ y, size_t incy,
                                       F f) {
  const size_t tid = gtid(), stride = gstride();
  if constexpr (!kUnit) {
    for (size_t i = tid; i < n; i += stride) {
      T a{}, b{};
      if (kRX) a = x[i * incx];
      if (kRY) b = y[i * incy];
      f(a, b, i);
      if (kWX) x[i * incx] = a;
      if (kWY) y[i * incy] = b;
    }
  } else {
    using W = V16<T>;
    using L = typename W::L;
    constexpr int V = W::kN;
    const size_t nv = n / V;
    L* xv = reinterpret_cast<L*>(x);
    L* yv = reinterpret_cast<L*>(y);
    auto body = [&](L& a, L& b, size_t j) {
#pragma unroll
      for (int e = 0; e < V; ++e) {
        T ta = W::get(a, e), tb = W::get(b, e);
        f(ta, tb, j * V + e);
        W::set(a, e, ta);
        W::set(b, e, tb);
      }
    };
    size_t j = tid;
    for (; j + (size_t)(kUnroll - 1) * stride < nv; j += (size_t)kUnroll * stride) {
      L a[kUnroll] = {}, b[kUnroll] = {};
#pragma unroll
      for (int u = 0; u < kUnroll; ++u) {
        if (kRX) a[u] = __ldcs(xv + j + u * stride);
        if (kRY) b[u] = __ldcs(yv + j + u * stride);
      }
#pragma unroll
      for (int u = 0; u < kUnroll; ++u) body(a[u], b[u], j + u * stride);
#pragma unroll
      for (int u = 0; u < kUnroll; ++u) {
        if (kWX) __stcs(xv + j + u * stride, a[u]);
        if (kWY) __stcs(yv + j + u * stride, b[u]);
      }
    }
    for (; j < nv; j += stride) {
      L a{}, b{};
      if (kRX) a = __ldcs(xv + j);
      if (kRY) b = __ldcs(yv + j);
      body(a, b, j);
      if (kWX) __stcs(xv + j, a);
      if (kWY) __stcs(yv + j, b);
    }
    for (size_t i = nv * V + tid; i < n; i += stride) {
      T a{}, b{};
      if (kRX) a = x[i];
      if (kRY) b = y[i];
      f(a, b, i);
      if (kWX) x[i] = a;
      if (kWY) y[i] = b;
    }
  }
}

// ---- dot (u / c) ------------------------------------------------------------
template <typename T, bool kConj, bool kUnit>
__global__ void __launch_bounds__(kL1)
k_dot_x(size_t n, const T* __restrict__ x, size_t incx, const T* __restrict__ y, size_t incy,
        double* part, unsigned* counter, T* out) {
  __shared__ double sh[32];
  double ar = 0.0, ai = 0.0;
  visit<T, kUnit>(n, x, incx, y, incy, [&](T a, T b, size_t) {
    const double xr = re_of(a), xi = kConj ? -im_of(a) : im_of(a), yr = re_of(b), yi = im_of(b);
    ar = fma(xr, yr, ar);
    if (IsCx<T>::v) {
      ar = fma(-xi, yi, ar);
      ai = fma(xr, yi, ai);
      ai = fma(xi, yr, ai);
    }
  });
  const double br = bsum(ar, sh);
  const double bi = IsCx<T>::v ? bsum(ai, sh) : 0.0;
  if (threadIdx.x == 0) {
    part[2 * blockIdx.x] = br;
    part[2 * blockIdx.x + 1] = bi;
  }
  if (!last_block_l1(counter)) return;
  double sr = 0.0, si = 0.0;
  for (unsigned b = threadIdx.x; b < gridDim.x; b += blockDim.x) {
    sr += __ldcg(part + 2 * b);
    si += __ldcg(part + 2 * b + 1);
  }
  sr = bsum(sr, sh);
  si = bsum(si, sh);
  if (threadIdx.x == 0) {
    *out = from2<T>(sr, si);
    *counter = 0;
  }
}

// ---- asum: sum of |x| (|re| + |im| for complex) --------------------------------
template <typename T, typename R, bool kUnit>
__global__ void __launch_bounds__(kL1)
k_asum_x(size_t n, const T* __restrict__ x, size_t incx, double* part, unsigned* counter, R* out) {
  __shared__ double sh[32];
  double a0 = 0.0;
  visit<T, kUnit>(n, x, incx, nullptr, 0, [&](T u, T, size_t) { a0 += fabs(re_of(u)) + fabs(im_of(u)); });
  const double b = bsum(a0, sh);
  if (threadIdx.x == 0) part[blockIdx.x] = b;
  if (!last_block_l1(counter)) return;
  double s = 0.0;
  for (unsigned k = threadIdx.x; k < gridDim.x; k += blockDim.x) s += __ldcg(part + k);
  s = bsum(s, sh);
  if (threadIdx.x == 0) {
    *out = (R)s;
    *counter = 0;
  }
}

// ---- nrm2 -------------------------------------------------------------------
// Pass 1: fp64 sum of squares and the largest |component|.  For fp64 data a
// sum that overflowed (inf) or underflowed (< 2^-960 with a nonzero entry)
// asks pass 2 to rescale: flag[0] = 1, mx in dmx.
template <typename T, typename R, bool kUnit>
__global__ void __launch_bounds__(kL1)
k_nrm2_x(size_t n, const T* __restrict__ x, size_t incx, double* part, unsigned* counter, unsigned* flag,
         double* dmx, R* out) {
  __shared__ double sh[32];
  double s = 0.0, m = 0.0;
  visit<T, kUnit>(n, x, incx, nullptr, 0, [&](T u, T, size_t) {
    const double r = re_of(u);
    s = fma(r, r, s);
    if constexpr (IsCx<T>::v) {
      const double im = im_of(u);
      s = fma(im, im, s);
      if constexpr (sizeof(R) == 8) m = fmax(m, fmax(fabs(r), fabs(im)));
    } else if constexpr (sizeof(R) == 8) {
      m = fmax(m, fabs(r));
    }
  });
  const double bs = bsum(s, sh), bm = bmax(m, sh);
  if (threadIdx.x == 0) {
    part[2 * blockIdx.x] = bs;
    part[2 * blockIdx.x + 1] = bm;
  }
  // the rescaling pass (a programmatic dependent) may start launching; it
  // waits for this whole grid before it reads anything
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
  if (!last_block_l1(counter)) return;
  double ts = 0.0, tm = 0.0;
  for (unsigned b = threadIdx.x; b < gridDim.x; b += blockDim.x) {
    ts += __ldcg(part + 2 * b);
    tm = fmax(tm, __ldcg(part + 2 * b + 1));
  }
  ts = bsum(ts, sh);
  tm = bmax(tm, sh);
  if (threadIdx.x == 0) {
    const bool rescale = sizeof(R) == 8 && !isnan(ts) && !isinf(tm) && (isinf(ts) || (ts < 0x1p-960 && tm > 0.0));
    if (rescale) {
      *flag = 1u;
      *dmx = tm;
    } else {
      *out = (R)sqrt(ts);
    }
    *counter = 0;
  }
}

// Pass 2 (only when pass 1 asked): sum of (x / mx)^2, result mx * sqrt(sum).
template <typename T, typename R, bool kUnit>
__global__ void __launch_bounds__(kL1)
k_nrm2_scaled(size_t n, const T* __restrict__ x, size_t incx, double* part, unsigned* counter,
              unsigned* flag, const double* dmx, R* out) {
  __shared__ double sh[32];
  asm volatile("griddepcontrol.wait;" ::: "memory");   // pass 1 complete and visible
  if (*(volatile unsigned*)flag == 0u) return;   // every block sees the same word
  const double inv = 1.0 / *dmx;
  double s = 0.0;
  visit<T, kUnit>(n, x, incx, nullptr, 0, [&](T u, T, size_t) {
    const double r = re_of(u) * inv;
    s = fma(r, r, s);
    if constexpr (IsCx<T>::v) {
      const double im = im_of(u) * inv;
      s = fma(im, im, s);
    }
  });
  const double bs = bsum(s, sh);
  if (threadIdx.x == 0) part[blockIdx.x] = bs;
  if (!last_block_l1(counter)) return;
  double ts = 0.0;
  for (unsigned b = threadIdx.x; b < gridDim.x; b += blockDim.x) ts += __ldcg(part + b);
  ts = bsum(ts, sh);
  if (threadIdx.x == 0) {
    *out = (R)(*dmx * sqrt(ts));
    *flag = 0u;
    *counter = 0;
  }
}

// ---- i?amax ------------------------------------------------------------------
struct Best {
  double v;
  unsigned long long i;
};
__device__ __forceinline__ bool better(const Best& a, const Best& b) {
  return a.v > b.v || (a.v == b.v && a.i < b.i);
}
__device__ Best bbest(Best a, Best* sh) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    Best b;
    b.v = __shfl_xor_sync(0xffffffffu, a.v, o);
    b.i = __shfl_xor_sync(0xffffffffu, a.i, o);
    if (better(b, a)) a = b;
  }
  if (lane == 0) sh[warp] = a;
  __syncthreads();
  Best r{-INFINITY, ~0ull};
  if (warp == 0) {
    if (lane < (int)(blockDim.x >> 5)) r = sh[lane];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      Best b;
      b.v = __shfl_xor_sync(0xffffffffu, r.v, o);
      b.i = __shfl_xor_sync(0xffffffffu, r.i, o);
      if (better(b, r)) r = b;
    }
  }
  __syncthreads();
  return r;
}
// metric in the element precision: |x|, or |re| + |im| (fp32 sum for complex64)
__device__ __forceinline__ double metric(double v) { return fabs(v); }
__device__ __forceinline__ double metric(float2 v) { return (double)(fabsf(v.x) + fabsf(v.y)); }
__device__ __forceinline__ double metric(double2 v) { return fabs(v.x) + fabs(v.y); }

template <typename T, bool kUnit>
__global__ void __launch_bounds__(kL1)
k_iamax_x(size_t n, const T* __restrict__ x, size_t incx, double* pv, unsigned long long* pi,
          unsigned* counter, unsigned long long* out) {
  __shared__ Best sh[32];
  Best best{-INFINITY, ~0ull};
  visit<T, kUnit>(n, x, incx, nullptr, 0, [&](T u, T, size_t i) {
    const Best c{metric(u), i};   // NaN never compares greater or equal
    if (better(c, best)) best = c;
  });
  const Best bb = bbest(best, sh);
  if (threadIdx.x == 0) {
    pv[blockIdx.x] = bb.v;
    pi[blockIdx.x] = bb.i;
  }
  if (!last_block_l1(counter)) return;
  Best r{-INFINITY, ~0ull};
  for (unsigned b = threadIdx.x; b < gridDim.x; b += blockDim.x) {
    const Best c{__ldcg(pv + b), __ldcg(pi + b)};
    if (better(c, r)) r = c;
  }
  r = bbest(r, sh);
  if (threadIdx.x == 0) {
    *out = r.i == ~0ull ? 0ull : r.i;
    *counter = 0;
  }
}

// ---- elementwise ---------------------------------------------------------------
// The reference's unit-stride loops run in NEON vectors of W elements and
// finish the last n % W scalarly; the vector body fuses where the scalar code
// rounds every product.  `nfused` = n - n % W on unit strides, 0 otherwise:
// element i < nfused takes the vector body's roundings, the rest the scalar
// code's (daxpy.rs, caxpy.rs, zaxpy.rs, cscal.rs, zscal.rs, srot.rs, drot.rs,
// csrot.rs, zdrot.rs, srotm.rs, drotm.rs).  The explicit _rn intrinsics keep
// the compiler from contracting the scalar forms.
__device__ __forceinline__ float mulr(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double mulr(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float addr(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ double addr(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ float subr(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ double subr(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ float fmar(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ double fmar(double a, double b, double c) { return __fma_rn(a, b, c); }

// y += alpha x
template <typename T, bool kUnit>
__global__ void __launch_bounds__(kL1)
k_axpy_x(size_t n, size_t nfused, T alpha, const T* __restrict__ x, size_t incx, T* __restrict__ y, size_t incy) {
  update<T, kUnit, true, false, true, true>(n, const_cast<T*>(x), incx, y, incy, [&](T& a, T& v, size_t i) {
    if constexpr (IsCx<T>::v) {
      if (i < nfused) {   // yr += ar xr; yr -= ai xi; yi += ar xi; yi += ai xr, each fused
        v.x = fmar(alpha.x, a.x, v.x);
        v.x = fmar(-alpha.y, a.y, v.x);
        v.y = fmar(alpha.x, a.y, v.y);
        v.y = fmar(alpha.y, a.x, v.y);
      } else {            // yr += ar xr - ai xi; yi += ar xi + ai xr
        v.x = addr(v.x, subr(mulr(alpha.x, a.x), mulr(alpha.y, a.y)));
        v.y = addr(v.y, addr(mulr(alpha.x, a.y), mulr(alpha.y, a.x)));
      }
    } else {
      v = i < nfused ? fmar(alpha, a, v) : addr(v, mulr(alpha, a));
    }
  });
}

// x <- alpha x; kReal: real alpha on both parts (dscal / csscal / zdscal)
template <typename T, bool kReal, bool kUnit>
__global__ void __launch_bounds__(kL1)
k_scal_x(size_t n, size_t nfused, T alpha, T* __restrict__ x, size_t incx) {
  update<T, kUnit, true, true, false, false>(n, x, incx, nullptr, 0, [&](T& v, T&, size_t i) {
    if constexpr (!IsCx<T>::v) {
      v = mulr(v, alpha);
    } else if constexpr (kReal) {
      v.x = mulr(v.x, alpha.x);
      v.y = mulr(v.y, alpha.x);
    } else if (i < nfused) {   // re = xr ar - xi ai, im = xi ar + xr ai, second term fused
      const auto re = fmar(-v.y, alpha.y, mulr(v.x, alpha.x));
      const auto im = fmar(v.x, alpha.y, mulr(v.y, alpha.x));
      v.x = re;
      v.y = im;
    } else {
      const auto re = subr(mulr(alpha.x, v.x), mulr(alpha.y, v.y));
      const auto im = addr(mulr(alpha.x, v.y), mulr(alpha.y, v.x));
      v.x = re;
      v.y = im;
    }
  });
}

template <typename E, bool kUnit>
__global__ void __launch_bounds__(kL1)
k_copy_x(size_t n, const E* __restrict__ x, size_t incx, E* __restrict__ y, size_t incy) {
  update<E, kUnit, true, false, false, true>(n, const_cast<E*>(x), incx, y, incy,
                                             [](E& a, E& b, size_t) { b = a; });
}

template <typename E, bool kUnit>
__global__ void __launch_bounds__(kL1)
k_swap_x(size_t n, E* __restrict__ x, size_t incx, E* __restrict__ y, size_t incy) {
  update<E, kUnit, true, true, true, true>(n, x, incx, y, incy, [](E& a, E& b, size_t) {
    const E t = a;
    a = b;
    b = t;
  });
}

// Plane rotation with real c, s: x' = c x + s y, y' = c y - s x, each part of
// a complex element independently.  Vector body: x' = fma(y, s, c x); real
// data also y' = fma(-s, x, c y), while csrot / zdrot round both products of y'.
template <typename R, bool kFuseY>
__device__ __forceinline__ void rot_part(R& xv, R& yv, R c, R s, bool fused) {
  R xn, yn;
  if (fused) {
    xn = fmar(yv, s, mulr(c, xv));
    yn = kFuseY ? fmar(-s, xv, mulr(c, yv)) : subr(mulr(c, yv), mulr(s, xv));
  } else {
    xn = addr(mulr(c, xv), mulr(s, yv));
    yn = subr(mulr(c, yv), mulr(s, xv));
  }
  xv = xn;
  yv = yn;
}
template <typename T, typename R, bool kUnit>
__global__ void __launch_bounds__(kL1)
k_rot_x(size_t n, size_t nfused, T* __restrict__ x, size_t incx, T* __restrict__ y, size_t incy, R c, R s) {
  update<T, kUnit, true, true, true, true>(n, x, incx, y, incy, [&](T& a, T& b, size_t i) {
    const bool f = i < nfused;
    if constexpr (IsCx<T>::v) {
      rot_part<R, false>(a.x, b.x, c, s, f);
      rot_part<R, false>(a.y, b.y, c, s, f);
    } else {
      rot_part<R, true>(a, b, c, s, f);
    }
  });
}

// Modified rotation (srotm.rs, drotm.rs), param = [flag, h11, h21, h12, h22]:
// flag < 0 full H; flag == 0 unit diagonal; otherwise (flag 1, or NaN)
// h12 = 1, h21 = -1.  flag == -2 returns on the host.
template <typename R, bool kUnit>
__global__ void __launch_bounds__(kL1)
k_rotm_x(size_t n, size_t nfused, R* __restrict__ x, size_t incx, R* __restrict__ y, size_t incy, R flag, R h11,
         R h21, R h12, R h22) {
  const int form = flag < (R)0 ? 0 : flag == (R)0 ? 1 : 2;
  update<R, kUnit, true, true, true, true>(n, x, incx, y, incy, [&](R& a, R& b, size_t i) {
    const bool f = i < nfused;
    R xn, yn;
    if (form == 0) {
      xn = f ? fmar(b, h12, mulr(h11, a)) : addr(mulr(h11, a), mulr(h12, b));
      yn = f ? fmar(a, h21, mulr(h22, b)) : addr(mulr(h21, a), mulr(h22, b));
    } else if (form == 1) {
      xn = f ? fmar(b, h12, a) : addr(a, mulr(h12, b));
      yn = f ? fmar(a, h21, b) : addr(mulr(h21, a), b);
    } else {
      xn = f ? fmar(a, h11, b) : addr(mulr(h11, a), b);
      yn = subr(mulr(h22, b), a);
    }
    a = xn;
    b = yn;
  });
}

// ---- rotation constructors (one thread) -------------------------------------------
// srotg.rs: r = scale sqrt((a/scale)^2 + (b/scale)^2) signed like the larger
// of a, b; c = a / r, s = b / r; z as in the reference; a <- r, b <- z.
template <typename R>
__global__ void k_rotg(R* a, R* b, R* c, R* s) {
  const R av = *a, bv = *b;
  const R roe = fabs(av) > fabs(bv) ? av : bv;
  const R scale = fabs(av) + fabs(bv);
  if (scale == (R)0) {
    *c = 1; *s = 0; *a = 0; *b = 0;
    return;
  }
  const R qa = av / scale, qb = bv / scale;
  R r = scale * sqrt(addr(mulr(qa, qa), mulr(qb, qb)));   // powi(2) products, each rounded
  if (roe < (R)0) r = -r;
  const R cv = av / r, sv = bv / r;
  R z = 1;
  if (fabs(av) > fabs(bv)) z = sv;
  if (fabs(bv) >= fabs(av) && cv != (R)0) z = (R)1 / cv;
  *c = cv; *s = sv; *a = r; *b = z;
}

// srotmg.rs: modified Givens construction with rescaling by gam = 4096.
constexpr int kRescaleSteps = 256;
template <typename R>
__global__ void k_rotmg(R* d1, R* d2, R* x1, R y1, R* param) {
  const R gam = 4096, gamsq = gam * gam, rgamsq = (R)1 / gamsq;
  R flag, h11 = 0, h12 = 0, h21 = 0, h22 = 0;
  R sd1 = *d1, sd2 = *d2, sx1 = *x1;
  if (sd1 < (R)0) {
    flag = -1; sd1 = 0; sd2 = 0; sx1 = 0;
  } else {
    const R p2 = sd2 * y1;
    if (p2 == (R)0) {
      param[0] = -2;
      return;
    }
    const R p1 = sd1 * sx1, q2 = p2 * y1, q1 = p1 * sx1;
    if (fabs(q1) > fabs(q2)) {
      h21 = -y1 / sx1;
      h12 = p2 / p1;
      const R u = subr((R)1, mulr(h12, h21));
      if (u <= (R)0) {
        flag = -1; sd1 = 0; sd2 = 0; sx1 = 0; h11 = 0; h12 = 0; h21 = 0; h22 = 0;
      } else {
        flag = 0; sd1 /= u; sd2 /= u; sx1 *= u;
      }
    } else {
      if (q2 < (R)0) {
        flag = -1; sd1 = 0; sd2 = 0; sx1 = 0; h11 = 0; h12 = 0; h21 = 0; h22 = 0;
      } else {
        flag = 1;
        h11 = p1 / p2;
        h22 = sx1 / y1;
        const R u = addr((R)1, mulr(h11, h22));
        const R t = sd2 / u;
        sd2 = sd1 / u;
        sd1 = t;
        sx1 = y1 * u;
      }
    }
    // The rescaling loops end after kRescaleSteps steps: finite inputs need
    // fewer than 100, an infinite d1 or d2 would never leave them.
    if (sd1 != (R)0) {
      for (int it = 0; it < kRescaleSteps && (sd1 <= rgamsq || sd1 >= gamsq); ++it) {
        if (flag == (R)0) { h11 = 1; h22 = 1; flag = -1; }
        else { h21 = -1; h12 = 1; flag = -1; }
        if (sd1 <= rgamsq) { sd1 *= gamsq; sx1 /= gam; h11 /= gam; h12 /= gam; }
        else { sd1 /= gamsq; sx1 *= gam; h11 *= gam; h12 *= gam; }
      }
    }
    if (sd2 != (R)0) {
      for (int it = 0; it < kRescaleSteps && (fabs(sd2) <= rgamsq || fabs(sd2) >= gamsq); ++it) {
        if (flag == (R)0) { h11 = 1; h22 = 1; flag = -1; }
        else { h21 = -1; h12 = 1; flag = -1; }
        if (fabs(sd2) <= rgamsq) { sd2 *= gamsq; h21 /= gam; h22 /= gam; }
        else { sd2 /= gamsq; h21 *= gam; h22 *= gam; }
      }
    }
  }
  param[1] = 0; param[2] = 0; param[3] = 0; param[4] = 0;
  if (flag < (R)0) { param[1] = h11; param[2] = h21; param[3] = h12; param[4] = h22; }
  else if (flag == (R)0) { param[2] = h21; param[3] = h12; }
  else { param[1] = h11; param[4] = h22; }
  param[0] = flag;
  *d1 = sd1; *d2 = sd2; *x1 = sx1;
}

// ---- host helpers ------------------------------------------------------------------
// Resident blocks of 256 threads per SM of a kernel, queried once per kernel.
int resident_blocks(const void* kernel) {
  static std::mutex mu;
  static std::unordered_map<const void*, int> cache;
  std::lock_guard<std::mutex> lock(mu);
  const auto it = cache.find(kernel);
  if (it != cache.end()) return it->second;
  int b = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, kernel, kL1, 0) != cudaSuccess || b < 1) {
    cudaGetLastError();
    b = 1;
  }
  cache.emplace(kernel, b);
  return b;
}

// Most blocks a level-1 launch uses (256 threads: at most 8 resident per SM);
// the reductions size their per-block partials for it.
size_t max_l1_blocks(Handle* h) { return (size_t)h->sm_count * 8; }

// Launches a streaming level-1 kernel on at most one wave of its resident
// blocks, each with at least 8 x 256 elements.
template <typename... P, typename... A>
void l1_launch(Handle* h, size_t n, void (*kernel)(P...), A&&... args) {
  const unsigned g = stream_grid(n, (size_t)kL1 * 8, h->sm_count, resident_blocks((const void*)kernel));
  kernel<<<g, kL1, 0, h->stream>>>(std::forward<A>(args)...);
}

// The same as a programmatic dependent of the previous kernel on the stream:
// its blocks are scheduled as that grid drains and must wait for it with
// griddepcontrol.wait before reading its results.
template <typename... P, typename... A>
cudaError_t l1_launch_dependent(Handle* h, size_t n, void (*kernel)(P...), A&&... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(stream_grid(n, (size_t)kL1 * 8, h->sm_count, resident_blocks((const void*)kernel)));
  cfg.blockDim = dim3(kL1);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = h->stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, kernel, std::forward<A>(args)...);
}

template <typename Out>
coral_status_t finish(Handle* H, Out* result, const void* dres, size_t bytes) {
  coral_status_t s = launch_status(H);
  if (s != CORAL_OK) return s;
  return deliver_result(H, result, dres, bytes);
}

// device staging of the rotation constructors' scalars (8 words)
double* stage(Handle* H) { return &H->words->stage[0]; }

}  // namespace
}  // namespace coral

using namespace coral;

namespace {

// unit strides with 16-byte-aligned operands take the vector path
bool unit_ok(size_t incx, size_t incy, const void* x, const void* y) {
  return incx == 1 && incy == 1 && aligned16(x) && aligned16(y);
}

template <typename T, bool kConj, typename Out>
coral_status_t dot_entry(coral_handle_t hh, size_t n, const void* x, size_t incx, const void* y, size_t incy,
                         Out* result, size_t align) {
  CORAL_HANDLE(hh);
  if (!result) return bad_arg(H, 6);
  T* dres = reinterpret_cast<T*>(&H->words->dresult[2]);
  if (n == 0) {   // cdotc.rs: empty -> 0
    CORAL_CUDA(H, cudaMemsetAsync(dres, 0, sizeof(T), H->stream));
    return deliver_result(H, result, dres, sizeof(T));
  }
  if (!x) return bad_arg(H, 2);
  if (incx == 0) return bad_arg(H, 3);
  if (!y) return bad_arg(H, 4);
  if (incy == 0) return bad_arg(H, 5);
  if (((uintptr_t)x | (uintptr_t)y) & (align - 1)) return bad_arg(H, 2);
  double* part = static_cast<double*>(scratch(H, max_l1_blocks(H) * 2 * sizeof(double)));
  if (!part) return CORAL_ERR_ALLOC;
  const T* xx = static_cast<const T*>(x);
  const T* yy = static_cast<const T*>(y);
  unsigned* ctr = &H->words->counters[kCtrMisc];
  if (unit_ok(incx, incy, x, y))
    l1_launch(H, n, k_dot_x<T, kConj, true>, n, xx, 1, yy, 1, part, ctr, dres);
  else
    l1_launch(H, n, k_dot_x<T, kConj, false>, n, xx, incx, yy, incy, part, ctr, dres);
  return finish(H, result, dres, sizeof(T));
}

template <typename T, typename R>
coral_status_t asum_entry(coral_handle_t hh, size_t n, const void* x, size_t incx, R* result, size_t align) {
  CORAL_HANDLE(hh);
  if (!result) return bad_arg(H, 4);
  R* dres = reinterpret_cast<R*>(&H->words->dresult[2]);
  if (n == 0 || incx == 0) {   // sasum.rs: n == 0 || incx == 0 -> 0
    CORAL_CUDA(H, cudaMemsetAsync(dres, 0, sizeof(R), H->stream));
    return deliver_result(H, result, dres, sizeof(R));
  }
  if (!x) return bad_arg(H, 2);
  if ((uintptr_t)x & (align - 1)) return bad_arg(H, 2);
  double* part = static_cast<double*>(scratch(H, max_l1_blocks(H) * sizeof(double)));
  if (!part) return CORAL_ERR_ALLOC;
  const T* xx = static_cast<const T*>(x);
  unsigned* ctr = &H->words->counters[kCtrMisc];
  if (unit_ok(incx, 1, x, x))
    l1_launch(H, n, k_asum_x<T, R, true>, n, xx, 1, part, ctr, dres);
  else
    l1_launch(H, n, k_asum_x<T, R, false>, n, xx, incx, part, ctr, dres);
  return finish(H, result, dres, sizeof(R));
}

template <typename T, typename R>
coral_status_t nrm2_entry(coral_handle_t hh, size_t n, const void* x, size_t incx, R* result, size_t align) {
  CORAL_HANDLE(hh);
  if (!result) return bad_arg(H, 4);
  R* dres = reinterpret_cast<R*>(&H->words->dresult[2]);
  if (n == 0 || incx == 0) {   // dnrm2.rs: n == 0 || incx == 0 -> 0
    CORAL_CUDA(H, cudaMemsetAsync(dres, 0, sizeof(R), H->stream));
    return deliver_result(H, result, dres, sizeof(R));
  }
  if (!x) return bad_arg(H, 2);
  if ((uintptr_t)x & (align - 1)) return bad_arg(H, 2);
  double* part = static_cast<double*>(scratch(H, max_l1_blocks(H) * 2 * sizeof(double)));
  if (!part) return CORAL_ERR_ALLOC;
  unsigned* flag = &H->words->counters[kCtrMisc + 1];
  double* dmx = &H->words->dresult[3];
  const T* xx = static_cast<const T*>(x);
  unsigned* ctr = &H->words->counters[kCtrMisc];
  const bool unit = unit_ok(incx, 1, x, x);
  if (unit)
    l1_launch(H, n, k_nrm2_x<T, R, true>, n, xx, 1, part, ctr, flag, dmx, dres);
  else
    l1_launch(H, n, k_nrm2_x<T, R, false>, n, xx, incx, part, ctr, flag, dmx, dres);
  coral_status_t s = launch_status(H);
  if (s != CORAL_OK) return s;
  if (sizeof(R) == 8) {   // fp64 data: rescaling pass (returns at once unless asked)
    const double* cmx = dmx;
    if (unit)
      CORAL_CUDA(H, l1_launch_dependent(H, n, k_nrm2_scaled<T, R, true>, n, xx, (size_t)1, part, ctr, flag, cmx,
                                        dres));
    else
      CORAL_CUDA(H, l1_launch_dependent(H, n, k_nrm2_scaled<T, R, false>, n, xx, incx, part, ctr, flag, cmx,
                                        dres));
  }
  return finish(H, result, dres, sizeof(R));
}

template <typename T>
coral_status_t iamax_entry(coral_handle_t hh, size_t n, const void* x, size_t incx, size_t* index, size_t align) {
  CORAL_HANDLE(hh);
  if (!index) return bad_arg(H, 4);
  unsigned long long* dres = &H->words->uresult[1];
  if (n == 0 || incx == 0) {   // idamax.rs: n == 0 || incx <= 0 -> 0
    CORAL_CUDA(H, cudaMemsetAsync(dres, 0, sizeof(unsigned long long), H->stream));
    return deliver_result(H, index, dres, sizeof(size_t));
  }
  if (!x) return bad_arg(H, 2);
  if ((uintptr_t)x & (align - 1)) return bad_arg(H, 2);
  char* sc = static_cast<char*>(scratch(H, max_l1_blocks(H) * 16));
  if (!sc) return CORAL_ERR_ALLOC;
  double* pv = reinterpret_cast<double*>(sc);
  unsigned long long* pi = reinterpret_cast<unsigned long long*>(sc + max_l1_blocks(H) * 8);
  const T* xx = static_cast<const T*>(x);
  unsigned* ctr = &H->words->counters[kCtrMisc];
  if (unit_ok(incx, 1, x, x))
    l1_launch(H, n, k_iamax_x<T, true>, n, xx, 1, pv, pi, ctr, dres);
  else
    l1_launch(H, n, k_iamax_x<T, false>, n, xx, incx, pv, pi, ctr, dres);
  return finish(H, index, dres, sizeof(size_t));
}

// n - n % W on unit strides (the reference's vector body), else 0
size_t fused_len(size_t n, size_t incx, size_t incy, size_t w) {
  return incx == 1 && incy == 1 ? n - n % w : 0;
}

template <typename T>
coral_status_t axpy_entry(coral_handle_t hh, size_t n, T alpha, bool alpha_zero, const void* x, size_t incx,
                          void* y, size_t incy, size_t align, size_t w) {
  CORAL_HANDLE(hh);
  if (n == 0 || alpha_zero) return CORAL_OK;   // caxpy.rs quick return
  if (!x) return bad_arg(H, 3);
  if (incx == 0) return bad_arg(H, 4);
  if (!y) return bad_arg(H, 5);
  if (incy == 0) return bad_arg(H, 6);
  if (((uintptr_t)x | (uintptr_t)y) & (align - 1)) return bad_arg(H, 3);
  const size_t nf = fused_len(n, incx, incy, w);
  const T* xx = static_cast<const T*>(x);
  T* yy = static_cast<T*>(y);
  if (unit_ok(incx, incy, x, y))
    l1_launch(H, n, k_axpy_x<T, true>, n, nf, alpha, xx, 1, yy, 1);
  else
    l1_launch(H, n, k_axpy_x<T, false>, n, nf, alpha, xx, incx, yy, incy);
  return launch_status(H);
}

template <typename T, bool kReal>
coral_status_t scal_entry(coral_handle_t hh, size_t n, T alpha, void* x, size_t incx, size_t align, size_t w) {
  CORAL_HANDLE(hh);
  if (n == 0 || incx == 0) return CORAL_OK;   // cscal.rs / zdscal.rs quick return
  if (!x) return bad_arg(H, 3);
  if ((uintptr_t)x & (align - 1)) return bad_arg(H, 3);
  const size_t nf = fused_len(n, incx, 1, w);
  T* xx = static_cast<T*>(x);
  if (unit_ok(incx, 1, x, x))
    l1_launch(H, n, k_scal_x<T, kReal, true>, n, nf, alpha, xx, 1);
  else
    l1_launch(H, n, k_scal_x<T, kReal, false>, n, nf, alpha, xx, incx);
  return launch_status(H);
}

template <typename E>
coral_status_t copy_entry(coral_handle_t hh, size_t n, const void* x, size_t incx, void* y, size_t incy,
                          bool swap) {
  CORAL_HANDLE(hh);
  if (n == 0) return CORAL_OK;   // dcopy.rs / dswap.rs
  if (!x) return bad_arg(H, 2);
  if (incx == 0) return bad_arg(H, 3);
  if (!y) return bad_arg(H, 4);
  if (incy == 0) return bad_arg(H, 5);
  if (((uintptr_t)x | (uintptr_t)y) & (alignof(E) - 1)) return bad_arg(H, 2);
  E* xx = static_cast<E*>(const_cast<void*>(x));
  E* yy = static_cast<E*>(y);
  const bool unit = unit_ok(incx, incy, x, y);
  if (swap) {
    if (unit) l1_launch(H, n, k_swap_x<E, true>, n, xx, 1, yy, 1);
    else l1_launch(H, n, k_swap_x<E, false>, n, xx, incx, yy, incy);
  } else {
    if (unit) l1_launch(H, n, k_copy_x<E, true>, n, xx, 1, yy, 1);
    else l1_launch(H, n, k_copy_x<E, false>, n, xx, incx, yy, incy);
  }
  return launch_status(H);
}

template <typename T, typename R>
coral_status_t rot_entry(coral_handle_t hh, size_t n, void* x, size_t incx, void* y, size_t incy, R c, R s,
                         size_t align, size_t w) {
  CORAL_HANDLE(hh);
  if (n == 0) return CORAL_OK;   // srot.rs / csrot.rs
  if (!x) return bad_arg(H, 2);
  if (incx == 0) return bad_arg(H, 3);
  if (!y) return bad_arg(H, 4);
  if (incy == 0) return bad_arg(H, 5);
  if (((uintptr_t)x | (uintptr_t)y) & (align - 1)) return bad_arg(H, 2);
  const size_t nf = fused_len(n, incx, incy, w);
  T* xx = static_cast<T*>(x);
  T* yy = static_cast<T*>(y);
  if (unit_ok(incx, incy, x, y))
    l1_launch(H, n, k_rot_x<T, R, true>, n, nf, xx, 1, yy, 1, c, s);
  else
    l1_launch(H, n, k_rot_x<T, R, false>, n, nf, xx, incx, yy, incy, c, s);
  return launch_status(H);
}

template <typename R>
coral_status_t rotm_entry(coral_handle_t hh, size_t n, R* x, size_t incx, R* y, size_t incy, const R param[5],
                          size_t w) {
  CORAL_HANDLE(hh);
  if (!param) return bad_arg(H, 6);
  if (n == 0) return CORAL_OK;           // srotm.rs:9-11
  if (param[0] == (R)-2) return CORAL_OK;
  if (!x) return bad_arg(H, 2);
  if (incx == 0) return bad_arg(H, 3);
  if (!y) return bad_arg(H, 4);
  if (incy == 0) return bad_arg(H, 5);
  if (((uintptr_t)x | (uintptr_t)y) & (sizeof(R) - 1)) return bad_arg(H, 2);
  const size_t nf = fused_len(n, incx, incy, w);
  if (unit_ok(incx, incy, x, y))
    l1_launch(H, n, k_rotm_x<R, true>, n, nf, x, 1, y, 1, param[0], param[1], param[2],
                                                             param[3], param[4]);
  else
    l1_launch(H, n, k_rotm_x<R, false>, n, nf, x, incx, y, incy, param[0], param[1],
                                                              param[2], param[3], param[4]);
  return launch_status(H);
}

// rotation constructors: in host pointer mode the scalars go through the
// handle's device words; in device pointer mode they are used in place
template <typename R>
coral_status_t rotg_entry(coral_handle_t hh, R* a, R* b, R* c, R* s) {
  CORAL_HANDLE(hh);
  if (!a || !b || !c || !s) return bad_arg(H, !a ? 1 : !b ? 2 : !c ? 3 : 4);
  if (H->pointer_mode == CORAL_POINTER_DEVICE) {
    k_rotg<R><<<1, 1, 0, H->stream>>>(a, b, c, s);
    return launch_status(H);
  }
  R* d = reinterpret_cast<R*>(stage(H));
  const R in[2] = {*a, *b};
  CORAL_CUDA(H, cudaMemcpyAsync(d, in, sizeof(in), cudaMemcpyHostToDevice, H->stream));
  k_rotg<R><<<1, 1, 0, H->stream>>>(d, d + 1, d + 2, d + 3);
  coral_status_t st = launch_status(H);
  if (st != CORAL_OK) return st;
  R out[4];
  CORAL_CUDA(H, cudaMemcpyAsync(H->host_pinned, d, sizeof(out), cudaMemcpyDeviceToHost, H->stream));
  CORAL_CUDA(H, cudaStreamSynchronize(H->stream));
  std::memcpy(out, H->host_pinned, sizeof(out));
  *a = out[0]; *b = out[1]; *c = out[2]; *s = out[3];
  return CORAL_OK;
}

template <typename R>
coral_status_t rotmg_entry(coral_handle_t hh, R* d1, R* d2, R* x1, R y1, R* param) {
  CORAL_HANDLE(hh);
  if (!d1 || !d2 || !x1 || !param) return bad_arg(H, !d1 ? 1 : !d2 ? 2 : !x1 ? 3 : 5);
  if (H->pointer_mode == CORAL_POINTER_DEVICE) {
    k_rotmg<R><<<1, 1, 0, H->stream>>>(d1, d2, x1, y1, param);
    return launch_status(H);
  }
  R* d = reinterpret_cast<R*>(stage(H));   // d1 d2 x1 | param[5]
  R in[8] = {*d1, *d2, *x1, param[0], param[1], param[2], param[3], param[4]};
  CORAL_CUDA(H, cudaMemcpyAsync(d, in, sizeof(in), cudaMemcpyHostToDevice, H->stream));
  k_rotmg<R><<<1, 1, 0, H->stream>>>(d, d + 1, d + 2, y1, d + 3);
  coral_status_t st = launch_status(H);
  if (st != CORAL_OK) return st;
  CORAL_CUDA(H, cudaMemcpyAsync(H->host_pinned, d, sizeof(in), cudaMemcpyDeviceToHost, H->stream));
  CORAL_CUDA(H, cudaStreamSynchronize(H->stream));
  R out[8];
  std::memcpy(out, H->host_pinned, sizeof(out));
  *d1 = out[0]; *d2 = out[1]; *x1 = out[2];
  for (int i = 0; i < 5; ++i) param[i] = out[3 + i];
  return CORAL_OK;
}

}  // namespace

extern "C" {

// ---- dot ----
coral_status_t coral_ddot(coral_handle_t h, size_t n, const double* x, size_t incx, const double* y, size_t incy,
                          double* result) {
  return dot_entry<double, false>(h, n, x, incx, y, incy, result, 8);
}
coral_status_t coral_cdotu(coral_handle_t h, size_t n, const float* x, size_t incx, const float* y, size_t incy,
                           float result[2]) {
  return dot_entry<float2, false>(h, n, x, incx, y, incy, result, 8);
}
coral_status_t coral_cdotc(coral_handle_t h, size_t n, const float* x, size_t incx, const float* y, size_t incy,
                           float result[2]) {
  return dot_entry<float2, true>(h, n, x, incx, y, incy, result, 8);
}
coral_status_t coral_zdotu(coral_handle_t h, size_t n, const double* x, size_t incx, const double* y,
                           size_t incy, double result[2]) {
  return dot_entry<double2, false>(h, n, x, incx, y, incy, result, 16);
}
coral_status_t coral_zdotc(coral_handle_t h, size_t n, const double* x, size_t incx, const double* y,
                           size_t incy, double result[2]) {
  return dot_entry<double2, true>(h, n, x, incx, y, incy, result, 16);
}

// ---- asum ----
coral_status_t coral_sasum(coral_handle_t h, size_t n, const float* x, size_t incx, float* result) {
  return asum_entry<float, float>(h, n, x, incx, result, 4);
}
coral_status_t coral_dasum(coral_handle_t h, size_t n, const double* x, size_t incx, double* result) {
  return asum_entry<double, double>(h, n, x, incx, result, 8);
}
coral_status_t coral_scasum(coral_handle_t h, size_t n, const float* x, size_t incx, float* result) {
  return asum_entry<float2, float>(h, n, x, incx, result, 8);
}
coral_status_t coral_dzasum(coral_handle_t h, size_t n, const double* x, size_t incx, double* result) {
  return asum_entry<double2, double>(h, n, x, incx, result, 16);
}

// ---- nrm2 ----
coral_status_t coral_dnrm2(coral_handle_t h, size_t n, const double* x, size_t incx, double* result) {
  return nrm2_entry<double, double>(h, n, x, incx, result, 8);
}
coral_status_t coral_scnrm2(coral_handle_t h, size_t n, const float* x, size_t incx, float* result) {
  return nrm2_entry<float2, float>(h, n, x, incx, result, 8);
}
coral_status_t coral_dznrm2(coral_handle_t h, size_t n, const double* x, size_t incx, double* result) {
  return nrm2_entry<double2, double>(h, n, x, incx, result, 16);
}
// snrm2.rs:45-149: the fp32 norm on the same streaming reduction (fp64 sum
// of squares of the fp32 values, which cannot overflow, then sqrt).
coral_status_t coral_snrm2(coral_handle_t h, size_t n, const float* x, size_t incx, float* result) {
  return nrm2_entry<float, float>(h, n, x, incx, result, 4);
}

// ---- i?amax ----
coral_status_t coral_idamax(coral_handle_t h, size_t n, const double* x, size_t incx, size_t* index) {
  return iamax_entry<double>(h, n, x, incx, index, 8);
}
coral_status_t coral_icamax(coral_handle_t h, size_t n, const float* x, size_t incx, size_t* index) {
  return iamax_entry<float2>(h, n, x, incx, index, 8);
}
coral_status_t coral_izamax(coral_handle_t h, size_t n, const double* x, size_t incx, size_t* index) {
  return iamax_entry<double2>(h, n, x, incx, index, 16);
}

// ---- axpy ----
coral_status_t coral_daxpy(coral_handle_t h, size_t n, double alpha, const double* x, size_t incx, double* y,
                           size_t incy) {
  return axpy_entry<double>(h, n, alpha, alpha == 0.0, x, incx, y, incy, 8, 4);   // daxpy.rs: 8- and 4-wide
}
coral_status_t coral_caxpy(coral_handle_t h, size_t n, const float alpha[2], const float* x, size_t incx,
                           float* y, size_t incy) {
  if (!alpha) return CORAL_ERR_INVALID_ARG;
  return axpy_entry<float2>(h, n, make_float2(alpha[0], alpha[1]), alpha[0] == 0.f && alpha[1] == 0.f, x, incx,
                            y, incy, 8, 4);
}
coral_status_t coral_zaxpy(coral_handle_t h, size_t n, const double alpha[2], const double* x, size_t incx,
                           double* y, size_t incy) {
  if (!alpha) return CORAL_ERR_INVALID_ARG;
  return axpy_entry<double2>(h, n, make_double2(alpha[0], alpha[1]), alpha[0] == 0.0 && alpha[1] == 0.0, x,
                             incx, y, incy, 16, 2);
}

// ---- scal ----
coral_status_t coral_dscal(coral_handle_t h, size_t n, double alpha, double* x, size_t incx) {
  return scal_entry<double, true>(h, n, alpha, x, incx, 8, 1);
}
coral_status_t coral_cscal(coral_handle_t h, size_t n, const float alpha[2], float* x, size_t incx) {
  if (!alpha) return CORAL_ERR_INVALID_ARG;
  return scal_entry<float2, false>(h, n, make_float2(alpha[0], alpha[1]), x, incx, 8, 4);
}
coral_status_t coral_zscal(coral_handle_t h, size_t n, const double alpha[2], double* x, size_t incx) {
  if (!alpha) return CORAL_ERR_INVALID_ARG;
  return scal_entry<double2, false>(h, n, make_double2(alpha[0], alpha[1]), x, incx, 16, 2);
}
coral_status_t coral_csscal(coral_handle_t h, size_t n, float alpha, float* x, size_t incx) {
  return scal_entry<float2, true>(h, n, make_float2(alpha, 0.f), x, incx, 8, 1);
}
coral_status_t coral_zdscal(coral_handle_t h, size_t n, double alpha, double* x, size_t incx) {
  return scal_entry<double2, true>(h, n, make_double2(alpha, 0.0), x, incx, 16, 1);
}

// ---- copy / swap ----
coral_status_t coral_dcopy(coral_handle_t h, size_t n, const double* x, size_t incx, double* y, size_t incy) {
  return copy_entry<double>(h, n, x, incx, y, incy, false);
}
coral_status_t coral_ccopy(coral_handle_t h, size_t n, const float* x, size_t incx, float* y, size_t incy) {
  return copy_entry<float2>(h, n, x, incx, y, incy, false);
}
coral_status_t coral_zcopy(coral_handle_t h, size_t n, const double* x, size_t incx, double* y, size_t incy) {
  return copy_entry<double2>(h, n, x, incx, y, incy, false);
}
coral_status_t coral_dswap(coral_handle_t h, size_t n, double* x, size_t incx, double* y, size_t incy) {
  return copy_entry<double>(h, n, x, incx, y, incy, true);
}
coral_status_t coral_cswap(coral_handle_t h, size_t n, float* x, size_t incx, float* y, size_t incy) {
  return copy_entry<float2>(h, n, x, incx, y, incy, true);
}
coral_status_t coral_zswap(coral_handle_t h, size_t n, double* x, size_t incx, double* y, size_t incy) {
  return copy_entry<double2>(h, n, x, incx, y, incy, true);
}
// sswap.rs:35: the fp32 swap on the same streaming kernel (a pure
// exchange, so bit-exact).
coral_status_t coral_sswap(coral_handle_t h, size_t n, float* x, size_t incx, float* y, size_t incy) {
  return copy_entry<float>(h, n, x, incx, y, incy, true);
}

// ---- rotations ----
coral_status_t coral_srot(coral_handle_t h, size_t n, float* x, size_t incx, float* y, size_t incy, float c,
                          float s) {
  return rot_entry<float, float>(h, n, x, incx, y, incy, c, s, 4, 4);
}
coral_status_t coral_drot(coral_handle_t h, size_t n, double* x, size_t incx, double* y, size_t incy, double c,
                          double s) {
  return rot_entry<double, double>(h, n, x, incx, y, incy, c, s, 8, 2);
}
coral_status_t coral_csrot(coral_handle_t h, size_t n, float* x, size_t incx, float* y, size_t incy, float c,
                           float s) {
  return rot_entry<float2, float>(h, n, x, incx, y, incy, c, s, 8, 2);
}
coral_status_t coral_zdrot(coral_handle_t h, size_t n, double* x, size_t incx, double* y, size_t incy, double c,
                           double s) {
  return rot_entry<double2, double>(h, n, x, incx, y, incy, c, s, 16, 1);
}
coral_status_t coral_srotm(coral_handle_t h, size_t n, float* x, size_t incx, float* y, size_t incy,
                           const float param[5]) {
  return rotm_entry<float>(h, n, x, incx, y, incy, param, 4);
}
coral_status_t coral_drotm(coral_handle_t h, size_t n, double* x, size_t incx, double* y, size_t incy,
                           const double param[5]) {
  return rotm_entry<double>(h, n, x, incx, y, incy, param, 2);
}
coral_status_t coral_srotg(coral_handle_t h, float* a, float* b, float* c, float* s) {
  return rotg_entry<float>(h, a, b, c, s);
}
coral_status_t coral_drotg(coral_handle_t h, double* a, double* b, double* c, double* s) {
  return rotg_entry<double>(h, a, b, c, s);
}
coral_status_t coral_srotmg(coral_handle_t h, float* d1, float* d2, float* x1, float y1, float param[5]) {
  return rotmg_entry<float>(h, d1, d2, x1, y1, param);
}
coral_status_t coral_drotmg(coral_handle_t h, double* d1, double* d2, double* x1, double y1, double param[5]) {
  return rotmg_entry<double>(h, d1, d2, x1, y1, param);
}

}  // extern "C"
