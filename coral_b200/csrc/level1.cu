// Level-1 routines: HBM-streaming kernels with 128-bit loads on the unit-stride
// path and single-launch deterministic reductions (per-block partials, the
// last block to arrive combines them in a fixed order).
//
// Semantics follow coral-aarch64/src/level1 (file:line cited per routine).
#include "common.cuh"

#include <cfloat>

namespace coral {
namespace {

constexpr int kRedThreads = 512;  // 4 blocks x 512 = 2048 threads per SM

struct ArgBest {
  float v;
  unsigned long long i;
};

__device__ __forceinline__ bool better(const ArgBest& a, const ArgBest& b) {
  return a.v > b.v || (a.v == b.v && a.i < b.i);
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

__device__ __forceinline__ ArgBest warp_best(ArgBest a) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    ArgBest b;
    b.v = __shfl_xor_sync(0xffffffffu, a.v, o);
    b.i = __shfl_xor_sync(0xffffffffu, a.i, o);
    if (better(b, a)) a = b;
  }
  return a;
}

// Fixed-order block sum (warp shuffles, then warp 0 over the warp sums).
__device__ double block_sum(double v, double* sh) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  v = warp_sum(v);
  if (lane == 0) sh[warp] = v;
  __syncthreads();
  double r = 0.0;
  if (warp == 0) {
    r = lane < (int)(blockDim.x >> 5) ? sh[lane] : 0.0;
    r = warp_sum(r);
  }
  __syncthreads();
  return r;  // valid in thread 0
}

__device__ ArgBest block_best(ArgBest a, ArgBest* sh) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  a = warp_best(a);
  if (lane == 0) sh[warp] = a;
  __syncthreads();
  ArgBest r{-INFINITY, ~0ull};
  if (warp == 0) {
    if (lane < (int)(blockDim.x >> 5)) r = sh[lane];
    r = warp_best(r);
  }
  __syncthreads();
  return r;
}

// Returns true in every thread of the block that arrives last at `counter`
// (after its partial was published); that block resets the counter.
__device__ bool last_block(unsigned* counter) {
  __shared__ bool is_last;
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    unsigned ticket = atomicAdd(counter, 1u);
    is_last = (ticket == gridDim.x - 1);
  }
  __syncthreads();
  return is_last;
}

// ---- sdot --------------------------------------------------------------------
// Each product of two fp32 values is exact in fp64; the sum is accumulated in
// fp64.  (snrm2 runs on the streaming reduction of level1_dcz.cu: an fp64 sum
// of fp32 squares can neither overflow nor underflow, which gives it the
// overflow safety of the reference's running (scale, ssq) pair,
// nrm2_helpers.rs:15-38, in a single pass.)
template <bool kVec>
__global__ void __launch_bounds__(kRedThreads)
k_dot(size_t n, const float* __restrict__ x, size_t incx, const float* __restrict__ y,
      size_t incy, double* partials, unsigned* counter, float* out) {
  __shared__ double sh[32];
  const size_t tid = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  const size_t stride = (size_t)gridDim.x * blockDim.x;
  double acc = 0.0;
  if (kVec) {
    const size_t n4 = n >> 2;
    const float4* x4 = reinterpret_cast<const float4*>(x);
    const float4* y4 = reinterpret_cast<const float4*>(y);
    // 8 independent 128-bit loads in flight per thread, 4 per operand
    constexpr int U = 4;
    size_t i = tid;
    double acc1 = 0.0;
    for (; i + (U - 1) * stride < n4; i += U * stride) {
      float4 a[U], b[U];
#pragma unroll
      for (int u = 0; u < U; ++u) a[u] = __ldcs(x4 + i + u * stride);
#pragma unroll
      for (int u = 0; u < U; ++u) b[u] = __ldcs(y4 + i + u * stride);
#pragma unroll
      for (int u = 0; u < U; ++u) {
        double& t = (u & 1) ? acc1 : acc;
        t += (double)a[u].x * b[u].x + (double)a[u].y * b[u].y + (double)a[u].z * b[u].z +
             (double)a[u].w * b[u].w;
      }
    }
    for (; i < n4; i += stride) {
      const float4 a = __ldcs(x4 + i), b = __ldcs(y4 + i);
      acc += (double)a.x * b.x + (double)a.y * b.y + (double)a.z * b.z + (double)a.w * b.w;
    }
    acc += acc1;
    for (size_t t = (n4 << 2) + tid; t < n; t += stride) acc += (double)x[t] * y[t];
  } else {
    for (size_t t = tid; t < n; t += stride) acc += (double)x[t * incx] * y[t * incy];
  }
  double bs = block_sum(acc, sh);
  if (threadIdx.x == 0) partials[blockIdx.x] = bs;
  if (!last_block(counter)) return;
  double s = 0.0;
  for (unsigned b = threadIdx.x; b < gridDim.x; b += blockDim.x) s += __ldcg(partials + b);
  s = block_sum(s, sh);
  if (threadIdx.x == 0) {
    *out = (float)s;
    *counter = 0;
  }
}

// ---- isamax ---------------------------------------------------------------
// First index of max |x_i|; NaN never wins (isamax.rs:72-76 maps NaN to -inf,
// the scalar paths' `v > best` rejects it); nothing valid -> index 0.
template <bool kVec>
__global__ void __launch_bounds__(kRedThreads)
k_iamax(size_t n, const float* __restrict__ x, size_t incx, float* pv,
        unsigned long long* pi, unsigned* counter, unsigned long long* out) {
  __shared__ ArgBest sh[32];
  const size_t tid = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  const size_t stride = (size_t)gridDim.x * blockDim.x;
  ArgBest best{-INFINITY, ~0ull};
  if (kVec) {
    const size_t n4 = n >> 2;
    const float4* x4 = reinterpret_cast<const float4*>(x);
    size_t i = tid;
    for (; i + 3 * stride < n4; i += 4 * stride) {  // 4 loads in flight, scanned in index order
      float4 a[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) a[u] = __ldcs(x4 + i + u * stride);
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const float v[4] = {fabsf(a[u].x), fabsf(a[u].y), fabsf(a[u].z), fabsf(a[u].w)};
#pragma unroll
        for (int e = 0; e < 4; ++e)
          if (v[e] > best.v) { best.v = v[e]; best.i = ((i + u * stride) << 2) + e; }
      }
    }
    for (; i < n4; i += stride) {
      float4 a = __ldcs(x4 + i);
      float v[4] = {fabsf(a.x), fabsf(a.y), fabsf(a.z), fabsf(a.w)};
#pragma unroll
      for (int e = 0; e < 4; ++e)
        if (v[e] > best.v) { best.v = v[e]; best.i = (i << 2) + e; }
    }
    for (size_t t = (n4 << 2) + tid; t < n; t += stride) {
      float v = fabsf(x[t]);
      if (v > best.v) { best.v = v; best.i = t; }
    }
  } else {
    for (size_t t = tid; t < n; t += stride) {
      float v = fabsf(x[t * incx]);
      if (v > best.v) { best.v = v; best.i = t; }
    }
  }
  ArgBest bb = block_best(best, sh);
  if (threadIdx.x == 0) { pv[blockIdx.x] = bb.v; pi[blockIdx.x] = bb.i; }
  if (!last_block(counter)) return;
  ArgBest r{-INFINITY, ~0ull};
  for (unsigned b = threadIdx.x; b < gridDim.x; b += blockDim.x) {
    ArgBest c{__ldcg(pv + b), __ldcg(pi + b)};
    if (better(c, r)) r = c;
  }
  r = block_best(r, sh);
  if (threadIdx.x == 0) {
    *out = (r.i == ~0ull) ? 0ull : r.i;
    *counter = 0;
  }
}

// ---- saxpy ----------------------------------------------------------------
// Bit-exact with saxpy.rs:42-131: on the unit-stride path the 16/8-wide NEON
// body (elements below n - n % 8) uses a fused multiply-add, the scalar tail
// and every strided element use `y += alpha * x` with two roundings.
__global__ void k_saxpy_unit(size_t n, float alpha, const float* __restrict__ x,
                             float* __restrict__ y, bool vec) {
  const size_t tid = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  const size_t stride = (size_t)gridDim.x * blockDim.x;
  const size_t nfused = n - (n & 7);
  size_t done = 0;
  if (vec) {
    const size_t n4 = nfused >> 2;  // nfused is a multiple of 8
    const float4* x4 = reinterpret_cast<const float4*>(x);
    float4* y4 = reinterpret_cast<float4*>(y);
    for (size_t i = tid; i < n4; i += stride) {
      float4 a = __ldcs(x4 + i), b = __ldcs(y4 + i);
      b.x = fmaf(alpha, a.x, b.x);
      b.y = fmaf(alpha, a.y, b.y);
      b.z = fmaf(alpha, a.z, b.z);
      b.w = fmaf(alpha, a.w, b.w);
      __stcs(y4 + i, b);
    }
    done = nfused;
  }
  for (size_t t = done + tid; t < n; t += stride) {
    float r = t < nfused ? fmaf(alpha, x[t], y[t]) : __fadd_rn(y[t], __fmul_rn(alpha, x[t]));
    y[t] = r;
  }
}

__global__ void k_saxpy_strided(size_t n, float alpha, const float* __restrict__ x, size_t incx,
                                float* __restrict__ y, size_t incy) {
  const size_t stride = (size_t)gridDim.x * blockDim.x;
  for (size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += stride)
    y[t * incy] = __fadd_rn(y[t * incy], __fmul_rn(alpha, x[t * incx]));
}

// ---- sscal / scopy / sswap --------------------------------------------------
__global__ void k_sscal(size_t n, float alpha, float* __restrict__ x, size_t incx, bool vec) {
  const size_t tid = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  const size_t stride = (size_t)gridDim.x * blockDim.x;
  size_t done = 0;
  if (vec) {
    const size_t n4 = n >> 2;
    float4* x4 = reinterpret_cast<float4*>(x);
    for (size_t i = tid; i < n4; i += stride) {
      float4 a = __ldcs(x4 + i);
      a.x = __fmul_rn(a.x, alpha);
      a.y = __fmul_rn(a.y, alpha);
      a.z = __fmul_rn(a.z, alpha);
      a.w = __fmul_rn(a.w, alpha);
      __stcs(x4 + i, a);
    }
    done = n4 << 2;
  }
  for (size_t t = done + tid; t < n; t += stride) x[t * incx] = __fmul_rn(x[t * incx], alpha);
}

__global__ void k_scopy_strided(size_t n, const float* __restrict__ x, size_t incx,
                                float* __restrict__ y, size_t incy) {
  const size_t stride = (size_t)gridDim.x * blockDim.x;
  for (size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += stride)
    y[t * incy] = x[t * incx];
}

}  // namespace

// Enqueue helpers shared with level 2 (GEMV's beta step is sscal).
coral_status_t enqueue_sscal(Handle* h, size_t n, float alpha, float* x, size_t incx) {
  bool vec = incx == 1 && aligned16(x);
  unsigned g = stream_grid(n, 256 * 4 * 4, h->sm_count, 8);
  k_sscal<<<g, 256, 0, h->stream>>>(n, alpha, x, incx, vec);
  return launch_status(h);
}

}  // namespace coral

using namespace coral;

extern "C" {

coral_status_t coral_sdot(coral_handle_t hh, size_t n, const float* x, size_t incx,
                          const float* y, size_t incy, float* result) {
  CORAL_HANDLE(hh);
  if (!result) return bad_arg(H, 7);
  DeviceWords* w = H->words;
  float* dres = reinterpret_cast<float*>(&w->dresult[0]);
  if (n == 0) {  // sdot.rs:50
    CORAL_CUDA(H, cudaMemsetAsync(dres, 0, sizeof(float), H->stream));
    return deliver_result(H, result, dres, sizeof(float));
  }
  if (!x) return bad_arg(H, 2);
  if (incx == 0) return bad_arg(H, 3);
  if (!y) return bad_arg(H, 4);
  if (incy == 0) return bad_arg(H, 5);
  bool vec = incx == 1 && incy == 1 && aligned16(x) && aligned16(y);
  unsigned g = stream_grid(n, (size_t)kRedThreads * 8, H->sm_count, 4);
  double* part = static_cast<double*>(scratch(H, g * sizeof(double)));
  if (!part) return CORAL_ERR_ALLOC;
  if (vec)
    k_dot<true><<<g, kRedThreads, 0, H->stream>>>(n, x, 1, y, 1, part, &w->counters[kCtrDot], dres);
  else
    k_dot<false><<<g, kRedThreads, 0, H->stream>>>(n, x, incx, y, incy, part, &w->counters[kCtrDot], dres);
  coral_status_t s = launch_status(H);
  if (s != CORAL_OK) return s;
  return deliver_result(H, result, dres, sizeof(float));
}

coral_status_t coral_isamax(coral_handle_t hh, size_t n, const float* x, size_t incx,
                            size_t* index) {
  CORAL_HANDLE(hh);
  if (!index) return bad_arg(H, 4);
  DeviceWords* w = H->words;
  unsigned long long* dres = &w->uresult[0];
  if (n == 0 || incx == 0) {  // isamax.rs:48
    CORAL_CUDA(H, cudaMemsetAsync(dres, 0, sizeof(unsigned long long), H->stream));
    return deliver_result(H, index, dres, sizeof(size_t));
  }
  if (!x) return bad_arg(H, 2);
  bool vec = incx == 1 && aligned16(x);
  unsigned g = stream_grid(n, (size_t)kRedThreads * 8, H->sm_count, 4);
  char* sc = static_cast<char*>(scratch(H, (size_t)g * 16));
  if (!sc) return CORAL_ERR_ALLOC;
  unsigned long long* pi = reinterpret_cast<unsigned long long*>(sc);
  float* pv = reinterpret_cast<float*>(sc + (size_t)g * 8);
  if (vec)
    k_iamax<true><<<g, kRedThreads, 0, H->stream>>>(n, x, 1, pv, pi, &w->counters[kCtrIamax], dres);
  else
    k_iamax<false><<<g, kRedThreads, 0, H->stream>>>(n, x, incx, pv, pi, &w->counters[kCtrIamax], dres);
  coral_status_t s = launch_status(H);
  if (s != CORAL_OK) return s;
  return deliver_result(H, index, dres, sizeof(size_t));
}

coral_status_t coral_saxpy(coral_handle_t hh, size_t n, float alpha, const float* x,
                           size_t incx, float* y, size_t incy) {
  CORAL_HANDLE(hh);
  if (n == 0 || alpha == 0.0f) return CORAL_OK;  // saxpy.rs:51-53
  if (!x) return bad_arg(H, 3);
  if (incx == 0) return bad_arg(H, 4);
  if (!y) return bad_arg(H, 5);
  if (incy == 0) return bad_arg(H, 6);
  if (incx == 1 && incy == 1) {
    bool vec = aligned16(x) && aligned16(y);
    unsigned g = stream_grid(n, 256 * 4 * 4, H->sm_count, 8);
    k_saxpy_unit<<<g, 256, 0, H->stream>>>(n, alpha, x, y, vec);
  } else {
    unsigned g = stream_grid(n, 256 * 4, H->sm_count, 8);
    k_saxpy_strided<<<g, 256, 0, H->stream>>>(n, alpha, x, incx, y, incy);
  }
  return launch_status(H);
}

coral_status_t coral_sscal(coral_handle_t hh, size_t n, float alpha, float* x, size_t incx) {
  CORAL_HANDLE(hh);
  if (n == 0 || incx == 0) return CORAL_OK;  // sscal.rs:37
  if (!x) return bad_arg(H, 3);
  return enqueue_sscal(H, n, alpha, x, incx);
}

coral_status_t coral_scopy(coral_handle_t hh, size_t n, const float* x, size_t incx, float* y,
                           size_t incy) {
  CORAL_HANDLE(hh);
  if (n == 0) return CORAL_OK;  // scopy.rs:36
  if (!x) return bad_arg(H, 2);
  if (incx == 0) return bad_arg(H, 3);
  if (!y) return bad_arg(H, 4);
  if (incy == 0) return bad_arg(H, 5);
  if (incx == 1 && incy == 1) {
    CORAL_CUDA(H, cudaMemcpyAsync(y, x, n * sizeof(float), cudaMemcpyDeviceToDevice, H->stream));
    return CORAL_OK;
  }
  unsigned g = stream_grid(n, 256 * 4, H->sm_count, 8);
  k_scopy_strided<<<g, 256, 0, H->stream>>>(n, x, incx, y, incy);
  return launch_status(H);
}


}  // extern "C"
