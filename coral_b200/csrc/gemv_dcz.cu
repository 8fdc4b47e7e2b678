// DGEMV, CGEMV, ZGEMV: y <- alpha * op(A) x + beta * y, column-major A,
// op in {N, T, C} (dgemv.rs, cgemv.rs:60-80, zgemv.rs; the *_notranspose,
// *_transpose and *_conjtranspose files).  Complex data is interleaved
// (re, im) with leading dimensions and increments in complex units.
//
// Same single-launch structure as SGEMV, templated on the element type
// (double, float2, double2): A is streamed once from HBM with 128-bit loads;
// blocks write partial sums to scratch and the last block of each output
// tile (arrival counter) adds them in a fixed order, so results are
// deterministic.
//
//   N: a block owns a 128-row strip of y and a chunk of columns; each lane
//      keeps 4 consecutive rows (one to four 16-byte loads per column).
//   T / C: a block owns a chunk of rows (alpha*x for them in shared memory)
//      and a group of columns; each warp forms whole column dot products
//      (conjugated elements for C) and reduces with shuffles.
//
// Reference semantics kept (zgemv_notranspose.rs:76-101 and the same lines
// of the other variants): quick return for an empty matrix or
// alpha == 0 && beta == 1; beta != 1 scales y by multiplication first
// (dscal; zdscal / csscal when Im(beta) == 0, else zscal / cscal), so beta
// == 0 keeps NaN; alpha == 0 then returns; x is scaled by alpha before the
// products.  Complex products use four fused multiply-adds per term.
#include "common.cuh"
#include "field.cuh"

#include <type_traits>

namespace coral {
namespace {

constexpr int kGThreads = 256;
constexpr int kGWarps = kGThreads / 32;
constexpr int kGStrip = 128;           // rows of y per N-block (32 lanes x 4)
constexpr int kGTBytes = 16384;        // bytes of alpha*x staged per T-block

__device__ bool arrive_last_g(unsigned* counter, unsigned total) {
  __shared__ bool last;
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    last = atomicAdd(counter, 1u) == total - 1;
    if (last) *counter = 0;
  }
  __syncthreads();
  if (last) __threadfence();
  return last;
}

// Four consecutive elements from a 16-byte aligned address, streaming.
__device__ __forceinline__ void load4(const double* p, double (&v)[4]) {
  const double2 a = __ldcs(reinterpret_cast<const double2*>(p));
  const double2 b = __ldcs(reinterpret_cast<const double2*>(p) + 1);
  v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y;
}
__device__ __forceinline__ void load4(const float2* p, float2 (&v)[4]) {
  const float4 a = __ldcs(reinterpret_cast<const float4*>(p));
  const float4 b = __ldcs(reinterpret_cast<const float4*>(p) + 1);
  v[0] = make_float2(a.x, a.y); v[1] = make_float2(a.z, a.w);
  v[2] = make_float2(b.x, b.y); v[3] = make_float2(b.z, b.w);
}
__device__ __forceinline__ void load4(const double2* p, double2 (&v)[4]) {
#pragma unroll
  for (int e = 0; e < 4; ++e) v[e] = __ldcs(p + e);
}

template <typename T, bool kVec>
__global__ void __launch_bounds__(kGThreads)
k_gemv_n_g(int m, int n, const T* __restrict__ A, size_t lda, const T* __restrict__ x,
           size_t incx, T alpha, T beta, int bmode, T* __restrict__ y, size_t incy,
           int cols_per_chunk, T* partials, unsigned* counters) {
  using F = Fld<T>;
  __shared__ T red[kGWarps][kGStrip];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int row0 = blockIdx.x * kGStrip;
  const int c0 = blockIdx.y * cols_per_chunk;
  const int c1 = min(n, c0 + cols_per_chunk);
  T acc[4] = {F::zero(), F::zero(), F::zero(), F::zero()};
  int rows[4];
#pragma unroll
  for (int e = 0; e < 4; ++e) rows[e] = kVec ? row0 + 4 * lane + e : row0 + lane + 32 * e;
  const bool full4 = kVec && (row0 + 4 * lane + 3 < m);
  auto load = [&](int j, T (&v)[4]) {
    const T* col = A + (size_t)j * lda;
    if (full4) {
      load4(col + rows[0], v);
    } else {
#pragma unroll
      for (int e = 0; e < 4; ++e) v[e] = rows[e] < m ? __ldcs(col + rows[e]) : F::zero();
    }
  };
  int j = c0 + warp;
  for (; j + 3 * kGWarps < c1; j += 4 * kGWarps) {
    T v[4][4], xs[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      load(j + u * kGWarps, v[u]);
      xs[u] = F::mul(alpha, __ldg(x + (size_t)(j + u * kGWarps) * incx));
    }
#pragma unroll
    for (int u = 0; u < 4; ++u)
#pragma unroll
      for (int e = 0; e < 4; ++e) F::mac(acc[e], v[u][e], xs[u]);
  }
  for (; j < c1; j += kGWarps) {
    T v[4];
    load(j, v);
    const T xs = F::mul(alpha, __ldg(x + (size_t)j * incx));
#pragma unroll
    for (int e = 0; e < 4; ++e) F::mac(acc[e], v[e], xs);
  }
#pragma unroll
  for (int e = 0; e < 4; ++e) red[warp][rows[e] - row0] = acc[e];
  __syncthreads();
  // fixed-order sum over the warps; thread t owns strip row t (t < 128)
  T s = F::zero();
  const int t = threadIdx.x;
  if (t < kGStrip) {
#pragma unroll
    for (int w = 0; w < kGWarps; ++w) s = F::add(s, red[w][t]);
  }
  const int r = row0 + t;
  if (gridDim.y == 1) {
    if (t < kGStrip && r < m) {
      T* yp = y + (size_t)r * incy;
      *yp = F::add(beta_scale(*yp, beta, bmode), s);
    }
    return;
  }
  if (t < kGStrip && r < m) partials[(size_t)blockIdx.y * m + r] = s;
  if (!arrive_last_g(counters + blockIdx.x, gridDim.y)) return;
  if (t < kGStrip && r < m) {
    T tot = F::zero();
    for (unsigned c = 0; c < gridDim.y; ++c) tot = F::add(tot, __ldcg(partials + (size_t)c * m + r));
    T* yp = y + (size_t)r * incy;
    *yp = F::add(beta_scale(*yp, beta, bmode), tot);
  }
}

// Two consecutive 8-byte elements (double or complex64) as one 16-byte load:
// streaming from global memory (load) or from shared memory (lds).
template <typename T> struct Pair;
template <> struct Pair<double> {
  static __device__ __forceinline__ void load(const double* p, double& a, double& b) {
    const double2 v = __ldcs(reinterpret_cast<const double2*>(p));
    a = v.x; b = v.y;
  }
  static __device__ __forceinline__ void lds(const double* p, double& a, double& b) {
    const double2 v = *reinterpret_cast<const double2*>(p);
    a = v.x; b = v.y;
  }
};
template <> struct Pair<float2> {
  static __device__ __forceinline__ void load(const float2* p, float2& a, float2& b) {
    const float4 v = __ldcs(reinterpret_cast<const float4*>(p));
    a = make_float2(v.x, v.y); b = make_float2(v.z, v.w);
  }
  static __device__ __forceinline__ void lds(const float2* p, float2& a, float2& b) {
    const float4 v = *reinterpret_cast<const float4*>(p);
    a = make_float2(v.x, v.y); b = make_float2(v.z, v.w);
  }
};
template <> struct Pair<double2> {  // 16-byte elements load whole already
  static __device__ __forceinline__ void load(const double2* p, double2& a, double2& b) {
    a = __ldcs(p); b = __ldcs(p + 1);
  }
  static __device__ __forceinline__ void lds(const double2* p, double2& a, double2& b) {
    a = p[0]; b = p[1];
  }
};

template <typename T, bool kConj, bool kPair>
__global__ void __launch_bounds__(kGThreads)
k_gemv_t_g(int m, int n, const T* __restrict__ A, size_t lda, const T* __restrict__ x,
           size_t incx, T alpha, T beta, int bmode, T* __restrict__ y, size_t incy,
           int rows_per_chunk, int cols_per_group, T* partials, unsigned* counters) {
  using F = Fld<T>;
  extern __shared__ __align__(16) unsigned char xs_raw[];
  T* xs = reinterpret_cast<T*>(xs_raw);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int r0 = blockIdx.y * rows_per_chunk;
  const int r1 = min(m, r0 + rows_per_chunk);
  const int nr = r1 - r0;
  for (int i = threadIdx.x; i < nr; i += blockDim.x)
    xs[i] = F::mul(alpha, __ldg(x + (size_t)(r0 + i) * incx));
  __syncthreads();
  const int g0 = blockIdx.x * cols_per_group;
  const int g1 = min(n, g0 + cols_per_group);
  auto op = [](T a) { return kConj ? F::conj(a) : a; };
  for (int j = g0 + warp; j < g1; j += kGWarps) {
    const T* col = A + (size_t)j * lda + r0;
    T acc0 = F::zero(), acc1 = F::zero();
    int i = lane;
    if (kPair) {
      // double: lane takes rows 2q, 2q + 1 with one 16-byte load (the chunk
      // start is even and the column 16-byte aligned)
      const int np = nr >> 1;
      int q = lane;
      for (; q + 96 < np; q += 128) {  // four 16-byte loads in flight per lane
        T a[4][2];
#pragma unroll
        for (int u = 0; u < 4; ++u) Pair<T>::load(col + 2 * (q + 32 * u), a[u][0], a[u][1]);
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          T x0, x1;
          Pair<T>::lds(xs + 2 * (q + 32 * u), x0, x1);
          F::mac(acc0, op(a[u][0]), x0);
          F::mac(acc1, op(a[u][1]), x1);
        }
      }
      for (; q < np; q += 32) {
        T a0, a1, x0, x1;
        Pair<T>::load(col + 2 * q, a0, a1);
        Pair<T>::lds(xs + 2 * q, x0, x1);
        F::mac(acc0, op(a0), x0);
        F::mac(acc1, op(a1), x1);
      }
      i = 2 * np + lane;  // odd tail row
    } else {
      for (; i + 96 < nr; i += 128) {
      const T a0 = __ldcs(col + i), a1 = __ldcs(col + i + 32);
      const T a2 = __ldcs(col + i + 64), a3 = __ldcs(col + i + 96);
      F::mac(acc0, op(a0), xs[i]);
      F::mac(acc1, op(a1), xs[i + 32]);
      F::mac(acc0, op(a2), xs[i + 64]);
      F::mac(acc1, op(a3), xs[i + 96]);
      }
    }
    for (; i < nr; i += 32) F::mac(acc0, op(__ldcs(col + i)), xs[i]);
    T s = F::add(acc0, acc1);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s = F::add(s, F::shfl_xor(s, o));
    if (lane == 0) {
      if (gridDim.y == 1) {
        T* yp = y + (size_t)j * incy;
        *yp = F::add(beta_scale(*yp, beta, bmode), s);
      } else {
        partials[(size_t)blockIdx.y * n + j] = s;
      }
    }
  }
  if (gridDim.y == 1) return;
  if (!arrive_last_g(counters + blockIdx.x, gridDim.y)) return;
  for (int j = g0 + threadIdx.x; j < g1; j += blockDim.x) {
    T tot = F::zero();
    for (unsigned c = 0; c < gridDim.y; ++c) tot = F::add(tot, __ldcg(partials + (size_t)c * n + j));
    T* yp = y + (size_t)j * incy;
    *yp = F::add(beta_scale(*yp, beta, bmode), tot);
  }
}

template <typename T>
__global__ void k_scal_g(size_t n, T beta, int bmode, T* __restrict__ y, size_t incy) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    y[i * incy] = beta_scale(y[i * incy], beta, bmode);
}

// op: 0 = N, 1 = T, 2 = C.  Sizes validated by the caller.
template <typename T>
coral_status_t gemv_g(Handle* h, int op, size_t m, size_t n, T alpha, bool alpha_zero, T beta,
                      int bmode, const T* A, size_t lda, const T* x, size_t incx, T* y, size_t incy) {
  if (m > INT32_MAX || n > INT32_MAX) return CORAL_ERR_NOT_SUPPORTED;
  const size_t ylen = op == 0 ? m : n;
  if (alpha_zero) {  // only the beta step
    if (bmode == 0) return CORAL_OK;
    const unsigned g = stream_grid(ylen, 256 * 4, h->sm_count, 8);
    k_scal_g<T><<<g, 256, 0, h->stream>>>(ylen, beta, bmode, y, incy);
    return launch_status(h);
  }
  const int target = h->sm_count * 8;
  if (op == 0) {
    const bool vec = (lda * sizeof(T)) % 16 == 0 && aligned16(A);
    const int strips = (int)((m + kGStrip - 1) / kGStrip);
    int chunks = (target + strips - 1) / strips;
    const int max_chunks = (int)((n + 63) / 64);
    if (chunks > max_chunks) chunks = max_chunks;
    if (chunks < 1) chunks = 1;
    const int cpc = (int)((n + chunks - 1) / chunks);
    chunks = (int)((n + cpc - 1) / cpc);
    if (strips > (int)kTrsvFlagBase) return CORAL_ERR_NOT_SUPPORTED;
    T* part = nullptr;
    if (chunks > 1) {
      part = static_cast<T*>(scratch(h, (size_t)chunks * m * sizeof(T)));
      if (!part) return CORAL_ERR_ALLOC;
    }
    const dim3 grid(strips, chunks);
    if (vec)
      k_gemv_n_g<T, true><<<grid, kGThreads, 0, h->stream>>>((int)m, (int)n, A, lda, x, incx, alpha, beta,
                                                            bmode, y, incy, cpc, part, h->counters);
    else
      k_gemv_n_g<T, false><<<grid, kGThreads, 0, h->stream>>>((int)m, (int)n, A, lda, x, incx, alpha, beta,
                                                             bmode, y, incy, cpc, part, h->counters);
    return launch_status(h);
  }
  constexpr int kRows = kGTBytes / (int)sizeof(T);
  const int rchunks = (int)((m + kRows - 1) / kRows);
  const int rpc = (int)(((m + rchunks - 1) / rchunks + 1) / 2 * 2);  // even: pairs stay aligned
  // paired 16-byte loads pay off for double (93% vs 81% of HBM); complex64
  // is faster with the one-element loop (81% vs 75%)
  const bool pair = std::is_same<T, double>::value && (lda * sizeof(T)) % 16 == 0 && aligned16(A);
  int groups = (target + rchunks - 1) / rchunks;
  const int max_groups = (int)((n + kGWarps - 1) / kGWarps);
  if (groups > max_groups) groups = max_groups;
  if (groups < 1) groups = 1;
  const int cpg = (int)((n + groups - 1) / groups);
  groups = (int)((n + cpg - 1) / cpg);
  if (groups > (int)kTrsvFlagBase) return CORAL_ERR_NOT_SUPPORTED;
  T* part = nullptr;
  if (rchunks > 1) {
    part = static_cast<T*>(scratch(h, (size_t)rchunks * n * sizeof(T)));
    if (!part) return CORAL_ERR_ALLOC;
  }
  const dim3 grid(groups, rchunks);
  const size_t smem = (size_t)rpc * sizeof(T);
#define CORAL_GEMV_T(CJ, PR)                                                                         \
  k_gemv_t_g<T, CJ, PR><<<grid, kGThreads, smem, h->stream>>>((int)m, (int)n, A, lda, x, incx, alpha, beta, \
                                                              bmode, y, incy, rpc, cpg, part, h->counters)
  if (op == 2) {
    if (pair) CORAL_GEMV_T(true, true);
    else CORAL_GEMV_T(true, false);
  } else {
    if (pair) CORAL_GEMV_T(false, true);
    else CORAL_GEMV_T(false, false);
  }
#undef CORAL_GEMV_T
  return launch_status(h);
}

// Shared argument checks (positions as in sgemv: trans 1, matrix 5, lda 6,
// x 7, incx 8, y 10, incy 11).
int gemv_bad(int trans, size_t n_rows, const void* matrix, size_t lda, const void* x, size_t incx,
             const void* y, size_t incy) {
  if (trans < CORAL_NO_TRANSPOSE || trans > CORAL_CONJ_TRANSPOSE) return 1;
  if (!matrix) return 5;
  if (lda < n_rows) return 6;
  if (!x) return 7;
  if (incx == 0) return 8;
  if (!y) return 10;
  if (incy == 0) return 11;
  return 0;
}

template <typename T, typename R>
coral_status_t complex_gemv(Handle* H, int trans, size_t n_rows, size_t n_cols, const R alpha[2],
                            const R* matrix, size_t lda, const R* x, size_t incx, const R beta[2],
                            R* y, size_t incy) {
  if (!alpha) return bad_arg(H, 4);
  if (!beta) return bad_arg(H, 9);
  if (trans < CORAL_NO_TRANSPOSE || trans > CORAL_CONJ_TRANSPOSE) return bad_arg(H, 1);
  if (n_rows == 0 || n_cols == 0) return CORAL_OK;                                   // :76
  if (alpha[0] == 0 && alpha[1] == 0 && beta[0] == 1 && beta[1] == 0) return CORAL_OK;  // :77
  if (const int bad = gemv_bad(trans, n_rows, matrix, lda, x, incx, y, incy)) return bad_arg(H, bad);
  if (((uintptr_t)matrix | (uintptr_t)x | (uintptr_t)y) % sizeof(T)) return bad_arg(H, 5);
  T a, b;
  a.x = alpha[0]; a.y = alpha[1];
  b.x = beta[0]; b.y = beta[1];
  const int bmode = (beta[0] == 1 && beta[1] == 0) ? 0 : (beta[1] == 0 ? 1 : 2);
  return gemv_g<T>(H, trans, n_rows, n_cols, a, alpha[0] == 0 && alpha[1] == 0, b, bmode,
                   reinterpret_cast<const T*>(matrix), lda, reinterpret_cast<const T*>(x), incx,
                   reinterpret_cast<T*>(y), incy);
}

// Fused level-1.5 updates (level1_special/*axpyf.rs, *dotf.rs): y += A x
// (axpyf, op 0) or out += op(A) x with op T (dotf / dotuf) or C (dotcf), on
// the GEMV kernels with alpha = beta = 1 (the beta step then leaves y alone).
// Argument positions follow the reference's lists: axpyf (n_rows 1, n_cols 2,
// x 3, incx 4, matrix 5, lda 6, y 7, incy 8); dotf (matrix 3, lda 4, x 5,
// incx 6, out 7; out is contiguous).
template <typename T>
coral_status_t fused_g(Handle* H, int op, size_t n_rows, size_t n_cols, const void* matrix, size_t lda,
                       const void* x, size_t incx, void* y, size_t incy) {
  const bool axpy = op == 0;
  if (n_rows == 0 || n_cols == 0) return CORAL_OK;   // saxpyf.rs:46-47, sdotf.rs:46-47
  if (axpy) {
    if (!x) return bad_arg(H, 3);
    if (incx == 0) return bad_arg(H, 4);
    if (!matrix) return bad_arg(H, 5);
    if (lda < n_rows) return bad_arg(H, 6);
    if (!y) return bad_arg(H, 7);
    if (incy == 0) return bad_arg(H, 8);
  } else {
    if (!matrix) return bad_arg(H, 3);
    if (lda < n_rows) return bad_arg(H, 4);
    if (!x) return bad_arg(H, 5);
    if (incx == 0) return bad_arg(H, 6);
    if (!y) return bad_arg(H, 7);
  }
  if (((uintptr_t)matrix | (uintptr_t)x | (uintptr_t)y) % sizeof(T)) return bad_arg(H, axpy ? 5 : 3);
  return gemv_g<T>(H, op, n_rows, n_cols, Fld<T>::one(), false, Fld<T>::one(), 0, static_cast<const T*>(matrix),
                   lda, static_cast<const T*>(x), incx, static_cast<T*>(y), axpy ? incy : 1);
}

}  // namespace
}  // namespace coral

using namespace coral;

extern "C" {

coral_status_t coral_daxpyf(coral_handle_t hh, size_t n_rows, size_t n_cols, const double* x, size_t incx,
                            const double* matrix, size_t lda, double* y, size_t incy) {
  CORAL_HANDLE(hh);
  return fused_g<double>(H, 0, n_rows, n_cols, matrix, lda, x, incx, y, incy);
}
coral_status_t coral_caxpyf(coral_handle_t hh, size_t n_rows, size_t n_cols, const float* x, size_t incx,
                            const float* matrix, size_t lda, float* y, size_t incy) {
  CORAL_HANDLE(hh);
  return fused_g<float2>(H, 0, n_rows, n_cols, matrix, lda, x, incx, y, incy);
}
coral_status_t coral_zaxpyf(coral_handle_t hh, size_t n_rows, size_t n_cols, const double* x, size_t incx,
                            const double* matrix, size_t lda, double* y, size_t incy) {
  CORAL_HANDLE(hh);
  return fused_g<double2>(H, 0, n_rows, n_cols, matrix, lda, x, incx, y, incy);
}
coral_status_t coral_ddotf(coral_handle_t hh, size_t n_rows, size_t n_cols, const double* matrix, size_t lda,
                           const double* x, size_t incx, double* out) {
  CORAL_HANDLE(hh);
  return fused_g<double>(H, 1, n_rows, n_cols, matrix, lda, x, incx, out, 1);
}
coral_status_t coral_cdotuf(coral_handle_t hh, size_t n_rows, size_t n_cols, const float* matrix, size_t lda,
                            const float* x, size_t incx, float* out) {
  CORAL_HANDLE(hh);
  return fused_g<float2>(H, 1, n_rows, n_cols, matrix, lda, x, incx, out, 1);
}
coral_status_t coral_cdotcf(coral_handle_t hh, size_t n_rows, size_t n_cols, const float* matrix, size_t lda,
                            const float* x, size_t incx, float* out) {
  CORAL_HANDLE(hh);
  return fused_g<float2>(H, 2, n_rows, n_cols, matrix, lda, x, incx, out, 1);
}
coral_status_t coral_zdotuf(coral_handle_t hh, size_t n_rows, size_t n_cols, const double* matrix, size_t lda,
                            const double* x, size_t incx, double* out) {
  CORAL_HANDLE(hh);
  return fused_g<double2>(H, 1, n_rows, n_cols, matrix, lda, x, incx, out, 1);
}
coral_status_t coral_zdotcf(coral_handle_t hh, size_t n_rows, size_t n_cols, const double* matrix, size_t lda,
                            const double* x, size_t incx, double* out) {
  CORAL_HANDLE(hh);
  return fused_g<double2>(H, 2, n_rows, n_cols, matrix, lda, x, incx, out, 1);
}

coral_status_t coral_dgemv(coral_handle_t hh, int trans, size_t n_rows, size_t n_cols, double alpha,
                           const double* matrix, size_t lda, const double* x, size_t incx,
                           double beta, double* y, size_t incy) {
  CORAL_HANDLE(hh);
  if (trans < CORAL_NO_TRANSPOSE || trans > CORAL_CONJ_TRANSPOSE) return bad_arg(H, 1);
  if (n_rows == 0 || n_cols == 0) return CORAL_OK;         // dgemv_notranspose.rs quick return
  if (alpha == 0.0 && beta == 1.0) return CORAL_OK;
  if (const int bad = gemv_bad(trans, n_rows, matrix, lda, x, incx, y, incy)) return bad_arg(H, bad);
  // ConjugateTranspose == Transpose for real data
  const int op = trans == CORAL_NO_TRANSPOSE ? 0 : 1;
  return gemv_g<double>(H, op, n_rows, n_cols, alpha, alpha == 0.0, beta, beta == 1.0 ? 0 : 1, matrix,
                        lda, x, incx, y, incy);
}

coral_status_t coral_cgemv(coral_handle_t hh, int trans, size_t n_rows, size_t n_cols,
                           const float alpha[2], const float* matrix, size_t lda, const float* x,
                           size_t incx, const float beta[2], float* y, size_t incy) {
  CORAL_HANDLE(hh);
  return complex_gemv<float2, float>(H, trans, n_rows, n_cols, alpha, matrix, lda, x, incx, beta, y, incy);
}

coral_status_t coral_zgemv(coral_handle_t hh, int trans, size_t n_rows, size_t n_cols,
                           const double alpha[2], const double* matrix, size_t lda, const double* x,
                           size_t incx, const double beta[2], double* y, size_t incy) {
  CORAL_HANDLE(hh);
  return complex_gemv<double2, double>(H, trans, n_rows, n_cols, alpha, matrix, lda, x, incx, beta, y, incy);
}

}  // extern "C"
