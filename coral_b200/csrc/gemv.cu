// SGEMV: y <- alpha * op(A) x + beta * y, column-major A (sgemv.rs:63-80).
//
// Both directions stream A exactly once from HBM with 128-bit loads and
// finish in one launch: blocks write partial sums to scratch and the last
// block of each output tile (arrival counter) adds them in a fixed order, so
// results are deterministic.
//
//   N (sgemv_notranspose.rs:63-177): a block owns a 128-row strip of y and a
//     chunk of columns; each warp reads whole 512-byte column segments
//     (lane = 4 rows) and keeps 4 row accumulators per lane.
//   T (sgemv_transpose.rs:64-182): a block owns a chunk of rows (alpha*x for
//     those rows staged in shared memory) and a group of columns; each warp
//     computes full dot products of column segments and reduces with shuffles.
//
// Reference semantics kept: quick return for an empty matrix or alpha == 0 &&
// beta == 1; beta != 1 scales y by multiplication (sscal, so beta == 0 keeps
// NaN * 0 = NaN as sscal.rs:41-51 does); x is pre-scaled by alpha in fp32
// (pack_and_scale_f32) before the products.
#include "common.cuh"

namespace coral {

coral_status_t enqueue_sscal(Handle* h, size_t n, float alpha, float* x, size_t incx);

namespace {

constexpr int kGemvThreads = 256;
constexpr int kGemvWarps = kGemvThreads / 32;
constexpr int kStripRows = 128;   // rows of y per N-block (32 lanes x 4)
constexpr int kTRows = 4096;      // rows per T-block chunk (16 KB of alpha*x)

__device__ bool arrive_last(unsigned* counter, unsigned total) {
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

__device__ __forceinline__ float scale_y(float y, float beta) {
  return beta != 1.0f ? __fmul_rn(beta, y) : y;
}

template <bool kVec>
__global__ void __launch_bounds__(kGemvThreads)
k_gemv_n(int m, int n, const float* __restrict__ A, size_t lda, const float* __restrict__ x,
         size_t incx, float alpha, float beta, float* __restrict__ y, size_t incy,
         int cols_per_chunk, float* partials, unsigned* counters) {
  __shared__ float red[kGemvWarps][kStripRows];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int row0 = blockIdx.x * kStripRows;
  const int c0 = blockIdx.y * cols_per_chunk;
  const int c1 = min(n, c0 + cols_per_chunk);
  float acc[4] = {0.f, 0.f, 0.f, 0.f};
  int rows[4];
#pragma unroll
  for (int e = 0; e < 4; ++e) rows[e] = kVec ? row0 + 4 * lane + e : row0 + lane + 32 * e;
  const bool full4 = kVec && (row0 + 4 * lane + 3 < m);

  auto load = [&](int j, float v[4]) {
    const float* col = A + (size_t)j * lda;
    if (full4) {
      float4 a = __ldcs(reinterpret_cast<const float4*>(col + rows[0]));
      v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w;
    } else {
#pragma unroll
      for (int e = 0; e < 4; ++e) v[e] = rows[e] < m ? __ldcs(col + rows[e]) : 0.f;
    }
  };

  int j = c0 + warp;
  for (; j + 3 * kGemvWarps < c1; j += 4 * kGemvWarps) {
    float v[4][4], xs[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      load(j + u * kGemvWarps, v[u]);
      xs[u] = __fmul_rn(alpha, __ldg(x + (size_t)(j + u * kGemvWarps) * incx));
    }
#pragma unroll
    for (int u = 0; u < 4; ++u)
#pragma unroll
      for (int e = 0; e < 4; ++e) acc[e] = fmaf(v[u][e], xs[u], acc[e]);
  }
  for (; j < c1; j += kGemvWarps) {
    float v[4];
    load(j, v);
    float xs = __fmul_rn(alpha, __ldg(x + (size_t)j * incx));
#pragma unroll
    for (int e = 0; e < 4; ++e) acc[e] = fmaf(v[e], xs, acc[e]);
  }
#pragma unroll
  for (int e = 0; e < 4; ++e) red[warp][rows[e] - row0] = acc[e];
  __syncthreads();
  // Fixed-order sum over the warps; thread t owns strip row t (t < 128).
  float s = 0.f;
  const int t = threadIdx.x;
  if (t < kStripRows) {
#pragma unroll
    for (int w = 0; w < kGemvWarps; ++w) s += red[w][t];
  }
  const int r = row0 + t;
  if (gridDim.y == 1) {
    if (t < kStripRows && r < m) {
      float* yp = y + (size_t)r * incy;
      *yp = scale_y(*yp, beta) + s;
    }
    return;
  }
  if (t < kStripRows && r < m) partials[(size_t)blockIdx.y * m + r] = s;
  if (!arrive_last(counters + blockIdx.x, gridDim.y)) return;
  if (t < kStripRows && r < m) {
    float tot = 0.f;
    for (unsigned c = 0; c < gridDim.y; ++c) tot += __ldcg(partials + (size_t)c * m + r);
    float* yp = y + (size_t)r * incy;
    *yp = scale_y(*yp, beta) + tot;
  }
}

template <bool kVec>
__global__ void __launch_bounds__(kGemvThreads)
k_gemv_t(int m, int n, const float* __restrict__ A, size_t lda, const float* __restrict__ x,
         size_t incx, float alpha, float beta, float* __restrict__ y, size_t incy,
         int rows_per_chunk, int cols_per_group, float* partials, unsigned* counters) {
  extern __shared__ float xs[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int r0 = blockIdx.y * rows_per_chunk;
  const int r1 = min(m, r0 + rows_per_chunk);
  const int nr = r1 - r0;
  // alpha*x for this row chunk: staged in shared memory for strided x;
  // unit-stride x is scaled on the fly from the read-only cache (xsc).
  const bool direct = kVec && incx == 1 && ((reinterpret_cast<uintptr_t>(x + r0) & 15) == 0);
  if (!direct) {
    for (int i = threadIdx.x; i < nr; i += blockDim.x)
      xs[i] = __fmul_rn(alpha, __ldg(x + (size_t)(r0 + i) * incx));
    __syncthreads();
  }
  const int g0 = blockIdx.x * cols_per_group;
  const int g1 = min(n, g0 + cols_per_group);
  for (int j = g0 + warp; j < g1; j += kGemvWarps) {
    const float* col = A + (size_t)j * lda + r0;
    float acc0 = 0.f, acc1 = 0.f;
    if (kVec) {
      const int n4 = nr >> 2;
      const float4* c4 = reinterpret_cast<const float4*>(col);
      const float4* x4 = reinterpret_cast<const float4*>(direct ? x + r0 : xs);
      auto xsc = [&](int q) {
        float4 v = direct ? __ldg(x4 + q) : x4[q];
        if (direct) {
          v.x = __fmul_rn(alpha, v.x); v.y = __fmul_rn(alpha, v.y);
          v.z = __fmul_rn(alpha, v.z); v.w = __fmul_rn(alpha, v.w);
        }
        return v;
      };
      int i = lane;
      for (; i + 96 < n4; i += 128) {
        float4 a0 = __ldcs(c4 + i), a1 = __ldcs(c4 + i + 32);
        float4 a2 = __ldcs(c4 + i + 64), a3 = __ldcs(c4 + i + 96);
        float4 b0 = xsc(i), b1 = xsc(i + 32), b2 = xsc(i + 64), b3 = xsc(i + 96);
        acc0 = fmaf(a0.x, b0.x, acc0); acc0 = fmaf(a0.y, b0.y, acc0);
        acc0 = fmaf(a0.z, b0.z, acc0); acc0 = fmaf(a0.w, b0.w, acc0);
        acc1 = fmaf(a1.x, b1.x, acc1); acc1 = fmaf(a1.y, b1.y, acc1);
        acc1 = fmaf(a1.z, b1.z, acc1); acc1 = fmaf(a1.w, b1.w, acc1);
        acc0 = fmaf(a2.x, b2.x, acc0); acc0 = fmaf(a2.y, b2.y, acc0);
        acc0 = fmaf(a2.z, b2.z, acc0); acc0 = fmaf(a2.w, b2.w, acc0);
        acc1 = fmaf(a3.x, b3.x, acc1); acc1 = fmaf(a3.y, b3.y, acc1);
        acc1 = fmaf(a3.z, b3.z, acc1); acc1 = fmaf(a3.w, b3.w, acc1);
      }
      for (; i < n4; i += 32) {
        float4 a = __ldcs(c4 + i), b = xsc(i);
        acc0 = fmaf(a.x, b.x, acc0); acc0 = fmaf(a.y, b.y, acc0);
        acc0 = fmaf(a.z, b.z, acc0); acc0 = fmaf(a.w, b.w, acc0);
      }
      for (int t = (n4 << 2) + lane; t < nr; t += 32)
        acc1 = fmaf(__ldcs(col + t), direct ? __fmul_rn(alpha, __ldg(x + r0 + t)) : xs[t], acc1);
    } else {
      int i = lane;
      for (; i + 32 < nr; i += 64) {
        acc0 = fmaf(__ldcs(col + i), xs[i], acc0);
        acc1 = fmaf(__ldcs(col + i + 32), xs[i + 32], acc1);
      }
      if (i < nr) acc0 = fmaf(__ldcs(col + i), xs[i], acc0);
    }
    float s = acc0 + acc1;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) {
      if (gridDim.y == 1) {
        float* yp = y + (size_t)j * incy;
        *yp = scale_y(*yp, beta) + s;
      } else {
        partials[(size_t)blockIdx.y * n + j] = s;
      }
    }
  }
  if (gridDim.y == 1) return;
  if (!arrive_last(counters + blockIdx.x, gridDim.y)) return;
  for (int j = g0 + threadIdx.x; j < g1; j += blockDim.x) {
    float tot = 0.f;
    for (unsigned c = 0; c < gridDim.y; ++c) tot += __ldcg(partials + (size_t)c * n + j);
    float* yp = y + (size_t)j * incy;
    *yp = scale_y(*yp, beta) + tot;
  }
}

}  // namespace

// Enqueues y <- beta*y + A*(alpha x) (trans == false) or A^T*(alpha x).
// Sizes are assumed validated; used by SGEMV and by the level-2 routines
// built on it (TRMV panels).
coral_status_t enqueue_gemv(Handle* h, bool trans, size_t m, size_t n, float alpha,
                            const float* A, size_t lda, const float* x, size_t incx, float beta,
                            float* y, size_t incy) {
  if (m > INT32_MAX || n > INT32_MAX) return CORAL_ERR_NOT_SUPPORTED;
  const bool vec = (lda % 4 == 0) && aligned16(A);
  const int target = h->sm_count * 8;
  if (!trans) {
    const int strips = (int)((m + kStripRows - 1) / kStripRows);
    int chunks = (target + strips - 1) / strips;
    int min_cols = 64;
    int max_chunks = (int)((n + min_cols - 1) / min_cols);
    if (chunks > max_chunks) chunks = max_chunks;
    if (chunks < 1) chunks = 1;
    int cpc = (int)((n + chunks - 1) / chunks);
    chunks = (int)((n + cpc - 1) / cpc);
    if (strips > (int)kTrsvFlagBase) return CORAL_ERR_NOT_SUPPORTED;
    float* part = nullptr;
    if (chunks > 1) {
      part = static_cast<float*>(scratch(h, (size_t)chunks * m * sizeof(float)));
      if (!part) return CORAL_ERR_ALLOC;
    }
    dim3 grid(strips, chunks);
    if (vec)
      k_gemv_n<true><<<grid, kGemvThreads, 0, h->stream>>>((int)m, (int)n, A, lda, x, incx, alpha,
                                                           beta, y, incy, cpc, part, h->counters);
    else
      k_gemv_n<false><<<grid, kGemvThreads, 0, h->stream>>>((int)m, (int)n, A, lda, x, incx, alpha,
                                                            beta, y, incy, cpc, part, h->counters);
    return launch_status(h);
  }
  const int rchunks = (int)((m + kTRows - 1) / kTRows);
  const int rpc = (int)(((m + rchunks - 1) / rchunks + 3) / 4 * 4);
  int groups = (target + rchunks - 1) / rchunks;
  int max_groups = (int)((n + kGemvWarps - 1) / kGemvWarps);
  if (groups > max_groups) groups = max_groups;
  if (groups < 1) groups = 1;
  int cpg = (int)((n + groups - 1) / groups);
  groups = (int)((n + cpg - 1) / cpg);
  if (groups > (int)kTrsvFlagBase) return CORAL_ERR_NOT_SUPPORTED;
  float* part = nullptr;
  if (rchunks > 1) {
    part = static_cast<float*>(scratch(h, (size_t)rchunks * n * sizeof(float)));
    if (!part) return CORAL_ERR_ALLOC;
  }
  dim3 grid(groups, rchunks);
  size_t smem = (size_t)rpc * sizeof(float);
  if (vec)
    k_gemv_t<true><<<grid, kGemvThreads, smem, h->stream>>>((int)m, (int)n, A, lda, x, incx, alpha,
                                                            beta, y, incy, rpc, cpg, part, h->counters);
  else
    k_gemv_t<false><<<grid, kGemvThreads, smem, h->stream>>>((int)m, (int)n, A, lda, x, incx, alpha,
                                                             beta, y, incy, rpc, cpg, part, h->counters);
  return launch_status(h);
}

}  // namespace coral

using namespace coral;

// Fused level-1.5 updates in fp32 (level1_special/saxpyf.rs:36-513,
// sdotf.rs:37-600): y += A x and out += A^T x on the SGEMV kernels with
// alpha = beta = 1.  Argument positions follow the reference's lists.
extern "C" coral_status_t coral_saxpyf(coral_handle_t hh, size_t n_rows, size_t n_cols, const float* x,
                                       size_t incx, const float* matrix, size_t lda, float* y, size_t incy) {
  CORAL_HANDLE(hh);
  if (n_rows == 0 || n_cols == 0) return CORAL_OK;   // saxpyf.rs:46-47
  if (!x) return bad_arg(H, 3);
  if (incx == 0) return bad_arg(H, 4);
  if (!matrix) return bad_arg(H, 5);
  if (lda < n_rows) return bad_arg(H, 6);
  if (!y) return bad_arg(H, 7);
  if (incy == 0) return bad_arg(H, 8);
  return enqueue_gemv(H, false, n_rows, n_cols, 1.0f, matrix, lda, x, incx, 1.0f, y, incy);
}

extern "C" coral_status_t coral_sdotf(coral_handle_t hh, size_t n_rows, size_t n_cols, const float* matrix,
                                      size_t lda, const float* x, size_t incx, float* out) {
  CORAL_HANDLE(hh);
  if (n_rows == 0 || n_cols == 0) return CORAL_OK;   // sdotf.rs:46-47
  if (!matrix) return bad_arg(H, 3);
  if (lda < n_rows) return bad_arg(H, 4);
  if (!x) return bad_arg(H, 5);
  if (incx == 0) return bad_arg(H, 6);
  if (!out) return bad_arg(H, 7);
  return enqueue_gemv(H, true, n_rows, n_cols, 1.0f, matrix, lda, x, incx, 1.0f, out, 1);
}

extern "C" coral_status_t coral_sgemv(coral_handle_t hh, int trans, size_t n_rows, size_t n_cols,
                                      float alpha, const float* matrix, size_t lda,
                                      const float* x, size_t incx, float beta, float* y,
                                      size_t incy) {
  CORAL_HANDLE(hh);
  if (trans < CORAL_NO_TRANSPOSE || trans > CORAL_CONJ_TRANSPOSE) return bad_arg(H, 1);
  if (n_cols == 0 || n_rows == 0) return CORAL_OK;           // sgemv_notranspose.rs:76
  if (alpha == 0.0f && beta == 1.0f) return CORAL_OK;        // sgemv_notranspose.rs:77
  if (!matrix) return bad_arg(H, 5);
  if (lda < n_rows) return bad_arg(H, 6);
  if (!x) return bad_arg(H, 7);
  if (incx == 0) return bad_arg(H, 8);
  if (!y) return bad_arg(H, 10);
  if (incy == 0) return bad_arg(H, 11);
  const bool t = trans != CORAL_NO_TRANSPOSE;  // ConjugateTranspose == Transpose (sgemv.rs:78)
  const size_t ylen = t ? n_cols : n_rows;
  if (alpha == 0.0f) return enqueue_sscal(H, ylen, beta, y, incy);  // :89-90
  return enqueue_gemv(H, t, n_rows, n_cols, alpha, matrix, lda, x, incx, beta, y, incy);
}
