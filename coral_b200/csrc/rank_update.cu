// Rank-1 / rank-2 updates SGER, SSYR, SSYR2: elementwise column streams,
// bit-exact with the reference's rounding.
//
// Every element of A is touched by exactly one thread, which applies the same
// sequence of roundings as the reference for that element:
//   unit-stride paths go through saxpy (saxpy.rs:63-114), which fuses the
//   multiply-add for the first len - len % 8 elements of the column segment
//   and rounds `y += alpha * x` twice for the rest;
//   strided paths use mul_add (one rounding) for every element.
// The per-column coefficient is alpha * y_j (or alpha * x_j) rounded to fp32,
// and a column whose coefficient is zero is left untouched (sger.rs:93-96,
// ssyr.rs:91-92, ssyr2.rs:84-104); the strided SSYR2 path skips a column only
// when both coefficients are zero (ssyr2.rs:150-153).
#include "common.cuh"

namespace coral {
namespace {

constexpr int kRowsPerBlock = 1024;
constexpr int kRankThreads = 256;

enum RankKind { kGer = 0, kSyr = 1, kSyr2 = 2 };

__device__ __forceinline__ float axpy_elem(float a, float coeff, float xv, bool fused) {
  return fused ? fmaf(xv, coeff, a) : __fadd_rn(a, __fmul_rn(coeff, xv));
}

template <int kKind>
__global__ void __launch_bounds__(kRankThreads)
k_rank(int m, int n, float alpha, const float* __restrict__ x, size_t incx,
       const float* __restrict__ y, size_t incy, float* __restrict__ A, size_t lda, bool lower,
       bool unit) {
  for (int j = blockIdx.y; j < n; j += gridDim.y) {
    int lo = 0, hi = m;
    if (kKind != kGer) {
      lo = lower ? j : 0;
      hi = lower ? n : j + 1;
    }
    const int len = hi - lo;
    const int base = lo + blockIdx.x * kRowsPerBlock;
    if (base >= hi) continue;
    const int nfused = unit ? len - (len & 7) : len;
    float* col = A + (size_t)j * lda;
    if (kKind == kGer || kKind == kSyr) {
      const float* cv = kKind == kGer ? y + (size_t)j * incy : x + (size_t)j * incx;
      const float coeff = __fmul_rn(alpha, *cv);
      if (coeff == 0.0f) continue;
#pragma unroll
      for (int e = 0; e < kRowsPerBlock / kRankThreads; ++e) {
        int i = base + threadIdx.x + e * kRankThreads;
        if (i >= hi) break;
        col[i] = axpy_elem(col[i], coeff, x[(size_t)i * incx], (i - lo) < nfused);
      }
    } else {
      const float ay = __fmul_rn(alpha, y[(size_t)j * incy]);
      const float ax = __fmul_rn(alpha, x[(size_t)j * incx]);
      if (unit) {
#pragma unroll
        for (int e = 0; e < kRowsPerBlock / kRankThreads; ++e) {
          int i = base + threadIdx.x + e * kRankThreads;
          if (i >= hi) break;
          const bool fused = (i - lo) < nfused;
          float a = col[i];
          if (ay != 0.0f) a = axpy_elem(a, ay, x[i], fused);
          if (ax != 0.0f) a = axpy_elem(a, ax, y[i], fused);
          col[i] = a;
        }
      } else {
        if (ay == 0.0f && ax == 0.0f) continue;
#pragma unroll
        for (int e = 0; e < kRowsPerBlock / kRankThreads; ++e) {
          int i = base + threadIdx.x + e * kRankThreads;
          if (i >= hi) break;
          float a = col[i];
          a = fmaf(x[(size_t)i * incx], ay, a);
          a = fmaf(y[(size_t)i * incy], ax, a);
          col[i] = a;
        }
      }
    }
  }
}

template <int kKind>
coral_status_t launch_rank(Handle* h, size_t m, size_t n, float alpha, const float* x, size_t incx,
                           const float* y, size_t incy, float* A, size_t lda, bool lower, bool unit) {
  if (m > INT32_MAX || n > INT32_MAX) return CORAL_ERR_NOT_SUPPORTED;
  const size_t rows = kKind == kGer ? m : n;
  dim3 grid((unsigned)((rows + kRowsPerBlock - 1) / kRowsPerBlock),
            (unsigned)(n < 65535 ? n : 65535));
  k_rank<kKind><<<grid, kRankThreads, 0, h->stream>>>((int)m, (int)n, alpha, x, incx, y, incy, A,
                                                      lda, lower, unit);
  return launch_status(h);
}

}  // namespace
}  // namespace coral

using namespace coral;

extern "C" {

coral_status_t coral_sger(coral_handle_t hh, size_t n_rows, size_t n_cols, float alpha,
                          const float* x, size_t incx, const float* y, size_t incy, float* matrix,
                          size_t lda) {
  CORAL_HANDLE(hh);
  if (n_rows == 0 || n_cols == 0 || alpha == 0.0f) return CORAL_OK;  // sger.rs:80
  if (!x) return bad_arg(H, 4);
  if (incx == 0) return bad_arg(H, 5);
  if (!y) return bad_arg(H, 6);
  if (incy == 0) return bad_arg(H, 7);
  if (!matrix) return bad_arg(H, 8);
  if (lda < n_rows) return bad_arg(H, 9);
  const bool unit = incx == 1 && incy == 1;  // sger.rs:91 fast path
  return launch_rank<kGer>(H, n_rows, n_cols, alpha, x, incx, y, incy, matrix, lda, false, unit);
}

coral_status_t coral_ssyr(coral_handle_t hh, int uplo, size_t n, float alpha, const float* x,
                          size_t incx, float* matrix, size_t lda) {
  CORAL_HANDLE(hh);
  if (uplo != CORAL_UPPER && uplo != CORAL_LOWER) return bad_arg(H, 1);
  if (n == 0 || alpha == 0.0f) return CORAL_OK;  // ssyr.rs:73-75
  if (!x) return bad_arg(H, 4);
  if (incx == 0) return bad_arg(H, 5);
  if (!matrix) return bad_arg(H, 6);
  if (lda < n) return bad_arg(H, 7);
  return launch_rank<kSyr>(H, n, n, alpha, x, incx, x, incx, matrix, lda, uplo == CORAL_LOWER,
                           incx == 1);
}

coral_status_t coral_ssyr2(coral_handle_t hh, int uplo, size_t n, float alpha, const float* x,
                           size_t incx, const float* y, size_t incy, float* matrix, size_t lda) {
  CORAL_HANDLE(hh);
  if (uplo != CORAL_UPPER && uplo != CORAL_LOWER) return bad_arg(H, 1);
  if (n == 0 || alpha == 0.0f) return CORAL_OK;  // ssyr2.rs:70-72
  if (!x) return bad_arg(H, 4);
  if (incx == 0) return bad_arg(H, 5);
  if (!y) return bad_arg(H, 6);
  if (incy == 0) return bad_arg(H, 7);
  if (!matrix) return bad_arg(H, 8);
  if (lda < n) return bad_arg(H, 9);
  return launch_rank<kSyr2>(H, n, n, alpha, x, incx, y, incy, matrix, lda, uplo == CORAL_LOWER,
                            incx == 1 && incy == 1);
}

}  // extern "C"
