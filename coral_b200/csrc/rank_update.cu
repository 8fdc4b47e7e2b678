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

// Vector form of the unit-stride path, for A, x (and y for SSYR2) on 16-byte
// boundaries with lda % 4 == 0. A thread owns 4 consecutive rows: it loads
// their x (and y) once and updates them in kVCols columns. All of those
// columns' A vectors are loaded, together with the columns' coefficients,
// before the first is written back, so 16 * kVCols bytes of A are in flight
// per thread instead of 4. A column whose coefficient is zero is loaded but
// not written, so it is left untouched as before. Each element gets exactly
// the roundings of k_rank's unit path. A vector that straddles the edge of a
// column's triangle, or the last row, is read and written element by
// element, in-range elements only.
constexpr int kVCols = 8;

template <int kKind>
__global__ void __launch_bounds__(kRankThreads, 3)
k_rank_vec(int m, int n, float alpha, const float* __restrict__ x, const float* __restrict__ y,
           float* __restrict__ A, size_t lda, bool lower) {
  const int rows = kKind == kGer ? m : n;
  // rows [lo, hi) of column j that the update touches
  auto range = [&](int j, int& lo, int& hi) {
    lo = kKind == kGer ? 0 : (lower ? j : 0);
    hi = kKind == kGer ? m : (lower ? n : j + 1);
  };
  // rows i0 .. i0+3 of columns jg .. jg+kVCols-1
  auto block = [&](int i0, int jg) {
    const bool full_rows = i0 + 4 <= rows;
    float xv[4], yv[4];
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      xv[e] = full_rows || i0 + e < rows ? x[i0 + e] : 0.0f;
      yv[e] = kKind == kSyr2 && (full_rows || i0 + e < rows) ? y[i0 + e] : 0.0f;
    }
    float4 a[kVCols];
    float c1[kVCols], c2[kVCols];
    unsigned on_mask = 0, whole_mask = 0;
#pragma unroll
    for (int c = 0; c < kVCols; ++c) {
      const int j = jg + c;
      int l, h;
      range(j, l, h);
      const bool on = j < n && i0 < h && i0 + 4 > l;
      const bool whole = on && i0 >= l && i0 + 4 <= h;
      on_mask |= on ? 1u << c : 0u;
      whole_mask |= whole ? 1u << c : 0u;
      c1[c] = c2[c] = 0.0f;
      if (on) {
        if (kKind == kGer) c1[c] = __fmul_rn(alpha, y[j]);
        if (kKind == kSyr) c1[c] = __fmul_rn(alpha, x[j]);
        if (kKind == kSyr2) {
          c1[c] = __fmul_rn(alpha, y[j]);  // coefficient of x
          c2[c] = __fmul_rn(alpha, x[j]);  // coefficient of y
        }
      }
      const float* col = A + (size_t)(on ? j : 0) * lda + i0;
      if (whole) {
        a[c] = *reinterpret_cast<const float4*>(col);
      } else {
        a[c].x = on && i0 >= l && i0 < h ? col[0] : 0.0f;
        a[c].y = on && i0 + 1 >= l && i0 + 1 < h ? col[1] : 0.0f;
        a[c].z = on && i0 + 2 >= l && i0 + 2 < h ? col[2] : 0.0f;
        a[c].w = on && i0 + 3 >= l && i0 + 3 < h ? col[3] : 0.0f;
      }
    }
#pragma unroll
    for (int c = 0; c < kVCols; ++c) {
      if (!(on_mask & (1u << c))) continue;
      if (c1[c] == 0.0f && c2[c] == 0.0f) continue;  // column left untouched
      const int j = jg + c;
      int l, h;
      range(j, l, h);
      const int len = h - l, nfused = len - (len & 7);
      float* av = &a[c].x;
      const float k1 = c1[c], k2 = c2[c];
      if (i0 + 3 - l < nfused) {
        // all four elements in the fused part (the common case)
#pragma unroll
        for (int e = 0; e < 4; ++e) {
          float v = av[e];
          if (k1 != 0.0f) v = fmaf(xv[e], k1, v);
          if (kKind == kSyr2 && k2 != 0.0f) v = fmaf(yv[e], k2, v);
          av[e] = v;
        }
      } else {
#pragma unroll
        for (int e = 0; e < 4; ++e) {
          const bool fused = (i0 + e - l) < nfused;
          float v = av[e];
          if (k1 != 0.0f) v = axpy_elem(v, k1, xv[e], fused);
          if (kKind == kSyr2 && k2 != 0.0f) v = axpy_elem(v, k2, yv[e], fused);
          av[e] = v;
        }
      }
      float* col = A + (size_t)j * lda + i0;
      if (whole_mask & (1u << c)) {
        *reinterpret_cast<float4*>(col) = a[c];
      } else {
#pragma unroll
        for (int e = 0; e < 4; ++e)
          if (i0 + e >= l && i0 + e < h) col[e] = av[e];
      }
    }
  };
  if (kKind == kGer) {
    // grid: x = 1024-row chunks, y = column groups
    const int i0 = (blockIdx.x * kRankThreads + threadIdx.x) * 4;
    if (i0 >= rows) return;
    for (int jg = blockIdx.y * kVCols; jg < n; jg += gridDim.y * kVCols) block(i0, jg);
  } else {
    // grid: x = column groups, each walking only the row chunks its
    // triangle columns touch; upper takes the longest groups first
    const int ngroups = (n + kVCols - 1) / kVCols;
    for (int gi = blockIdx.x; gi < ngroups; gi += gridDim.x) {
      const int jg = (lower ? gi : ngroups - 1 - gi) * kVCols;
      const int jl = min(n, jg + kVCols) - 1;
      const int r_lo = lower ? jg : 0, r_hi = lower ? n : jl + 1;
      for (int rb = r_lo / (4 * kRankThreads); rb * 4 * kRankThreads < r_hi; ++rb) {
        const int i0 = (rb * kRankThreads + threadIdx.x) * 4;
        if (i0 < r_hi && i0 + 4 > r_lo) block(i0, jg);
      }
    }
  }
}

template <int kKind>
coral_status_t launch_rank(Handle* h, size_t m, size_t n, float alpha, const float* x, size_t incx,
                           const float* y, size_t incy, float* A, size_t lda, bool lower, bool unit) {
  if (m > INT32_MAX || n > INT32_MAX) return CORAL_ERR_NOT_SUPPORTED;
  const size_t rows = kKind == kGer ? m : n;
  if (unit && aligned16(A) && lda % 4 == 0 && aligned16(x) && (kKind != kSyr2 || aligned16(y))) {
    const size_t groups = (n + kVCols - 1) / kVCols;
    const dim3 vgrid = kKind == kGer
        ? dim3((unsigned)((rows + 4 * kRankThreads - 1) / (4 * kRankThreads)),
               (unsigned)(groups < 65535 ? groups : 65535))
        : dim3((unsigned)(groups < (1u << 30) ? groups : (1u << 30)));
    k_rank_vec<kKind><<<vgrid, kRankThreads, 0, h->stream>>>((int)m, (int)n, alpha, x, y, A, lda, lower);
    return launch_status(h);
  }
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
