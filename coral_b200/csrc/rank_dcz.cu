// Double and complex rank-1 / rank-2 updates: DGER, CGERU/CGERC, ZGERU/ZGERC,
// DSYR, DSYR2, CHER/ZHER, CHER2/ZHER2 (level2/*ger*.rs, dsyr.rs, dsyr2.rs,
// cher.rs, cher2.rs, zher.rs, zher2.rs).  Complex data is interleaved
// (re, im), leading dimensions and increments in complex units.
//
// One pass over the touched part of A: every element is read and written by
// exactly one thread.  Per column j the coefficients are formed as the
// reference forms them -- ger: alpha*y_j; gerc: alpha*conj(y_j); syr:
// alpha*x_j; her: alpha*conj(x_j) with real alpha; syr2: alpha*y_j and
// alpha*x_j; her2: alpha*conj(y_j) and conj(alpha)*conj(x_j) -- and a term
// whose coefficient is zero is skipped, so the column (or that term) is left
// untouched as in the reference (dger.rs fast path, cher.rs, cher2.rs).  The
// Hermitian updates then store a real diagonal: her when column j was
// updated (cher.rs), her2 for every column (cher2.rs).  syr / her touch the
// `uplo` triangle only.
#include "common.cuh"
#include "field.cuh"

namespace coral {
namespace {

constexpr int kRRows = 1024;      // rows per block
constexpr int kRThreads = 256;

enum RankKindG { kGerU = 0, kGerC = 1, kSyrG = 2, kHerG = 3, kSyr2G = 4, kHer2G = 5 };

__device__ __forceinline__ bool nz(double a) { return a != 0.0; }
__device__ __forceinline__ bool nz(float2 a) { return a.x != 0.f || a.y != 0.f; }
__device__ __forceinline__ bool nz(double2 a) { return a.x != 0.0 || a.y != 0.0; }

// alpha * y_j, conjugating y_j when kConj
template <typename T, bool kConj>
__device__ __forceinline__ T coeff(T alpha, T v) {
  return Fld<T>::mul(alpha, kConj ? Fld<T>::conj(v) : v);
}

template <typename T, int kKind>
__global__ void __launch_bounds__(kRThreads)
k_rank_g(int m, int n, T alpha, const T* __restrict__ x, size_t incx, const T* __restrict__ y,
         size_t incy, T* __restrict__ A, size_t lda, bool lower) {
  using F = Fld<T>;
  constexpr bool kTri = kKind >= kSyrG;
  constexpr bool kHerm = kKind == kHerG || kKind == kHer2G;
  for (int j = blockIdx.y; j < n; j += gridDim.y) {
    int lo = 0, hi = m;
    if (kTri) {
      lo = lower ? j : 0;
      hi = lower ? n : j + 1;
    }
    const int base = lo + blockIdx.x * kRRows;
    if (base >= hi) continue;
    T c1 = F::zero(), c2 = F::zero();   // coefficient of x (and of y for rank 2)
    if (kKind == kGerU) c1 = coeff<T, false>(alpha, y[(size_t)j * incy]);
    if (kKind == kGerC) c1 = coeff<T, true>(alpha, y[(size_t)j * incy]);
    if (kKind == kSyrG || kKind == kHerG) c1 = coeff<T, kHerm>(alpha, x[(size_t)j * incx]);
    if (kKind == kSyr2G || kKind == kHer2G) {
      c1 = coeff<T, kHerm>(alpha, y[(size_t)j * incy]);
      c2 = coeff<T, kHerm>(kHerm ? F::conj(alpha) : alpha, x[(size_t)j * incx]);
    }
    const bool u1 = nz(c1), u2 = nz(c2);
    if (!u1 && !u2 && kKind != kHer2G) continue;
    T* col = A + (size_t)j * lda;
#pragma unroll
    for (int e = 0; e < kRRows / kRThreads; ++e) {
      const int i = base + threadIdx.x + e * kRThreads;
      if (i >= hi) break;
      T a = col[i];
      if (u1) F::mac(a, x[(size_t)i * incx], c1);
      if (u2) F::mac(a, y[(size_t)i * incy], c2);
      if (kHerm && i == j) a = F::re(a);   // real diagonal
      col[i] = a;
    }
  }
}

template <typename T, int kKind>
coral_status_t launch_rank_g(Handle* h, size_t m, size_t n, T alpha, const T* x, size_t incx, const T* y,
                             size_t incy, T* A, size_t lda, bool lower) {
  if (m > INT32_MAX || n > INT32_MAX) return CORAL_ERR_NOT_SUPPORTED;
  const size_t rows = kKind >= kSyrG ? n : m;
  const dim3 grid((unsigned)((rows + kRRows - 1) / kRRows), (unsigned)(n < 65535 ? n : 65535));
  k_rank_g<T, kKind><<<grid, kRThreads, 0, h->stream>>>((int)m, (int)n, alpha, x, incx, y, incy, A, lda,
                                                        lower);
  return launch_status(h);
}

// General update (ger*): positions of the checks as in sger.
template <typename T, int kKind>
coral_status_t ger_g(Handle* H, size_t m, size_t n, T alpha, bool alpha_zero, const void* x, size_t incx,
                     const void* y, size_t incy, void* A, size_t lda, size_t align) {
  if (m == 0 || n == 0 || alpha_zero) return CORAL_OK;   // dger.rs / cgeru.rs quick return
  if (!x) return bad_arg(H, 4);
  if (incx == 0) return bad_arg(H, 5);
  if (!y) return bad_arg(H, 6);
  if (incy == 0) return bad_arg(H, 7);
  if (!A) return bad_arg(H, 8);
  if (lda < m) return bad_arg(H, 9);
  if (((uintptr_t)x | (uintptr_t)y | (uintptr_t)A) & (align - 1)) return bad_arg(H, 4);
  return launch_rank_g<T, kKind>(H, m, n, alpha, static_cast<const T*>(x), incx, static_cast<const T*>(y),
                                 incy, static_cast<T*>(A), lda, false);
}

// Triangle updates (syr*, her*): positions as in ssyr / ssyr2.
template <typename T, int kKind>
coral_status_t tri_g(Handle* H, int uplo, size_t n, T alpha, bool alpha_zero, const void* x, size_t incx,
                     const void* y, size_t incy, void* A, size_t lda, size_t align) {
  constexpr bool kTwo = kKind == kSyr2G || kKind == kHer2G;
  if (uplo != CORAL_UPPER && uplo != CORAL_LOWER) return bad_arg(H, 1);
  if (n == 0 || alpha_zero) return CORAL_OK;              // dsyr.rs / cher.rs quick return
  if (!x) return bad_arg(H, 4);
  if (incx == 0) return bad_arg(H, 5);
  if (kTwo) {
    if (!y) return bad_arg(H, 6);
    if (incy == 0) return bad_arg(H, 7);
  }
  if (!A) return bad_arg(H, kTwo ? 8 : 6);
  if (lda < n) return bad_arg(H, kTwo ? 9 : 7);
  if (((uintptr_t)x | (uintptr_t)(kTwo ? y : x) | (uintptr_t)A) & (align - 1)) return bad_arg(H, 4);
  return launch_rank_g<T, kKind>(H, n, n, alpha, static_cast<const T*>(x), incx,
                                 static_cast<const T*>(kTwo ? y : x), kTwo ? incy : incx, static_cast<T*>(A),
                                 lda, uplo == CORAL_LOWER);
}

float2 c2f(const float a[2]) { return make_float2(a[0], a[1]); }
double2 c2d(const double a[2]) { return make_double2(a[0], a[1]); }

}  // namespace
}  // namespace coral

using namespace coral;

extern "C" {

coral_status_t coral_dger(coral_handle_t hh, size_t n_rows, size_t n_cols, double alpha, const double* x,
                          size_t incx, const double* y, size_t incy, double* matrix, size_t lda) {
  CORAL_HANDLE(hh);
  return ger_g<double, kGerU>(H, n_rows, n_cols, alpha, alpha == 0.0, x, incx, y, incy, matrix, lda, 8);
}

#define CORAL_CGER(NAME, T, R, KIND, AL)                                                           \
  coral_status_t NAME(coral_handle_t hh, size_t n_rows, size_t n_cols, const R alpha[2], const R* x, \
                      size_t incx, const R* y, size_t incy, R* matrix, size_t lda) {               \
    CORAL_HANDLE(hh);                                                                              \
    if (!alpha) return bad_arg(H, 3);                                                              \
    return ger_g<T, KIND>(H, n_rows, n_cols, AL(alpha), alpha[0] == 0 && alpha[1] == 0, x, incx, y,  \
                          incy, matrix, lda, sizeof(T));                                           \
  }
CORAL_CGER(coral_cgeru, float2, float, kGerU, c2f)
CORAL_CGER(coral_cgerc, float2, float, kGerC, c2f)
CORAL_CGER(coral_zgeru, double2, double, kGerU, c2d)
CORAL_CGER(coral_zgerc, double2, double, kGerC, c2d)
#undef CORAL_CGER

coral_status_t coral_dsyr(coral_handle_t hh, int uplo, size_t n, double alpha, const double* x, size_t incx,
                          double* matrix, size_t lda) {
  CORAL_HANDLE(hh);
  return tri_g<double, kSyrG>(H, uplo, n, alpha, alpha == 0.0, x, incx, nullptr, 0, matrix, lda, 8);
}

coral_status_t coral_dsyr2(coral_handle_t hh, int uplo, size_t n, double alpha, const double* x, size_t incx,
                           const double* y, size_t incy, double* matrix, size_t lda) {
  CORAL_HANDLE(hh);
  return tri_g<double, kSyr2G>(H, uplo, n, alpha, alpha == 0.0, x, incx, y, incy, matrix, lda, 8);
}

coral_status_t coral_cher(coral_handle_t hh, int uplo, size_t n, float alpha, const float* x, size_t incx,
                          float* matrix, size_t lda) {
  CORAL_HANDLE(hh);
  return tri_g<float2, kHerG>(H, uplo, n, make_float2(alpha, 0.f), alpha == 0.f, x, incx, nullptr, 0, matrix,
                              lda, 8);
}

coral_status_t coral_zher(coral_handle_t hh, int uplo, size_t n, double alpha, const double* x, size_t incx,
                          double* matrix, size_t lda) {
  CORAL_HANDLE(hh);
  return tri_g<double2, kHerG>(H, uplo, n, make_double2(alpha, 0.0), alpha == 0.0, x, incx, nullptr, 0, matrix,
                               lda, 16);
}

coral_status_t coral_cher2(coral_handle_t hh, int uplo, size_t n, const float alpha[2], const float* x,
                           size_t incx, const float* y, size_t incy, float* matrix, size_t lda) {
  CORAL_HANDLE(hh);
  if (!alpha) return bad_arg(H, 3);
  return tri_g<float2, kHer2G>(H, uplo, n, c2f(alpha), alpha[0] == 0.f && alpha[1] == 0.f, x, incx, y, incy,
                               matrix, lda, 8);
}

coral_status_t coral_zher2(coral_handle_t hh, int uplo, size_t n, const double alpha[2], const double* x,
                           size_t incx, const double* y, size_t incy, double* matrix, size_t lda) {
  CORAL_HANDLE(hh);
  if (!alpha) return bad_arg(H, 3);
  return tri_g<double2, kHer2G>(H, uplo, n, c2d(alpha), alpha[0] == 0.0 && alpha[1] == 0.0, x, incx, y, incy,
                                matrix, lda, 16);
}

}  // extern "C"
