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

// Vector form for unit-stride x (and y for the rank-2 updates) with A and
// those vectors on 16-byte boundaries and lda * sizeof(T) a multiple of 16.
// A thread owns one 16-byte vector of rows (kV elements): it loads their x
// (and y) once and updates them in kGCols columns. All of those columns' A
// vectors are loaded, together with the columns' coefficients, before the
// first is written back; a column whose coefficients are zero is loaded but
// not written (her2 excepted: its diagonal is made real in every column).
// Each element gets exactly k_rank_g's arithmetic. A vector that straddles
// the edge of a column's triangle, or the last row, is read and written
// element by element, in-range elements only.
// Columns per thread: 8, or 4 for CHER2, whose two complex coefficients per
// column would otherwise hold the kernel to two CTAs per SM.
template <typename T, int kKind>
constexpr int gcols() { return (kKind == kHer2G && sizeof(T) == 8) ? 2 : 8; }

template <typename T>
struct alignas(16) Pack16 {
  static constexpr int kV = (int)(16 / sizeof(T));
  T v[kV];
};

template <typename T, int kKind>
__global__ void __launch_bounds__(kRThreads, gcols<T, kKind>() < 8 ? 6 : (kKind == kSyr2G || kKind == kHer2G) ? 2 : 3)
k_rank_g_vec(int m, int n, T alpha, const T* __restrict__ x, const T* __restrict__ y, size_t incy,
             T* __restrict__ A, size_t lda, bool lower) {
  using F = Fld<T>;
  using P = Pack16<T>;
  constexpr int kV = P::kV;
  constexpr bool kTri = kKind >= kSyrG;
  constexpr bool kHerm = kKind == kHerG || kKind == kHer2G;
  constexpr bool kTwo = kKind == kSyr2G || kKind == kHer2G;
  constexpr int kGCols = gcols<T, kKind>();
  const int rows = kTri ? n : m;
  // rows [lo, hi) of column j that the update touches
  auto range = [&](int j, int& lo, int& hi) {
    lo = kTri ? (lower ? j : 0) : 0;
    hi = kTri ? (lower ? n : j + 1) : m;
  };
  // rows i0 .. i0+kV-1 of columns jg .. jg+kGCols-1
  auto block = [&](int i0, int jg) {
    const bool full_rows = i0 + kV <= rows;
    T xv[kV], yv[kV];
#pragma unroll
    for (int e = 0; e < kV; ++e) {
      const bool in = full_rows || i0 + e < rows;
      xv[e] = in ? x[i0 + e] : F::zero();
      yv[e] = kTwo && in ? y[i0 + e] : F::zero();
    }
    P a[kGCols];
    T c1[kGCols], c2[kGCols];
    unsigned on_mask = 0, whole_mask = 0;
#pragma unroll
    for (int c = 0; c < kGCols; ++c) {
      const int j = jg + c;
      int l, h;
      range(j, l, h);
      const bool on = j < n && i0 < h && i0 + kV > l;
      const bool whole = on && i0 >= l && i0 + kV <= h;
      on_mask |= on ? 1u << c : 0u;
      whole_mask |= whole ? 1u << c : 0u;
      c1[c] = c2[c] = F::zero();
      if (on) {
        // x and (for rank 2) y have unit stride here; GER's y may not
        if (kKind == kGerU) c1[c] = coeff<T, false>(alpha, y[(size_t)j * incy]);
        if (kKind == kGerC) c1[c] = coeff<T, true>(alpha, y[(size_t)j * incy]);
        if (kKind == kSyrG || kKind == kHerG) c1[c] = coeff<T, kHerm>(alpha, x[j]);
        if (kTwo) {
          c1[c] = coeff<T, kHerm>(alpha, y[j]);
          c2[c] = coeff<T, kHerm>(kHerm ? F::conj(alpha) : alpha, x[j]);
        }
      }
      const T* col = A + (size_t)(on ? j : 0) * lda + i0;
      if (whole) {
        a[c] = *reinterpret_cast<const P*>(col);
      } else {
#pragma unroll
        for (int e = 0; e < kV; ++e) a[c].v[e] = on && i0 + e >= l && i0 + e < h ? col[e] : F::zero();
      }
    }
#pragma unroll
    for (int c = 0; c < kGCols; ++c) {
      if (!(on_mask & (1u << c))) continue;
      const bool u1 = nz(c1[c]), u2 = nz(c2[c]);
      if (!u1 && !u2 && kKind != kHer2G) continue;  // column left untouched
      const int j = jg + c;
      int l, h;
      range(j, l, h);
#pragma unroll
      for (int e = 0; e < kV; ++e) {
        T v = a[c].v[e];
        if (u1) F::mac(v, xv[e], c1[c]);
        if (u2) F::mac(v, yv[e], c2[c]);
        if (kHerm && i0 + e == j) v = F::re(v);  // real diagonal
        a[c].v[e] = v;
      }
      T* col = A + (size_t)j * lda + i0;
      if (whole_mask & (1u << c)) {
        *reinterpret_cast<P*>(col) = a[c];
      } else {
#pragma unroll
        for (int e = 0; e < kV; ++e)
          if (i0 + e >= l && i0 + e < h) col[e] = a[c].v[e];
      }
    }
  };
  if (!kTri) {
    // grid: x = row chunks of kV * kRThreads rows, y = column groups
    const int i0 = (blockIdx.x * kRThreads + threadIdx.x) * kV;
    if (i0 >= rows) return;
    for (int jg = blockIdx.y * kGCols; jg < n; jg += gridDim.y * kGCols) block(i0, jg);
  } else {
    // grid: x = column groups, each walking only the row chunks its
    // triangle columns touch; upper takes the longest groups first
    const int ngroups = (n + kGCols - 1) / kGCols;
    for (int gi = blockIdx.x; gi < ngroups; gi += gridDim.x) {
      const int jg = (lower ? gi : ngroups - 1 - gi) * kGCols;
      const int jl = min(n, jg + kGCols) - 1;
      const int r_lo = lower ? jg : 0, r_hi = lower ? n : jl + 1;
      for (int rb = r_lo / (kV * kRThreads); rb * kV * kRThreads < r_hi; ++rb) {
        const int i0 = (rb * kRThreads + threadIdx.x) * kV;
        if (i0 < r_hi && i0 + kV > r_lo) block(i0, jg);
      }
    }
  }
}

template <typename T, int kKind>
coral_status_t launch_rank_g(Handle* h, size_t m, size_t n, T alpha, const T* x, size_t incx, const T* y,
                             size_t incy, T* A, size_t lda, bool lower) {
  if (m > INT32_MAX || n > INT32_MAX) return CORAL_ERR_NOT_SUPPORTED;
  const size_t rows = kKind >= kSyrG ? n : m;
  constexpr bool kTwo = kKind == kSyr2G || kKind == kHer2G;
  // complex128 keeps the element kernel: with one element per 16-byte
  // vector it already streams at 81-98% of HBM.
  constexpr bool kVecOk = sizeof(T) < 16;
  if constexpr (kVecOk) {  // the vector kernel is only instantiated where it is used
    if (incx == 1 && (!kTwo || incy == 1) && aligned16(A) && (lda * sizeof(T)) % 16 == 0 && aligned16(x) &&
        (!kTwo || aligned16(y))) {
      constexpr int kV = Pack16<T>::kV;
      constexpr int kGCols = gcols<T, kKind>();
      const size_t groups = (n + kGCols - 1) / kGCols;
      const dim3 vgrid = kKind < kSyrG
          ? dim3((unsigned)((rows + (size_t)kV * kRThreads - 1) / ((size_t)kV * kRThreads)),
                 (unsigned)(groups < 65535 ? groups : 65535))
          : dim3((unsigned)(groups < (1u << 30) ? groups : (1u << 30)));
      k_rank_g_vec<T, kKind><<<vgrid, kRThreads, 0, h->stream>>>((int)m, (int)n, alpha, x, y, incy, A, lda,
                                                                   lower);
      return launch_status(h);
    }
  }
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
