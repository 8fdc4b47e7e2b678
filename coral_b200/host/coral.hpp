// coral.hpp -- C++ host mirror of CORAL's routine signatures over the C ABI.
//
// The reference (coral-aarch64/src) exposes free functions in modules
// `level1`, `level2`, `level3` with the enums of enums.rs; this header gives
// the same names, argument order and meaning in namespace `coral`, with Rust
// slices as (pointer) arguments in host memory.  Each call goes through one
// host-slice entry point of libcoral_b200 (coral_host_*: arguments checked,
// copy in, compute on the GPU, copy out, synchronise).  Errors throw
// coral::Error (the reference panics in debug builds).
#pragma once

#include <cstddef>
#include <stdexcept>
#include <string>

#include "../../include/coral_b200.h"

namespace coral {

enum class CoralTranspose : int { NoTranspose = 0, Transpose = 1, ConjugateTranspose = 2 };
enum class CoralTriangular : int { UpperTriangular = 0, LowerTriangular = 1 };
enum class CoralDiagonal : int { UnitDiagonal = 0, NonUnitDiagonal = 1 };

struct Error : std::runtime_error {
  coral_status_t status;
  Error(const char* routine, coral_status_t s)
      : std::runtime_error(std::string(routine) + ": " + coral_status_string(s)), status(s) {}
};

inline void check(const char* routine, coral_status_t s) {
  if (s != CORAL_OK) throw Error(routine, s);
}

namespace level3 {
// sgemm.rs:106-130
inline void sgemm(CoralTranspose op_a, CoralTranspose op_b, size_t m, size_t n, size_t k,
                  float alpha, const float* a, size_t lda, const float* b, size_t ldb, float beta,
                  float* c, size_t ldc) {
  check("sgemm", coral_host_sgemm(static_cast<int>(op_a), static_cast<int>(op_b), m, n, k, alpha,
                                  a, lda, b, ldb, beta, c, ldc));
}
// dgemm.rs:107
inline void dgemm(CoralTranspose op_a, CoralTranspose op_b, size_t m, size_t n, size_t k,
                  double alpha, const double* a, size_t lda, const double* b, size_t ldb,
                  double beta, double* c, size_t ldc) {
  check("dgemm", coral_host_dgemm(static_cast<int>(op_a), static_cast<int>(op_b), m, n, k, alpha,
                                  a, lda, b, ldb, beta, c, ldc));
}
// cgemm.rs:127-157 (alpha, beta: [re, im]; interleaved complex64 operands)
inline void cgemm(CoralTranspose op_a, CoralTranspose op_b, size_t m, size_t n, size_t k,
                  const float alpha[2], const float* a, size_t lda, const float* b, size_t ldb,
                  const float beta[2], float* c, size_t ldc) {
  check("cgemm", coral_host_cgemm(static_cast<int>(op_a), static_cast<int>(op_b), m, n, k, alpha,
                                  a, lda, b, ldb, beta, c, ldc));
}
// zgemm.rs:123
inline void zgemm(CoralTranspose op_a, CoralTranspose op_b, size_t m, size_t n, size_t k,
                  const double alpha[2], const double* a, size_t lda, const double* b, size_t ldb,
                  const double beta[2], double* c, size_t ldc) {
  check("zgemm", coral_host_zgemm(static_cast<int>(op_a), static_cast<int>(op_b), m, n, k, alpha,
                                  a, lda, b, ldb, beta, c, ldc));
}
}  // namespace level3

namespace level2 {
// sgemv.rs:63-80
inline void sgemv(CoralTranspose trans, size_t n_rows, size_t n_cols, float alpha,
                  const float* matrix, size_t lda, const float* x, size_t incx, float beta,
                  float* y, size_t incy) {
  check("sgemv", coral_host_sgemv(static_cast<int>(trans), n_rows, n_cols, alpha, matrix, lda, x,
                                  incx, beta, y, incy));
}
// strsv.rs:60-74
inline void strsv(CoralTriangular uplo, CoralTranspose trans, CoralDiagonal diag, size_t n,
                  const float* matrix, size_t lda, float* x, size_t incx) {
  check("strsv", coral_host_strsv(static_cast<int>(uplo), static_cast<int>(trans),
                                  static_cast<int>(diag), n, matrix, lda, x, incx));
}
// strmv.rs:59-73
inline void strmv(CoralTriangular uplo, CoralTranspose trans, CoralDiagonal diag, size_t n,
                  const float* matrix, size_t lda, float* x, size_t incx) {
  check("strmv", coral_host_strmv(static_cast<int>(uplo), static_cast<int>(trans),
                                  static_cast<int>(diag), n, matrix, lda, x, incx));
}
// ssymv.rs:99-110
inline void ssymv(CoralTriangular uplo, size_t n, float alpha, const float* matrix, size_t lda,
                  const float* x, size_t incx, float beta, float* y, size_t incy) {
  check("ssymv", coral_host_ssymv(static_cast<int>(uplo), n, alpha, matrix, lda, x, incx, beta, y,
                                  incy));
}
// chemv.rs:96-107
inline void chemv(CoralTriangular uplo, size_t n, const float alpha[2], const float* matrix,
                  size_t lda, const float* x, size_t incx, const float beta[2], float* y,
                  size_t incy) {
  check("chemv", coral_host_chemv(static_cast<int>(uplo), n, alpha, matrix, lda, x, incx, beta, y,
                                  incy));
}
// sger.rs:68-78
inline void sger(size_t n_rows, size_t n_cols, float alpha, const float* x, size_t incx,
                 const float* y, size_t incy, float* matrix, size_t lda) {
  check("sger", coral_host_sger(n_rows, n_cols, alpha, x, incx, y, incy, matrix, lda));
}
// ssyr.rs:63-71
inline void ssyr(CoralTriangular uplo, size_t n, float alpha, const float* x, size_t incx,
                 float* matrix, size_t lda) {
  check("ssyr", coral_host_ssyr(static_cast<int>(uplo), n, alpha, x, incx, matrix, lda));
}
// ssyr2.rs:59-69
inline void ssyr2(CoralTriangular uplo, size_t n, float alpha, const float* x, size_t incx,
                  const float* y, size_t incy, float* matrix, size_t lda) {
  check("ssyr2", coral_host_ssyr2(static_cast<int>(uplo), n, alpha, x, incx, y, incy, matrix, lda));
}
}  // namespace level2

namespace level1 {
// sdot.rs:42-161
inline float sdot(size_t n, const float* x, size_t incx, const float* y, size_t incy) {
  float r = 0.0f;
  check("sdot", coral_host_sdot(n, x, incx, y, incy, &r));
  return r;
}
// saxpy.rs:42-131
inline void saxpy(size_t n, float alpha, const float* x, size_t incx, float* y, size_t incy) {
  check("saxpy", coral_host_saxpy(n, alpha, x, incx, y, incy));
}
// isamax.rs:43-151
inline size_t isamax(size_t n, const float* x, size_t incx) {
  size_t r = 0;
  check("isamax", coral_host_isamax(n, x, incx, &r));
  return r;
}
// snrm2.rs:45-149
inline float snrm2(size_t n, const float* x, size_t incx) {
  float r = 0.0f;
  check("snrm2", coral_host_snrm2(n, x, incx, &r));
  return r;
}
// scopy.rs:28-58
inline void scopy(size_t n, const float* x, size_t incx, float* y, size_t incy) {
  check("scopy", coral_host_scopy(n, x, incx, y, incy));
}
// sswap.rs:35-118
inline void sswap(size_t n, float* x, size_t incx, float* y, size_t incy) {
  check("sswap", coral_host_sswap(n, x, incx, y, incy));
}
// sscal.rs:30-66
inline void sscal(size_t n, float alpha, float* x, size_t incx) {
  check("sscal", coral_host_sscal(n, alpha, x, incx));
}
}  // namespace level1

// Selects the GEMM arithmetic of this thread's host-slice calls.
inline void set_gemm_mode(int mode) { check("set_gemm_mode", coral_host_set_gemm_mode(mode)); }

}  // namespace coral
