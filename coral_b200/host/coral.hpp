// coral.hpp -- C++ host mirror of CORAL's routine signatures over the C ABI.
//
// The reference (coral-aarch64/src) exposes free functions in modules
// `level1`, `level2`, `level3` with the enums of enums.rs; this header gives
// the same names, argument order and meaning in namespace `coral`, with Rust
// slices as (pointer) arguments in host memory.  Each call goes through the
// host-slice entry points of libcoral_b200 (copy in, compute on the GPU, copy
// out) or, for routines without one, through a per-thread handle and
// device staging managed here.  Errors throw coral::Error (the reference
// panics in debug builds).
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
}  // namespace level1

// Selects the GEMM arithmetic of this thread's host-slice calls.
inline void set_gemm_mode(int mode) { check("set_gemm_mode", coral_host_set_gemm_mode(mode)); }

}  // namespace coral
