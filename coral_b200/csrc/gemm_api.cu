// C-ABI entry points of level 3: argument checks, quick returns and the
// dispatch between native FMA tiles and the emulated tensor-core paths
// selected by the handle's GEMM mode.
#include "common.cuh"

namespace coral {

int gemm_bad_arg(int op_a, int op_b, size_t m, size_t n, size_t k, const void* a, size_t lda,
                 const void* b, size_t ldb, const void* c, size_t ldc, bool complex_ops);
template <typename T>
coral_status_t enqueue_gemm_simt(Handle* h, int op_a, int op_b, size_t m, size_t n, size_t k,
                                 T alpha, const T* A, size_t lda, const T* B, size_t ldb, T beta,
                                 T* C, size_t ldc);
coral_status_t enqueue_sgemm_split(Handle* h, int terms, int op_a, int op_b, size_t m, size_t n,
                                   size_t k, float alpha, const float* A, size_t lda,
                                   const float* B, size_t ldb, float beta, float* C, size_t ldc);
coral_status_t enqueue_dgemm_ozaki(Handle* h, int op_a, int op_b, size_t m, size_t n, size_t k,
                                   double alpha, const double* A, size_t lda, const double* B,
                                   size_t ldb, double beta, double* C, size_t ldc);
coral_status_t enqueue_cgemm_split(Handle* h, int terms, int op_a, int op_b, size_t m, size_t n,
                                   size_t k, float2 alpha, const float2* A, size_t lda,
                                   const float2* B, size_t ldb, float2 beta, float2* C, size_t ldc);
coral_status_t enqueue_zgemm_ozaki(Handle* h, int op_a, int op_b, size_t m, size_t n, size_t k,
                                   double2 alpha, const double2* A, size_t lda, const double2* B,
                                   size_t ldb, double2 beta, double2* C, size_t ldc);

static coral_status_t check(Handle* H, int op_a, int op_b, size_t m, size_t n, size_t k,
                            const void* a, size_t lda, const void* b, size_t ldb, const void* c,
                            size_t ldc) {
  int bad = gemm_bad_arg(op_a, op_b, m, n, k, a, lda, b, ldb, c, ldc, true);
  if (bad > 0) return bad_arg(H, bad);
  if (bad < 0) return CORAL_ERR_NOT_SUPPORTED;
  return CORAL_OK;
}

}  // namespace coral

using namespace coral;

extern "C" {

coral_status_t coral_sgemm(coral_handle_t hh, int op_a, int op_b, size_t m, size_t n, size_t k,
                           float alpha, const float* a, size_t lda, const float* b, size_t ldb,
                           float beta, float* c, size_t ldc) {
  CORAL_HANDLE(hh);
  coral_status_t s = check(H, op_a, op_b, m, n, k, a, lda, b, ldb, c, ldc);
  if (s != CORAL_OK) return s;
  const bool compute = m && n && k && alpha != 0.0f;
  if (compute && (H->gemm_mode == CORAL_GEMM_SPLIT_BF16X3 || H->gemm_mode == CORAL_GEMM_SPLIT_BF16X6))
    return enqueue_sgemm_split(H, H->gemm_mode == CORAL_GEMM_SPLIT_BF16X6 ? 6 : 3, op_a, op_b, m,
                               n, k, alpha, a, lda, b, ldb, beta, c, ldc);
  return enqueue_gemm_simt<float>(H, op_a, op_b, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc);
}

coral_status_t coral_dgemm(coral_handle_t hh, int op_a, int op_b, size_t m, size_t n, size_t k,
                           double alpha, const double* a, size_t lda, const double* b, size_t ldb,
                           double beta, double* c, size_t ldc) {
  CORAL_HANDLE(hh);
  coral_status_t s = check(H, op_a, op_b, m, n, k, a, lda, b, ldb, c, ldc);
  if (s != CORAL_OK) return s;
  const bool compute = m && n && k && alpha != 0.0;
  if (compute && H->gemm_mode == CORAL_GEMM_OZAKI_INT8)
    return enqueue_dgemm_ozaki(H, op_a, op_b, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc);
  return enqueue_gemm_simt<double>(H, op_a, op_b, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc);
}

coral_status_t coral_cgemm(coral_handle_t hh, int op_a, int op_b, size_t m, size_t n, size_t k,
                           const float alpha[2], const float* a, size_t lda, const float* b,
                           size_t ldb, const float beta[2], float* c, size_t ldc) {
  CORAL_HANDLE(hh);
  if (!alpha) return bad_arg(H, 6);
  if (!beta) return bad_arg(H, 11);
  coral_status_t s = check(H, op_a, op_b, m, n, k, a, lda, b, ldb, c, ldc);
  if (s != CORAL_OK) return s;
  if (((uintptr_t)a | (uintptr_t)b | (uintptr_t)c) & 7) return bad_arg(H, 7);  // complex64 alignment
  float2 al = make_float2(alpha[0], alpha[1]), be = make_float2(beta[0], beta[1]);
  const bool compute = m && n && k && !(alpha[0] == 0.f && alpha[1] == 0.f);
  if (compute && (H->gemm_mode == CORAL_GEMM_SPLIT_BF16X3 || H->gemm_mode == CORAL_GEMM_SPLIT_BF16X6))
    return enqueue_cgemm_split(H, H->gemm_mode == CORAL_GEMM_SPLIT_BF16X6 ? 6 : 3, op_a, op_b, m,
                               n, k, al, reinterpret_cast<const float2*>(a), lda,
                               reinterpret_cast<const float2*>(b), ldb, be,
                               reinterpret_cast<float2*>(c), ldc);
  return enqueue_gemm_simt<float2>(H, op_a, op_b, m, n, k, al, reinterpret_cast<const float2*>(a),
                                   lda, reinterpret_cast<const float2*>(b), ldb, be,
                                   reinterpret_cast<float2*>(c), ldc);
}

coral_status_t coral_zgemm(coral_handle_t hh, int op_a, int op_b, size_t m, size_t n, size_t k,
                           const double alpha[2], const double* a, size_t lda, const double* b,
                           size_t ldb, const double beta[2], double* c, size_t ldc) {
  CORAL_HANDLE(hh);
  if (!alpha) return bad_arg(H, 6);
  if (!beta) return bad_arg(H, 11);
  coral_status_t s = check(H, op_a, op_b, m, n, k, a, lda, b, ldb, c, ldc);
  if (s != CORAL_OK) return s;
  if (((uintptr_t)a | (uintptr_t)b | (uintptr_t)c) & 15) return bad_arg(H, 7);  // complex128 alignment
  double2 al = make_double2(alpha[0], alpha[1]), be = make_double2(beta[0], beta[1]);
  const bool compute = m && n && k && !(alpha[0] == 0.0 && alpha[1] == 0.0);
  if (compute && H->gemm_mode == CORAL_GEMM_OZAKI_INT8)
    return enqueue_zgemm_ozaki(H, op_a, op_b, m, n, k, al, reinterpret_cast<const double2*>(a), lda,
                               reinterpret_cast<const double2*>(b), ldb, be,
                               reinterpret_cast<double2*>(c), ldc);
  return enqueue_gemm_simt<double2>(H, op_a, op_b, m, n, k, al, reinterpret_cast<const double2*>(a),
                                    lda, reinterpret_cast<const double2*>(b), ldb, be,
                                    reinterpret_cast<double2*>(c), ldc);
}

}  // extern "C"
