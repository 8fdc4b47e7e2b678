/*
 * coral_b200.h -- C ABI of the B200 BLAS engine.
 *
 * Drop-in boundary for CORAL's column-major BLAS routines (devdeliw/CORAL,
 * crate coral-blas-aarch64).  Every routine keeps the reference's argument
 * order and meaning; what changes is only what the Rust signature cannot say
 * across an FFI boundary:
 *
 *   - a leading `coral_handle_t` carries the CUDA stream, scratch memory and
 *     the device status word (bounded waits report CORAL_ERR_TIMEOUT);
 *   - Rust slices become a plain pointer (length is implied by n/inc/ld, the
 *     same relation the reference checks with `required_len_ok*`,
 *     coral-aarch64/src/level1/assert_length_helpers.rs:8-15 and
 *     coral-aarch64/src/level2/assert_length_helpers.rs:4-16);
 *   - complex scalars `[f32; 2]` / `[f64; 2]` become `const float[2]` /
 *     `const double[2]` (host memory);
 *   - scalar results (`sdot`, `snrm2`, `isamax`) come back through an
 *     out-pointer, interpreted per the handle's pointer mode (host by default);
 *   - every call returns a coral_status_t instead of panicking.
 *
 * Matrix/vector pointers of the `coral_*` entry points are DEVICE pointers;
 * kernels are enqueued on the handle's stream and the call returns without
 * waiting (scalar results in host pointer mode wait for the stream).
 * The `coral_host_*` entry points take HOST pointers with exactly the
 * reference's argument list and semantics (no handle): they copy in, compute,
 * copy out and synchronise, so a caller that holds host slices -- as every
 * caller of the reference does -- can switch with no other change.
 *
 * Enum values follow the declaration order of coral-aarch64/src/enums.rs:1-18
 * (what `as i32` yields on the Rust side):
 *   CoralTranspose  { NoTranspose = 0, Transpose = 1, ConjugateTranspose = 2 }
 *   CoralTriangular { UpperTriangular = 0, LowerTriangular = 1 }
 *   CoralDiagonal   { UnitDiagonal = 0, NonUnitDiagonal = 1 }
 *
 * Increments are unsigned (`usize` in the reference) and must be >= 1 where
 * the reference asserts `inc > 0`.
 */
#ifndef CORAL_B200_H
#define CORAL_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CORAL_B200_ABI_VERSION 1

typedef enum coral_status {
  CORAL_OK = 0,
  CORAL_ERR_INVALID_ARG = 1,   /* argument check failed (see coral_last_bad_arg) */
  CORAL_ERR_CUDA = 2,          /* a CUDA runtime call failed */
  CORAL_ERR_TIMEOUT = 3,       /* a bounded device wait gave up (status word set) */
  CORAL_ERR_ALLOC = 4,         /* device/host allocation failed */
  CORAL_ERR_NOT_SUPPORTED = 5, /* size or mode outside what the kernels handle */
  CORAL_ERR_NO_DEVICE = 6      /* no sm_100 device visible */
} coral_status_t;

enum { CORAL_NO_TRANSPOSE = 0, CORAL_TRANSPOSE = 1, CORAL_CONJ_TRANSPOSE = 2 };
enum { CORAL_UPPER = 0, CORAL_LOWER = 1 };
enum { CORAL_UNIT = 0, CORAL_NON_UNIT = 1 };
enum { CORAL_POINTER_HOST = 0, CORAL_POINTER_DEVICE = 1 };

/* GEMM arithmetic for coral_sgemm / coral_cgemm / coral_dgemm / coral_zgemm. */
enum {
  CORAL_GEMM_NATIVE = 0,       /* FP32/FP64 FMA pipes, (complex: direct 4M) */
  CORAL_GEMM_SPLIT_BF16X3 = 1, /* s/c: 2-way BF16 split, 3 tcgen05 products */
  CORAL_GEMM_OZAKI_INT8 = 2,   /* d/z: INT8-slice emulation on tcgen05 */
  CORAL_GEMM_SPLIT_BF16X6 = 3  /* s/c: 3-way BF16 split, 6 tcgen05 products */
};

/* How the emulated complex GEMMs (coral_cgemm in the split-BF16 modes,
 * coral_zgemm in the Ozaki mode) map onto real tensor-core products. */
enum {
  CORAL_COMPLEX_4M = 0, /* one real GEMM of m x 2n x 2k: Re and Im exact per term */
  CORAL_COMPLEX_3M = 1  /* three real GEMMs of m x n x k (3/4 of the work); the
                           imaginary part is T3 - T1 - T2, with its error bounded
                           by (|Re A| + |Im A|)(|Re B| + |Im B|) */
};

/* Kernel form of SYMV / HEMV / TRMV (coral_set_strip_form). */
enum {
  CORAL_STRIPS_REGISTER = 0, /* register-streaming strips, diagonal tiles on a side stream, combine */
  CORAL_STRIPS_TMA = 1       /* one TMA-fed persistent pass over the whole triangle, combine */
};

typedef struct coral_handle_s* coral_handle_t;

/* ---- handle ------------------------------------------------------------ */
/* No reference counterpart: CORAL's routines are stateless free functions
 * (coral-aarch64/src/lib.rs:70-82 exports modules of plain `pub fn`s).  The
 * handle holds the stream, the device scratch, the status word that bounded
 * waits set, and the per-handle configuration. */
coral_status_t coral_create(coral_handle_t* handle);
coral_status_t coral_destroy(coral_handle_t handle);
/* `stream` is a cudaStream_t (NULL = legacy default stream). */
coral_status_t coral_set_stream(coral_handle_t handle, void* stream);
coral_status_t coral_get_stream(coral_handle_t handle, void** stream);
coral_status_t coral_set_pointer_mode(coral_handle_t handle, int mode);
coral_status_t coral_set_gemm_mode(coral_handle_t handle, int mode);
coral_status_t coral_get_gemm_mode(coral_handle_t handle, int* mode);
/* K depth, in 64-element slabs, of each tensor-core accumulation chunk of the
 * split-BF16 GEMMs before it is added into fp32 registers (default 16). */
coral_status_t coral_set_split_chunk(coral_handle_t handle, int slabs);
/* Complex mapping of the emulated CGEMM / ZGEMM: CORAL_COMPLEX_4M (default) or 3M. */
coral_status_t coral_set_complex_mapping(coral_handle_t handle, int mapping);
/* Kernel form of the SYMV / HEMV / TRMV family: CORAL_STRIPS_REGISTER
 * (default, the faster on the measured sizes) or CORAL_STRIPS_TMA (used when
 * the matrix is 16-byte aligned with a leading dimension of a multiple of 16
 * bytes, else the register form runs). Results agree to rounding; the two
 * forms add the partials of a row in different orders. */
coral_status_t coral_set_strip_form(coral_handle_t handle, int form);
/* Iteration limit of every bounded device wait (0 restores the default). */
coral_status_t coral_set_wait_limit(coral_handle_t handle, uint64_t spins);
/* Kernel timing: when enabled, the handle brackets the dominant kernel of each
 * call (the GEMM main loop for level 3) with CUDA events on its stream;
 * coral_get_kernel_timing waits for the stream and returns the summed
 * duration (ms) and number of timed launches since the last query. */
coral_status_t coral_set_kernel_timing(coral_handle_t handle, int enable);
coral_status_t coral_get_kernel_timing(coral_handle_t handle, double* total_ms, uint64_t* launches);
/* Wait for the stream, then report and clear the device status word. */
coral_status_t coral_sync(coral_handle_t handle);
/* 1-based position of the offending argument after CORAL_ERR_INVALID_ARG
 * (the handle counts as position 0), as BLAS xerbla reports it. */
int coral_last_bad_arg(coral_handle_t handle);
const char* coral_status_string(coral_status_t status);
const char* coral_last_cuda_error(coral_handle_t handle);
int coral_abi_version(void);
/* Number of CUDA kernels this library has launched in this process. */
uint64_t coral_kernel_launches(void);

/* ---- level 1 (coral-aarch64/src/level1) --------------------------------- */
/* sdot.rs:42-161 */
coral_status_t coral_sdot(coral_handle_t h, size_t n, const float* x, size_t incx,
                          const float* y, size_t incy, float* result);
/* saxpy.rs:42-131 */
coral_status_t coral_saxpy(coral_handle_t h, size_t n, float alpha, const float* x,
                           size_t incx, float* y, size_t incy);
/* snrm2.rs:45-149 */
coral_status_t coral_snrm2(coral_handle_t h, size_t n, const float* x, size_t incx,
                           float* result);
/* isamax.rs:43-151 -- 0-based index of the first max |x_i| */
coral_status_t coral_isamax(coral_handle_t h, size_t n, const float* x, size_t incx,
                            size_t* index);
/* scopy.rs:28-58 */
coral_status_t coral_scopy(coral_handle_t h, size_t n, const float* x, size_t incx,
                           float* y, size_t incy);
/* sswap.rs:35-118 */
coral_status_t coral_sswap(coral_handle_t h, size_t n, float* x, size_t incx,
                           float* y, size_t incy);
/* sscal.rs:30-66 */
coral_status_t coral_sscal(coral_handle_t h, size_t n, float alpha, float* x,
                           size_t incx);

/* Double and complex level 1.  Complex vectors are interleaved (re, im) and
 * increments count complex elements; complex scalars are [re, im] arrays.
 * Scalar results follow the pointer mode like coral_sdot; complex results
 * are written as two words. */
/* ddot.rs:43-163 */
coral_status_t coral_ddot(coral_handle_t h, size_t n, const double* x, size_t incx,
                          const double* y, size_t incy, double* result);
/* cdotu.rs:46-178 -- sum x_i y_i */
coral_status_t coral_cdotu(coral_handle_t h, size_t n, const float* x, size_t incx,
                           const float* y, size_t incy, float result[2]);
/* cdotc.rs:46-176 -- sum conj(x_i) y_i */
coral_status_t coral_cdotc(coral_handle_t h, size_t n, const float* x, size_t incx,
                           const float* y, size_t incy, float result[2]);
/* zdotu.rs:45-176 */
coral_status_t coral_zdotu(coral_handle_t h, size_t n, const double* x, size_t incx,
                           const double* y, size_t incy, double result[2]);
/* zdotc.rs:45-175 */
coral_status_t coral_zdotc(coral_handle_t h, size_t n, const double* x, size_t incx,
                           const double* y, size_t incy, double result[2]);
/* sasum.rs:40-107, dasum.rs:41-110 -- sum |x_i| */
coral_status_t coral_sasum(coral_handle_t h, size_t n, const float* x, size_t incx,
                           float* result);
coral_status_t coral_dasum(coral_handle_t h, size_t n, const double* x, size_t incx,
                           double* result);
/* scasum.rs:40-108, dzasum.rs:40-111 -- sum |re| + |im| */
coral_status_t coral_scasum(coral_handle_t h, size_t n, const float* x, size_t incx,
                            float* result);
coral_status_t coral_dzasum(coral_handle_t h, size_t n, const double* x, size_t incx,
                            double* result);
/* dnrm2.rs:45-152, scnrm2.rs:44-155, dznrm2.rs:43-156 */
coral_status_t coral_dnrm2(coral_handle_t h, size_t n, const double* x, size_t incx,
                           double* result);
coral_status_t coral_scnrm2(coral_handle_t h, size_t n, const float* x, size_t incx,
                            float* result);
coral_status_t coral_dznrm2(coral_handle_t h, size_t n, const double* x, size_t incx,
                            double* result);
/* idamax.rs:43-159, icamax.rs:48-166, izamax.rs:33-163 -- 0-based index of
 * the first max |x_i| (|re| + |im| for complex) */
coral_status_t coral_idamax(coral_handle_t h, size_t n, const double* x, size_t incx,
                            size_t* index);
coral_status_t coral_icamax(coral_handle_t h, size_t n, const float* x, size_t incx,
                            size_t* index);
coral_status_t coral_izamax(coral_handle_t h, size_t n, const double* x, size_t incx,
                            size_t* index);
/* daxpy.rs:42-133, caxpy.rs:45-172, zaxpy.rs:44-172 */
coral_status_t coral_daxpy(coral_handle_t h, size_t n, double alpha, const double* x,
                           size_t incx, double* y, size_t incy);
coral_status_t coral_caxpy(coral_handle_t h, size_t n, const float alpha[2],
                           const float* x, size_t incx, float* y, size_t incy);
coral_status_t coral_zaxpy(coral_handle_t h, size_t n, const double alpha[2],
                           const double* x, size_t incx, double* y, size_t incy);
/* dscal.rs:30-66, cscal.rs:43-111, zscal.rs:41-109, csscal.rs:39-88 and
 * zdscal.rs:38-88 (real alpha on complex x) */
coral_status_t coral_dscal(coral_handle_t h, size_t n, double alpha, double* x,
                           size_t incx);
coral_status_t coral_cscal(coral_handle_t h, size_t n, const float alpha[2], float* x,
                           size_t incx);
coral_status_t coral_zscal(coral_handle_t h, size_t n, const double alpha[2], double* x,
                           size_t incx);
coral_status_t coral_csscal(coral_handle_t h, size_t n, float alpha, float* x,
                            size_t incx);
coral_status_t coral_zdscal(coral_handle_t h, size_t n, double alpha, double* x,
                            size_t incx);
/* dcopy.rs:28-57, ccopy.rs:29-58, zcopy.rs:28-61 */
coral_status_t coral_dcopy(coral_handle_t h, size_t n, const double* x, size_t incx,
                           double* y, size_t incy);
coral_status_t coral_ccopy(coral_handle_t h, size_t n, const float* x, size_t incx,
                           float* y, size_t incy);
coral_status_t coral_zcopy(coral_handle_t h, size_t n, const double* x, size_t incx,
                           double* y, size_t incy);
/* dswap.rs:35-119, cswap.rs:36-120, zswap.rs:35-120 */
coral_status_t coral_dswap(coral_handle_t h, size_t n, double* x, size_t incx,
                           double* y, size_t incy);
coral_status_t coral_cswap(coral_handle_t h, size_t n, float* x, size_t incx,
                           float* y, size_t incy);
coral_status_t coral_zswap(coral_handle_t h, size_t n, double* x, size_t incx,
                           double* y, size_t incy);
/* srot.rs:51-180, drot.rs:48-178, csrot.rs:50-166, zdrot.rs:51-166 --
 * x' = c x + s y, y' = c y - s x with real c, s */
coral_status_t coral_srot(coral_handle_t h, size_t n, float* x, size_t incx, float* y,
                          size_t incy, float c, float s);
coral_status_t coral_drot(coral_handle_t h, size_t n, double* x, size_t incx, double* y,
                          size_t incy, double c, double s);
coral_status_t coral_csrot(coral_handle_t h, size_t n, float* x, size_t incx, float* y,
                           size_t incy, float c, float s);
coral_status_t coral_zdrot(coral_handle_t h, size_t n, double* x, size_t incx, double* y,
                           size_t incy, double c, double s);
/* srotm.rs:47-412, drotm.rs:47-410 -- param = [flag, h11, h21, h12, h22] in
 * host memory */
coral_status_t coral_srotm(coral_handle_t h, size_t n, float* x, size_t incx, float* y,
                           size_t incy, const float param[5]);
coral_status_t coral_drotm(coral_handle_t h, size_t n, double* x, size_t incx, double* y,
                           size_t incy, const double param[5]);
/* srotg.rs:40-75, drotg.rs:40-71 -- a, b, c, s follow the pointer mode */
coral_status_t coral_srotg(coral_handle_t h, float* a, float* b, float* c, float* s);
coral_status_t coral_drotg(coral_handle_t h, double* a, double* b, double* c, double* s);
/* srotmg.rs:42-199, drotmg.rs:41-195 -- d1, d2, x1 and param follow the
 * pointer mode; y1 by value */
coral_status_t coral_srotmg(coral_handle_t h, float* d1, float* d2, float* x1, float y1,
                            float param[5]);
coral_status_t coral_drotmg(coral_handle_t h, double* d1, double* d2, double* x1,
                            double y1, double param[5]);

/* ---- fused level 1.5 (coral-aarch64/src/level1_special) ------------------ */
/* y[0..n_rows) += A x (x: n_cols elements), the reference's argument lists:
 * saxpyf.rs:36-513, daxpyf.rs:45-518, caxpyf.rs:48-696, zaxpyf.rs:49-697 */
coral_status_t coral_saxpyf(coral_handle_t h, size_t n_rows, size_t n_cols, const float* x,
                            size_t incx, const float* matrix, size_t lda, float* y, size_t incy);
coral_status_t coral_daxpyf(coral_handle_t h, size_t n_rows, size_t n_cols, const double* x,
                            size_t incx, const double* matrix, size_t lda, double* y, size_t incy);
coral_status_t coral_caxpyf(coral_handle_t h, size_t n_rows, size_t n_cols, const float* x,
                            size_t incx, const float* matrix, size_t lda, float* y, size_t incy);
coral_status_t coral_zaxpyf(coral_handle_t h, size_t n_rows, size_t n_cols, const double* x,
                            size_t incx, const double* matrix, size_t lda, double* y, size_t incy);
/* out[0..n_cols) += A^T x (x: n_rows elements, out contiguous): sdotf.rs:37-600,
 * ddotf.rs:37-596, cdotuf.rs:41-764, zdotuf.rs:41-665; out += A^H x:
 * cdotcf.rs:42-765, zdotcf.rs:41-1000 */
coral_status_t coral_sdotf(coral_handle_t h, size_t n_rows, size_t n_cols, const float* matrix,
                           size_t lda, const float* x, size_t incx, float* out);
coral_status_t coral_ddotf(coral_handle_t h, size_t n_rows, size_t n_cols, const double* matrix,
                           size_t lda, const double* x, size_t incx, double* out);
coral_status_t coral_cdotuf(coral_handle_t h, size_t n_rows, size_t n_cols, const float* matrix,
                            size_t lda, const float* x, size_t incx, float* out);
coral_status_t coral_cdotcf(coral_handle_t h, size_t n_rows, size_t n_cols, const float* matrix,
                            size_t lda, const float* x, size_t incx, float* out);
coral_status_t coral_zdotuf(coral_handle_t h, size_t n_rows, size_t n_cols, const double* matrix,
                            size_t lda, const double* x, size_t incx, double* out);
coral_status_t coral_zdotcf(coral_handle_t h, size_t n_rows, size_t n_cols, const double* matrix,
                            size_t lda, const double* x, size_t incx, double* out);

/* ---- level 2 (coral-aarch64/src/level2) --------------------------------- */
/* sgemv.rs:63-80 */
coral_status_t coral_sgemv(coral_handle_t h, int trans, size_t n_rows, size_t n_cols,
                           float alpha, const float* matrix, size_t lda,
                           const float* x, size_t incx, float beta, float* y,
                           size_t incy);
/* dgemv.rs (dgemv_notranspose.rs / dgemv_transpose.rs) -- same arguments as
 * sgemv in double; ConjugateTranspose == Transpose */
coral_status_t coral_dgemv(coral_handle_t h, int trans, size_t n_rows, size_t n_cols,
                           double alpha, const double* matrix, size_t lda,
                           const double* x, size_t incx, double beta, double* y,
                           size_t incy);
/* cgemv.rs:60-80 -- interleaved complex64, ld/inc in complex units; trans
 * N, T or C (conjugate transpose) */
coral_status_t coral_cgemv(coral_handle_t h, int trans, size_t n_rows, size_t n_cols,
                           const float alpha[2], const float* matrix, size_t lda,
                           const float* x, size_t incx, const float beta[2], float* y,
                           size_t incy);
/* zgemv.rs -- interleaved complex128, as cgemv */
coral_status_t coral_zgemv(coral_handle_t h, int trans, size_t n_rows, size_t n_cols,
                           const double alpha[2], const double* matrix, size_t lda,
                           const double* x, size_t incx, const double beta[2], double* y,
                           size_t incy);
/* ssymv.rs:99-110 */
coral_status_t coral_ssymv(coral_handle_t h, int uplo, size_t n, float alpha,
                           const float* matrix, size_t lda, const float* x,
                           size_t incx, float beta, float* y, size_t incy);
/* chemv.rs:96-107 -- interleaved (re, im) complex64, ld in complex units */
coral_status_t coral_chemv(coral_handle_t h, int uplo, size_t n, const float alpha[2],
                           const float* matrix, size_t lda, const float* x,
                           size_t incx, const float beta[2], float* y, size_t incy);
/* dsymv.rs:99-110 -- double */
coral_status_t coral_dsymv(coral_handle_t h, int uplo, size_t n, double alpha,
                           const double* matrix, size_t lda, const double* x,
                           size_t incx, double beta, double* y, size_t incy);
/* zhemv.rs:96-107 -- interleaved complex128 */
coral_status_t coral_zhemv(coral_handle_t h, int uplo, size_t n, const double alpha[2],
                           const double* matrix, size_t lda, const double* x,
                           size_t incx, const double beta[2], double* y, size_t incy);
/* dtrmv.rs -- double; ConjugateTranspose == Transpose */
coral_status_t coral_dtrmv(coral_handle_t h, int uplo, int trans, int diag, size_t n,
                           const double* matrix, size_t lda, double* x, size_t incx);
/* ctrmv.rs:58-72 -- interleaved complex64; trans N, T or C */
coral_status_t coral_ctrmv(coral_handle_t h, int uplo, int trans, int diag, size_t n,
                           const float* matrix, size_t lda, float* x, size_t incx);
/* ztrmv.rs -- interleaved complex128; trans N, T or C */
coral_status_t coral_ztrmv(coral_handle_t h, int uplo, int trans, int diag, size_t n,
                           const double* matrix, size_t lda, double* x, size_t incx);
/* dtrsv.rs -- double; ConjugateTranspose == Transpose */
coral_status_t coral_dtrsv(coral_handle_t h, int uplo, int trans, int diag, size_t n,
                           const double* matrix, size_t lda, double* x, size_t incx);
/* ctrsv.rs -- interleaved complex64; trans N, T or C */
coral_status_t coral_ctrsv(coral_handle_t h, int uplo, int trans, int diag, size_t n,
                           const float* matrix, size_t lda, float* x, size_t incx);
/* ztrsv.rs -- interleaved complex128; trans N, T or C */
coral_status_t coral_ztrsv(coral_handle_t h, int uplo, int trans, int diag, size_t n,
                           const double* matrix, size_t lda, double* x, size_t incx);
/* strsv.rs:60-74 */
coral_status_t coral_strsv(coral_handle_t h, int uplo, int trans, int diag, size_t n,
                           const float* matrix, size_t lda, float* x, size_t incx);
/* strmv.rs:59-73 */
coral_status_t coral_strmv(coral_handle_t h, int uplo, int trans, int diag, size_t n,
                           const float* matrix, size_t lda, float* x, size_t incx);
/* sger.rs:68-78 */
coral_status_t coral_sger(coral_handle_t h, size_t n_rows, size_t n_cols, float alpha,
                          const float* x, size_t incx, const float* y, size_t incy,
                          float* matrix, size_t lda);
/* ssyr.rs:63-71 */
coral_status_t coral_ssyr(coral_handle_t h, int uplo, size_t n, float alpha,
                          const float* x, size_t incx, float* matrix, size_t lda);
/* ssyr2.rs:59-69 */
coral_status_t coral_ssyr2(coral_handle_t h, int uplo, size_t n, float alpha,
                           const float* x, size_t incx, const float* y, size_t incy,
                           float* matrix, size_t lda);
/* dger.rs -- A += alpha x y^T in double */
coral_status_t coral_dger(coral_handle_t h, size_t n_rows, size_t n_cols, double alpha,
                          const double* x, size_t incx, const double* y, size_t incy,
                          double* matrix, size_t lda);
/* cgeru.rs / cgerc.rs -- A += alpha x y^T / alpha x y^H, interleaved complex64 */
coral_status_t coral_cgeru(coral_handle_t h, size_t n_rows, size_t n_cols, const float alpha[2],
                           const float* x, size_t incx, const float* y, size_t incy,
                           float* matrix, size_t lda);
coral_status_t coral_cgerc(coral_handle_t h, size_t n_rows, size_t n_cols, const float alpha[2],
                           const float* x, size_t incx, const float* y, size_t incy,
                           float* matrix, size_t lda);
/* zgeru.rs / zgerc.rs -- interleaved complex128 */
coral_status_t coral_zgeru(coral_handle_t h, size_t n_rows, size_t n_cols, const double alpha[2],
                           const double* x, size_t incx, const double* y, size_t incy,
                           double* matrix, size_t lda);
coral_status_t coral_zgerc(coral_handle_t h, size_t n_rows, size_t n_cols, const double alpha[2],
                           const double* x, size_t incx, const double* y, size_t incy,
                           double* matrix, size_t lda);
/* dsyr.rs / dsyr2.rs -- double */
coral_status_t coral_dsyr(coral_handle_t h, int uplo, size_t n, double alpha,
                          const double* x, size_t incx, double* matrix, size_t lda);
coral_status_t coral_dsyr2(coral_handle_t h, int uplo, size_t n, double alpha,
                           const double* x, size_t incx, const double* y, size_t incy,
                           double* matrix, size_t lda);
/* cher.rs / zher.rs -- A += alpha x x^H, real alpha; diagonal stored real */
coral_status_t coral_cher(coral_handle_t h, int uplo, size_t n, float alpha,
                          const float* x, size_t incx, float* matrix, size_t lda);
coral_status_t coral_zher(coral_handle_t h, int uplo, size_t n, double alpha,
                          const double* x, size_t incx, double* matrix, size_t lda);
/* cher2.rs / zher2.rs -- A += alpha x y^H + conj(alpha) y x^H */
coral_status_t coral_cher2(coral_handle_t h, int uplo, size_t n, const float alpha[2],
                           const float* x, size_t incx, const float* y, size_t incy,
                           float* matrix, size_t lda);
coral_status_t coral_zher2(coral_handle_t h, int uplo, size_t n, const double alpha[2],
                           const double* x, size_t incx, const double* y, size_t incy,
                           double* matrix, size_t lda);

/* ---- level 3 (coral-aarch64/src/level3) --------------------------------- */
/* sgemm.rs:106-130; arithmetic per coral_set_gemm_mode (NATIVE or SPLIT_BF16X3/X6) */
coral_status_t coral_sgemm(coral_handle_t h, int op_a, int op_b, size_t m, size_t n,
                           size_t k, float alpha, const float* a, size_t lda,
                           const float* b, size_t ldb, float beta, float* c,
                           size_t ldc);
/* dgemm.rs:107; arithmetic per coral_set_gemm_mode (NATIVE or OZAKI_INT8) */
coral_status_t coral_dgemm(coral_handle_t h, int op_a, int op_b, size_t m, size_t n,
                           size_t k, double alpha, const double* a, size_t lda,
                           const double* b, size_t ldb, double beta, double* c,
                           size_t ldc);
/* cgemm.rs:127-157 -- op in {N, T, C}; interleaved complex64 */
coral_status_t coral_cgemm(coral_handle_t h, int op_a, int op_b, size_t m, size_t n,
                           size_t k, const float alpha[2], const float* a, size_t lda,
                           const float* b, size_t ldb, const float beta[2], float* c,
                           size_t ldc);
/* zgemm.rs:123 -- op in {N, T, C}; interleaved complex128 */
coral_status_t coral_zgemm(coral_handle_t h, int op_a, int op_b, size_t m, size_t n,
                           size_t k, const double alpha[2], const double* a, size_t lda,
                           const double* b, size_t ldb, const double beta[2], double* c,
                           size_t ldc);

/* ---- batched / grouped (no reference counterpart) ----------------------- */
/* One instance of a grouped SGEMM: the arguments of coral_sgemm.  `a`, `b`
 * are float or bf16 (per the call's input type), `c` is float. */
typedef struct coral_sgemm_problem {
  int32_t op_a, op_b, m, n, k;
  float alpha, beta;
  int32_t reserved;
  const void* a;
  const void* b;
  float* c;
  int64_t lda, ldb, ldc;
} coral_sgemm_problem_t;
enum { CORAL_INPUT_F32 = 0, CORAL_INPUT_BF16 = 1 };
/* Computes every instance of `problems` (an array of `count` descriptors in
 * DEVICE memory) with coral_sgemm's semantics; bf16 inputs accumulate in
 * fp32.  A fixed number of kernels, no host work per instance: capturable in
 * a CUDA graph once a first uncaptured call has sized the handle's scratch.
 * bf16 inputs, and fp32 inputs when the handle's GEMM mode is
 * CORAL_GEMM_SPLIT_BF16X3, run on the tensor cores (fp32 as split-BF16x3);
 * fp32 inputs in the other modes run on FP32 FMA tiles.  On the tensor-core
 * path each instance's N tile width comes from the handle's grouped policy
 * (coral_set_grouped_config), unless its `reserved` field is 64, 128 or 256. */
coral_status_t coral_sgemm_grouped(coral_handle_t h, int input_type, size_t count,
                                   const coral_sgemm_problem_t* problems);
/* Tensor-core grouped GEMM tile widths (64, 128 or 256) for the instance
 * classes n <= 64, n <= 128, n <= 256, n > 256; NULL restores the default
 * {64, 128, 128, 256}. */
coral_status_t coral_set_grouped_config(coral_handle_t h, const int tile_n[4]);
coral_status_t coral_get_grouped_config(coral_handle_t h, int tile_n[4]);
/* Exhaustive tuning of that policy on one batch (descriptors in DEVICE
 * memory): all 36 assignments (class 0 and 1 in {64, 128}, class 2 and 3 in
 * {64, 128, 256}; class 0 varies slowest) run once untimed and `reps` times
 * between CUDA events; per-candidate milliseconds go to ms_out[36], the
 * fastest index to `best` and its widths to tile_n, and that policy is
 * installed on the handle.  fp32 inputs are tuned in split-BF16x3 mode.  The
 * instances' C is overwritten. */
coral_status_t coral_autotune_sgemm_grouped(coral_handle_t h, int input_type, size_t count,
                                            const coral_sgemm_problem_t* problems, int reps,
                                            float* ms_out, int* best, int tile_n[4]);
/* One instance of a batched STRSV: the arguments of coral_strsv. */
typedef struct coral_strsv_problem {
  int32_t uplo, trans, diag, n;
  const float* a;
  float* x;
  int64_t lda, incx;
} coral_strsv_problem_t;
/* Solves every instance (descriptors in DEVICE memory) in one launch. */
coral_status_t coral_strsv_batched(coral_handle_t h, size_t count,
                                   const coral_strsv_problem_t* problems);

/* ---- configuration, autotuning and the learned selector ----------------- */
/* (No reference counterpart.)  Split-BF16 GEMM configuration: N tile width
 * (128 or 256) and split-K factor (1..64); 0 leaves the choice to the
 * selector (when set) or to the default rule. */
coral_status_t coral_set_gemm_config(coral_handle_t h, int tile_n, int split_k);
/* Same, with the tile height: tile_m 128 runs one CTA per 128 x tile_n tile;
 * tile_m 256 (with tile_n 256) runs a cluster of two CTAs per 256 x 256 tile,
 * whose tensor-core products read each CTA's half of A and of B
 * (tcgen05 cta_group::2).  All zero leaves the choice to the policy. */
coral_status_t coral_set_gemm_tile(coral_handle_t h, int tile_m, int tile_n, int split_k);
/* The tile a split-BF16 SGEMM of this shape would use now. */
coral_status_t coral_get_gemm_tile(coral_handle_t h, int products, int op_a, int op_b, size_t m,
                                   size_t n, size_t k, int* tile_m, int* tile_n, int* split_k);
/* M-tiles per raster group of the CTA-pair tiles (1..64; 0 restores 8). */
coral_status_t coral_set_pair_raster(coral_handle_t h, int group);
/* The configuration a split-BF16 SGEMM of this shape would use now. */
coral_status_t coral_get_gemm_config(coral_handle_t h, int products, int op_a, int op_b, size_t m,
                                     size_t n, size_t k, int* tile_n, int* split_k);
/* Features the selector network sees for (shape, configuration); 13 floats.
 * Needs no device.  tile_n and split_k must be positive; sides past INT_MAX
 * return CORAL_ERR_NOT_SUPPORTED (as the GEMM entry points do). */
coral_status_t coral_selector_features(int products, int op_a, int op_b, size_t m, size_t n,
                                       size_t k, int tile_n, int split_k, float* out);
/* Exhaustive autotuning of one split-BF16 SGEMM shape on the given device
 * buffers: times every (tile_n, split_k) candidate `reps` times (after one
 * warm-up) with CUDA events; writes per-candidate milliseconds in the order
 * tile_n in {256, 128} x split_k in {1, 2, 4, 8, 16} (10 values, products 6:
 * only the 5 tile_n = 128 values) and the index of the fastest.  C is
 * overwritten.  Restores the handle's previous configuration. */
coral_status_t coral_autotune_sgemm(coral_handle_t h, int products, int op_a, int op_b, size_t m,
                                    size_t n, size_t k, const float* a, size_t lda, const float* b,
                                    size_t ldb, float* c, size_t ldc, int reps, float* ms_out,
                                    int* best);

/* Exhaustive autotuning over tile shapes too: the configurations
 * (tile_m x tile_n) in {256 x 256 (a CTA pair, cta_group::2), 128 x 256,
 * 128 x 128} x split_k in {1, 2, 4, 8, 16}, in that order (15 values;
 * products 6: 10, without 128 x 256).  `capacity` is the length of ms_out;
 * the number written goes to *count and the fastest index to *best.  C is
 * overwritten; the handle's configuration is restored. */
coral_status_t coral_autotune_sgemm_tiles(coral_handle_t h, int products, int op_a, int op_b, size_t m,
                                          size_t n, size_t k, const float* a, size_t lda, const float* b,
                                          size_t ldb, float* c, size_t ldc, int reps, float* ms_out,
                                          int capacity, int* count, int* best);
/* Selector features of (shape, tile_m x tile_n, split_k); 13 floats.  Same
 * checks, and tile_m must be 128 or 256. */
coral_status_t coral_selector_features_tile(int products, int op_a, int op_b, size_t m, size_t n,
                                            size_t k, int tile_m, int tile_n, int split_k, float* out);

/* A small MLP (in -> hidden -> hidden -> out, ReLU) trained and evaluated by
 * the library's own kernels; used as the configuration selector (in = 13,
 * out = 1: predicted log milliseconds). */
typedef struct coral_mlp_s* coral_mlp_t;
coral_status_t coral_mlp_create(coral_handle_t h, int in_dim, int hidden, int out_dim,
                                uint64_t seed, coral_mlp_t* mlp);
coral_status_t coral_mlp_destroy(coral_mlp_t mlp);
size_t coral_mlp_param_count(coral_mlp_t mlp);
coral_status_t coral_mlp_get_params(coral_mlp_t mlp, float* host, size_t count);
coral_status_t coral_mlp_set_params(coral_mlp_t mlp, const float* host, size_t count);
/* x: DEVICE [batch][in], y: DEVICE [batch][out]. */
coral_status_t coral_mlp_forward(coral_mlp_t mlp, const float* x, int batch, float* y);
/* Gradient of mean((y - target)^2) w.r.t. the packed parameters into the
 * DEVICE array `grads` (may be NULL); loss to host memory (may be NULL). */
coral_status_t coral_mlp_gradients(coral_mlp_t mlp, const float* x, const float* target, int batch,
                                   float* grads, float* loss);
/* One Adam step (beta1 0.9, beta2 0.999) on a batch; loss to host (may be NULL). */
coral_status_t coral_mlp_train_step(coral_mlp_t mlp, const float* x, const float* target, int batch,
                                    float lr, float* loss);
/* Features (13 floats) of a uniform batch of `batch` instances of one shape
 * in the tensor-core grouped GEMM under N tile width tile_n, for training a
 * network that predicts the batch's log time. */
coral_status_t coral_grouped_features(int input_type, int op_a, int op_b, size_t m, size_t n, size_t k,
                                      size_t batch, int tile_n, float* out);
/* Learned grouped tile-width policy: for each instance class present in
 * `problems_host` (a HOST copy of the descriptors), the network (trained on
 * coral_grouped_features) scores the allowed widths for the class's median
 * shape and instance count; the argmin per class is installed on the handle
 * and returned in tile_n.  Synchronises with the handle's stream. */
coral_status_t coral_select_grouped_config(coral_handle_t h, coral_mlp_t mlp, int input_type, size_t count,
                                           const coral_sgemm_problem_t* problems_host, int tile_n[4]);
/* Attach (or, with NULL, detach) a trained selector to a handle.  Decisions
 * are cached per shape; the first call for a shape waits for one forward
 * pass, so make it outside stream capture. */
coral_status_t coral_set_selector(coral_handle_t h, coral_mlp_t mlp);

/* ---- allocation-free split-BF16x3 SGEMM --------------------------------- */
/* No counterpart in the reference (CORAL allocates its packing buffers on
 * every call).  Same arguments and result as coral_sgemm in
 * CORAL_GEMM_SPLIT_BF16X3 mode, with a cudaStream_t (NULL = legacy default
 * stream) in place of the handle, for callers that must not have device
 * memory allocated behind their back: a process that reserves nearly all of
 * HBM up front and sub-allocates it itself, a latency-critical loop that
 * cannot take cudaMalloc's implicit synchronisation, or a deployment that
 * forbids device allocation after start-up.  It calls no cudaMalloc or
 * cudaFree: the bf16 operand pieces live in a fixed 32 MiB device array that
 * every GPU loading this library holds until the process exits.
 *   - Sizes whose pieces need more than 32 MiB, i.e. 4 * (m + n) * kp bytes
 *     with kp = k rounded up to a multiple of 8 (about m = n = k = 2048), are
 *     rejected with CORAL_ERR_NOT_SUPPORTED before any work is enqueued.
 *   - The first call on a device looks up the array's device address and sets
 *     the kernel's shared-memory limit for that device; make that first call
 *     before any stream capture on the device.
 *   - All calls share the one array: calls whose work can overlap on the GPU
 *     (different streams, or other host threads) race on it and must be
 *     serialised by the caller.
 *   - alpha == 0 or k == 0 only scales C by beta and uses no scratch, so it
 *     is accepted at any size; m == 0 or n == 0 returns at once.
 *   - The kernel's bounded waits cannot report through the return value (the
 *     call returns before the kernel runs): a give-up sets a fixed device
 *     status word, read by coral_sgemm_bf16x3_noalloc_status.
 * Device pointers; asynchronous on `stream`. */
coral_status_t coral_sgemm_bf16x3_noalloc(void* stream, int op_a, int op_b, size_t m, size_t n,
                                          size_t k, float alpha, const float* a, size_t lda,
                                          const float* b, size_t ldb, float beta, float* c,
                                          size_t ldc);
/* Waits for `stream`, then reads and clears the current device's status word
 * of coral_sgemm_bf16x3_noalloc: CORAL_ERR_TIMEOUT when a call since the last
 * query gave up a bounded wait (its C may be incomplete), else CORAL_OK.
 * Allocates nothing. */
coral_status_t coral_sgemm_bf16x3_noalloc_status(void* stream);

/* ---- host-slice drop-ins: the reference's exact argument lists ---------- */
/* Pointers are HOST memory.  Return value as above; scalar-returning routines
 * write through the trailing out-pointer.  Thread-safe: each host thread gets
 * its own internal handle. */
coral_status_t coral_host_sgemm(int op_a, int op_b, size_t m, size_t n, size_t k,
                                float alpha, const float* a, size_t lda, const float* b,
                                size_t ldb, float beta, float* c, size_t ldc);
coral_status_t coral_host_sgemv(int trans, size_t n_rows, size_t n_cols, float alpha,
                                const float* matrix, size_t lda, const float* x,
                                size_t incx, float beta, float* y, size_t incy);
coral_status_t coral_host_sdot(size_t n, const float* x, size_t incx, const float* y,
                               size_t incy, float* result);
coral_status_t coral_host_saxpy(size_t n, float alpha, const float* x, size_t incx,
                                float* y, size_t incy);
coral_status_t coral_host_isamax(size_t n, const float* x, size_t incx, size_t* index);
coral_status_t coral_host_strsv(int uplo, int trans, int diag, size_t n,
                                const float* matrix, size_t lda, float* x, size_t incx);
/* level2/ssymv.rs:99-110 */
coral_status_t coral_host_ssymv(int uplo, size_t n, float alpha, const float* matrix, size_t lda,
                                const float* x, size_t incx, float beta, float* y, size_t incy);
/* level2/chemv.rs:96-107 -- interleaved complex64, complex scalars [re, im] */
coral_status_t coral_host_chemv(int uplo, size_t n, const float alpha[2], const float* matrix,
                                size_t lda, const float* x, size_t incx, const float beta[2],
                                float* y, size_t incy);
/* level2/strmv.rs:59-73 */
coral_status_t coral_host_strmv(int uplo, int trans, int diag, size_t n, const float* matrix,
                                size_t lda, float* x, size_t incx);
/* level2/sger.rs:68-78 */
coral_status_t coral_host_sger(size_t n_rows, size_t n_cols, float alpha, const float* x,
                               size_t incx, const float* y, size_t incy, float* matrix, size_t lda);
/* level2/ssyr.rs:63-71 */
coral_status_t coral_host_ssyr(int uplo, size_t n, float alpha, const float* x, size_t incx,
                               float* matrix, size_t lda);
/* level2/ssyr2.rs:59-69 */
coral_status_t coral_host_ssyr2(int uplo, size_t n, float alpha, const float* x, size_t incx,
                                const float* y, size_t incy, float* matrix, size_t lda);
/* level1/snrm2.rs:45-149 -- result through the out-pointer */
coral_status_t coral_host_snrm2(size_t n, const float* x, size_t incx, float* result);
/* level1/scopy.rs:28-58 */
coral_status_t coral_host_scopy(size_t n, const float* x, size_t incx, float* y, size_t incy);
/* level1/sswap.rs:35-118 */
coral_status_t coral_host_sswap(size_t n, float* x, size_t incx, float* y, size_t incy);
/* level1/sscal.rs:30-66 */
coral_status_t coral_host_sscal(size_t n, float alpha, float* x, size_t incx);
/* level3/dgemm.rs:107 -- arithmetic per coral_host_set_gemm_mode */
coral_status_t coral_host_dgemm(int op_a, int op_b, size_t m, size_t n, size_t k, double alpha,
                                const double* a, size_t lda, const double* b, size_t ldb,
                                double beta, double* c, size_t ldc);
/* level3/cgemm.rs:127-157 -- interleaved complex64 */
coral_status_t coral_host_cgemm(int op_a, int op_b, size_t m, size_t n, size_t k,
                                const float alpha[2], const float* a, size_t lda, const float* b,
                                size_t ldb, const float beta[2], float* c, size_t ldc);
/* level3/zgemm.rs:123 -- interleaved complex128 */
coral_status_t coral_host_zgemm(int op_a, int op_b, size_t m, size_t n, size_t k,
                                const double alpha[2], const double* a, size_t lda,
                                const double* b, size_t ldb, const double beta[2], double* c,
                                size_t ldc);
/* Select the GEMM arithmetic of this thread's internal handle. */
coral_status_t coral_host_set_gemm_mode(int mode);

#ifdef __cplusplus
}
#endif
#endif /* CORAL_B200_H */
