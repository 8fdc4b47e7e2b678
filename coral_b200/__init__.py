"""coral_b200 -- CORAL's column-major BLAS API on one NVIDIA B200.

Hand-written sm_100a CUDA kernels behind a C ABI (include/coral_b200.h,
libcoral_b200.so); this package is the Python mirror of the reference's
routine signatures (``coral_b200.blas``) plus the ctypes binding
(``coral_b200._lib``).
"""
from .blas import (  # noqa: F401
    CoralDiagonal, CoralError, CoralTranspose, CoralTriangular, GemmMode, Handle, cgemm,
    chemv, dgemm, gemm_mode, handle, isamax, saxpy, scopy, sdot, set_gemm_mode, sgemm, sgemv,
    sger, snrm2, sscal, sswap, ssymv, ssyr, ssyr2, strmv, strsv, zgemm, sgemm_grouped,
    strsv_batched, sgemm_problem_dtype, strsv_problem_dtype, dgemv, cgemv, zgemv,
    dsymv, zhemv, dtrmv, ctrmv, ztrmv, dger, cgeru, cgerc, zgeru, zgerc, dsyr, dsyr2, cher, zher,
    cher2, zher2, dtrsv, ctrsv, ztrsv,
    ddot, cdotu, cdotc, zdotu, zdotc, sasum, dasum, scasum, dzasum, dnrm2, scnrm2, dznrm2, idamax,
    icamax, izamax, daxpy, caxpy, zaxpy, dscal, cscal, zscal, csscal, zdscal, dcopy, ccopy, zcopy,
    dswap, cswap, zswap, srot, drot, csrot, zdrot, srotm, drotm, srotg, drotg, srotmg, drotmg,
    saxpyf, daxpyf, caxpyf, zaxpyf, sdotf, ddotf, cdotuf, cdotcf, zdotuf, zdotcf,
    set_grouped_config, grouped_config, autotune_sgemm_grouped,
)

__all__ = [
    "CoralDiagonal", "CoralError", "CoralTranspose", "CoralTriangular", "GemmMode", "Handle",
    "cgemm", "chemv", "dgemm", "gemm_mode", "handle", "isamax", "saxpy", "scopy", "sdot",
    "set_gemm_mode", "sgemm", "sgemv", "sger", "snrm2", "sscal", "sswap", "ssymv", "ssyr",
    "ssyr2", "strmv", "strsv", "zgemm", "sgemm_grouped", "strsv_batched", "sgemm_problem_dtype",
    "strsv_problem_dtype", "dgemv", "cgemv", "zgemv",
    "dsymv", "zhemv", "dtrmv", "ctrmv", "ztrmv", "dger", "cgeru", "cgerc", "zgeru", "zgerc", "dsyr",
    "dsyr2", "cher", "zher", "cher2", "zher2", "dtrsv", "ctrsv", "ztrsv",
    "ddot", "cdotu", "cdotc", "zdotu", "zdotc", "sasum", "dasum", "scasum", "dzasum", "dnrm2", "scnrm2", "dznrm2",
    "idamax", "icamax", "izamax", "daxpy", "caxpy", "zaxpy", "dscal", "cscal", "zscal", "csscal", "zdscal", "dcopy",
    "ccopy", "zcopy", "dswap", "cswap", "zswap", "srot", "drot", "csrot", "zdrot", "srotm", "drotm", "srotg", "drotg", "srotmg", "drotmg",
    "saxpyf", "daxpyf", "caxpyf", "zaxpyf", "sdotf", "ddotf", "cdotuf", "cdotcf", "zdotuf", "zdotcf",
    "set_grouped_config", "grouped_config", "autotune_sgemm_grouped",
]
