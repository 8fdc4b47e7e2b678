"""ctypes binding of libcoral_b200.so (the C ABI declared in include/coral_b200.h).

The library is loaded from the package directory, where
``python -m coral_b200.build`` (or ``__graft_entry__.build()``) puts it.  There
is no fallback: if the library is missing or cannot be loaded, every call
raises.
"""
from __future__ import annotations

import ctypes as C
import os
import re

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "libcoral_b200.so")
HEADER = os.path.join(os.path.dirname(PKG), "include", "coral_b200.h")

_lib = None

_sz = C.c_size_t
_i = C.c_int
_f = C.c_float
_d = C.c_double
_vp = C.c_void_p
_h = C.c_void_p
_st = C.c_int

# name -> argtypes (restype is coral_status_t = int unless listed in _RESTYPE)
SIGNATURES = {
    "coral_create": [C.POINTER(_h)],
    "coral_destroy": [_h],
    "coral_set_stream": [_h, _vp],
    "coral_get_stream": [_h, C.POINTER(_vp)],
    "coral_set_pointer_mode": [_h, _i],
    "coral_set_gemm_mode": [_h, _i],
    "coral_get_gemm_mode": [_h, C.POINTER(_i)],
    "coral_set_wait_limit": [_h, C.c_uint64],
    "coral_set_split_chunk": [_h, _i],
    "coral_set_complex_mapping": [_h, _i],
    "coral_set_strip_form": [_h, _i],
    "coral_sync": [_h],
    "coral_set_kernel_timing": [_h, _i],
    "coral_get_kernel_timing": [_h, C.POINTER(_d), C.POINTER(C.c_uint64)],
    "coral_last_bad_arg": [_h],
    "coral_status_string": [_st],
    "coral_last_cuda_error": [_h],
    "coral_abi_version": [],
    "coral_kernel_launches": [],
    "coral_sdot": [_h, _sz, _vp, _sz, _vp, _sz, _vp],
    "coral_saxpy": [_h, _sz, _f, _vp, _sz, _vp, _sz],
    "coral_snrm2": [_h, _sz, _vp, _sz, _vp],
    "coral_isamax": [_h, _sz, _vp, _sz, _vp],
    "coral_scopy": [_h, _sz, _vp, _sz, _vp, _sz],
    "coral_sswap": [_h, _sz, _vp, _sz, _vp, _sz],
    "coral_sscal": [_h, _sz, _f, _vp, _sz],
    "coral_ddot": [_h, _sz, _vp, _sz, _vp, _sz, _vp],
    "coral_cdotu": [_h, _sz, _vp, _sz, _vp, _sz, _vp],
    "coral_cdotc": [_h, _sz, _vp, _sz, _vp, _sz, _vp],
    "coral_zdotu": [_h, _sz, _vp, _sz, _vp, _sz, _vp],
    "coral_zdotc": [_h, _sz, _vp, _sz, _vp, _sz, _vp],
    "coral_sasum": [_h, _sz, _vp, _sz, _vp],
    "coral_dasum": [_h, _sz, _vp, _sz, _vp],
    "coral_scasum": [_h, _sz, _vp, _sz, _vp],
    "coral_dzasum": [_h, _sz, _vp, _sz, _vp],
    "coral_dnrm2": [_h, _sz, _vp, _sz, _vp],
    "coral_scnrm2": [_h, _sz, _vp, _sz, _vp],
    "coral_dznrm2": [_h, _sz, _vp, _sz, _vp],
    "coral_idamax": [_h, _sz, _vp, _sz, _vp],
    "coral_icamax": [_h, _sz, _vp, _sz, _vp],
    "coral_izamax": [_h, _sz, _vp, _sz, _vp],
    "coral_daxpy": [_h, _sz, _d, _vp, _sz, _vp, _sz],
    "coral_caxpy": [_h, _sz, _vp, _vp, _sz, _vp, _sz],
    "coral_zaxpy": [_h, _sz, _vp, _vp, _sz, _vp, _sz],
    "coral_dscal": [_h, _sz, _d, _vp, _sz],
    "coral_cscal": [_h, _sz, _vp, _vp, _sz],
    "coral_zscal": [_h, _sz, _vp, _vp, _sz],
    "coral_csscal": [_h, _sz, _f, _vp, _sz],
    "coral_zdscal": [_h, _sz, _d, _vp, _sz],
    "coral_dcopy": [_h, _sz, _vp, _sz, _vp, _sz],
    "coral_ccopy": [_h, _sz, _vp, _sz, _vp, _sz],
    "coral_zcopy": [_h, _sz, _vp, _sz, _vp, _sz],
    "coral_dswap": [_h, _sz, _vp, _sz, _vp, _sz],
    "coral_cswap": [_h, _sz, _vp, _sz, _vp, _sz],
    "coral_zswap": [_h, _sz, _vp, _sz, _vp, _sz],
    "coral_srot": [_h, _sz, _vp, _sz, _vp, _sz, _f, _f],
    "coral_drot": [_h, _sz, _vp, _sz, _vp, _sz, _d, _d],
    "coral_csrot": [_h, _sz, _vp, _sz, _vp, _sz, _f, _f],
    "coral_zdrot": [_h, _sz, _vp, _sz, _vp, _sz, _d, _d],
    "coral_srotm": [_h, _sz, _vp, _sz, _vp, _sz, _vp],
    "coral_drotm": [_h, _sz, _vp, _sz, _vp, _sz, _vp],
    "coral_srotg": [_h, _vp, _vp, _vp, _vp],
    "coral_drotg": [_h, _vp, _vp, _vp, _vp],
    "coral_srotmg": [_h, _vp, _vp, _vp, _f, _vp],
    "coral_drotmg": [_h, _vp, _vp, _vp, _d, _vp],
    "coral_saxpyf": [_h, _sz, _sz, _vp, _sz, _vp, _sz, _vp, _sz],
    "coral_daxpyf": [_h, _sz, _sz, _vp, _sz, _vp, _sz, _vp, _sz],
    "coral_caxpyf": [_h, _sz, _sz, _vp, _sz, _vp, _sz, _vp, _sz],
    "coral_zaxpyf": [_h, _sz, _sz, _vp, _sz, _vp, _sz, _vp, _sz],
    "coral_sdotf": [_h, _sz, _sz, _vp, _sz, _vp, _sz, _vp],
    "coral_ddotf": [_h, _sz, _sz, _vp, _sz, _vp, _sz, _vp],
    "coral_cdotuf": [_h, _sz, _sz, _vp, _sz, _vp, _sz, _vp],
    "coral_cdotcf": [_h, _sz, _sz, _vp, _sz, _vp, _sz, _vp],
    "coral_zdotuf": [_h, _sz, _sz, _vp, _sz, _vp, _sz, _vp],
    "coral_zdotcf": [_h, _sz, _sz, _vp, _sz, _vp, _sz, _vp],
    "coral_sgemv": [_h, _i, _sz, _sz, _f, _vp, _sz, _vp, _sz, _f, _vp, _sz],
    "coral_dgemv": [_h, _i, _sz, _sz, _d, _vp, _sz, _vp, _sz, _d, _vp, _sz],
    "coral_cgemv": [_h, _i, _sz, _sz, _vp, _vp, _sz, _vp, _sz, _vp, _vp, _sz],
    "coral_zgemv": [_h, _i, _sz, _sz, _vp, _vp, _sz, _vp, _sz, _vp, _vp, _sz],
    "coral_dsymv": [_h, _i, _sz, _d, _vp, _sz, _vp, _sz, _d, _vp, _sz],
    "coral_zhemv": [_h, _i, _sz, _vp, _vp, _sz, _vp, _sz, _vp, _vp, _sz],
    "coral_dtrmv": [_h, _i, _i, _i, _sz, _vp, _sz, _vp, _sz],
    "coral_ctrmv": [_h, _i, _i, _i, _sz, _vp, _sz, _vp, _sz],
    "coral_ztrmv": [_h, _i, _i, _i, _sz, _vp, _sz, _vp, _sz],
    "coral_dger": [_h, _sz, _sz, _d, _vp, _sz, _vp, _sz, _vp, _sz],
    "coral_cgeru": [_h, _sz, _sz, _vp, _vp, _sz, _vp, _sz, _vp, _sz],
    "coral_cgerc": [_h, _sz, _sz, _vp, _vp, _sz, _vp, _sz, _vp, _sz],
    "coral_zgeru": [_h, _sz, _sz, _vp, _vp, _sz, _vp, _sz, _vp, _sz],
    "coral_zgerc": [_h, _sz, _sz, _vp, _vp, _sz, _vp, _sz, _vp, _sz],
    "coral_dsyr": [_h, _i, _sz, _d, _vp, _sz, _vp, _sz],
    "coral_dsyr2": [_h, _i, _sz, _d, _vp, _sz, _vp, _sz, _vp, _sz],
    "coral_cher": [_h, _i, _sz, _f, _vp, _sz, _vp, _sz],
    "coral_zher": [_h, _i, _sz, _d, _vp, _sz, _vp, _sz],
    "coral_cher2": [_h, _i, _sz, _vp, _vp, _sz, _vp, _sz, _vp, _sz],
    "coral_zher2": [_h, _i, _sz, _vp, _vp, _sz, _vp, _sz, _vp, _sz],
    "coral_dtrsv": [_h, _i, _i, _i, _sz, _vp, _sz, _vp, _sz],
    "coral_ctrsv": [_h, _i, _i, _i, _sz, _vp, _sz, _vp, _sz],
    "coral_ztrsv": [_h, _i, _i, _i, _sz, _vp, _sz, _vp, _sz],
    "coral_ssymv": [_h, _i, _sz, _f, _vp, _sz, _vp, _sz, _f, _vp, _sz],
    "coral_chemv": [_h, _i, _sz, _vp, _vp, _sz, _vp, _sz, _vp, _vp, _sz],
    "coral_strsv": [_h, _i, _i, _i, _sz, _vp, _sz, _vp, _sz],
    "coral_strmv": [_h, _i, _i, _i, _sz, _vp, _sz, _vp, _sz],
    "coral_sger": [_h, _sz, _sz, _f, _vp, _sz, _vp, _sz, _vp, _sz],
    "coral_ssyr": [_h, _i, _sz, _f, _vp, _sz, _vp, _sz],
    "coral_ssyr2": [_h, _i, _sz, _f, _vp, _sz, _vp, _sz, _vp, _sz],
    "coral_sgemm": [_h, _i, _i, _sz, _sz, _sz, _f, _vp, _sz, _vp, _sz, _f, _vp, _sz],
    "coral_dgemm": [_h, _i, _i, _sz, _sz, _sz, _d, _vp, _sz, _vp, _sz, _d, _vp, _sz],
    "coral_cgemm": [_h, _i, _i, _sz, _sz, _sz, _vp, _vp, _sz, _vp, _sz, _vp, _vp, _sz],
    "coral_zgemm": [_h, _i, _i, _sz, _sz, _sz, _vp, _vp, _sz, _vp, _sz, _vp, _vp, _sz],
    "coral_sgemm_grouped": [_h, _i, _sz, _vp],
    "coral_set_grouped_config": [_h, _vp],
    "coral_get_grouped_config": [_h, _vp],
    "coral_autotune_sgemm_grouped": [_h, _i, _sz, _vp, _i, _vp, C.POINTER(_i), _vp],
    "coral_set_gemm_config": [_h, _i, _i],
    "coral_set_gemm_tile": [_h, _i, _i, _i],
    "coral_get_gemm_tile": [_h, _i, _i, _i, _sz, _sz, _sz, C.POINTER(_i), C.POINTER(_i), C.POINTER(_i)],
    "coral_set_pair_raster": [_h, _i],
    "coral_autotune_sgemm_tiles": [_h, _i, _i, _i, _sz, _sz, _sz, _vp, _sz, _vp, _sz, _vp, _sz, _i,
                                   C.POINTER(_f), _i, C.POINTER(_i), C.POINTER(_i)],
    "coral_selector_features_tile": [_i, _i, _i, _sz, _sz, _sz, _i, _i, _i, C.POINTER(_f)],
    "coral_get_gemm_config": [_h, _i, _i, _i, _sz, _sz, _sz, C.POINTER(_i), C.POINTER(_i)],
    "coral_selector_features": [_i, _i, _i, _sz, _sz, _sz, _i, _i, C.POINTER(_f)],
    "coral_autotune_sgemm": [_h, _i, _i, _i, _sz, _sz, _sz, _vp, _sz, _vp, _sz, _vp, _sz, _i,
                             C.POINTER(_f), C.POINTER(_i)],
    "coral_mlp_create": [_h, _i, _i, _i, C.c_uint64, C.POINTER(_vp)],
    "coral_mlp_destroy": [_vp],
    "coral_mlp_param_count": [_vp],
    "coral_mlp_get_params": [_vp, C.POINTER(_f), _sz],
    "coral_mlp_set_params": [_vp, C.POINTER(_f), _sz],
    "coral_mlp_forward": [_vp, _vp, _i, _vp],
    "coral_mlp_gradients": [_vp, _vp, _vp, _i, _vp, C.POINTER(_f)],
    "coral_mlp_train_step": [_vp, _vp, _vp, _i, _f, C.POINTER(_f)],
    "coral_set_selector": [_h, _vp],
    "coral_grouped_features": [_i, _i, _i, _sz, _sz, _sz, _sz, _i, C.POINTER(_f)],
    "coral_select_grouped_config": [_h, _vp, _i, _sz, _vp, _vp],
    "coral_strsv_batched": [_h, _sz, _vp],
    "coral_sgemm_bf16x3_noalloc": [_vp, _i, _i, _sz, _sz, _sz, _f, _vp, _sz, _vp, _sz, _f, _vp, _sz],
    "coral_sgemm_bf16x3_noalloc_status": [_vp],
    "coral_host_sgemm": [_i, _i, _sz, _sz, _sz, _f, _vp, _sz, _vp, _sz, _f, _vp, _sz],
    "coral_host_sgemv": [_i, _sz, _sz, _f, _vp, _sz, _vp, _sz, _f, _vp, _sz],
    "coral_host_sdot": [_sz, _vp, _sz, _vp, _sz, _vp],
    "coral_host_saxpy": [_sz, _f, _vp, _sz, _vp, _sz],
    "coral_host_isamax": [_sz, _vp, _sz, _vp],
    "coral_host_strsv": [_i, _i, _i, _sz, _vp, _sz, _vp, _sz],
    "coral_host_set_gemm_mode": [_i],
    "coral_host_ssymv": [_i, _sz, _f, _vp, _sz, _vp, _sz, _f, _vp, _sz],
    "coral_host_chemv": [_i, _sz, _vp, _vp, _sz, _vp, _sz, _vp, _vp, _sz],
    "coral_host_strmv": [_i, _i, _i, _sz, _vp, _sz, _vp, _sz],
    "coral_host_sger": [_sz, _sz, _f, _vp, _sz, _vp, _sz, _vp, _sz],
    "coral_host_ssyr": [_i, _sz, _f, _vp, _sz, _vp, _sz],
    "coral_host_ssyr2": [_i, _sz, _f, _vp, _sz, _vp, _sz, _vp, _sz],
    "coral_host_snrm2": [_sz, _vp, _sz, _vp],
    "coral_host_scopy": [_sz, _vp, _sz, _vp, _sz],
    "coral_host_sswap": [_sz, _vp, _sz, _vp, _sz],
    "coral_host_sscal": [_sz, _f, _vp, _sz],
    "coral_host_dgemm": [_i, _i, _sz, _sz, _sz, _d, _vp, _sz, _vp, _sz, _d, _vp, _sz],
    "coral_host_cgemm": [_i, _i, _sz, _sz, _sz, _vp, _vp, _sz, _vp, _sz, _vp, _vp, _sz],
    "coral_host_zgemm": [_i, _i, _sz, _sz, _sz, _vp, _vp, _sz, _vp, _sz, _vp, _vp, _sz],
}

_RESTYPE = {
    "coral_last_bad_arg": C.c_int,
    "coral_status_string": C.c_char_p,
    "coral_last_cuda_error": C.c_char_p,
    "coral_abi_version": C.c_int,
    "coral_kernel_launches": C.c_uint64,
    "coral_mlp_param_count": C.c_size_t,
}


def header_symbols(path: str = HEADER) -> list[str]:
    """Names of every function declared in include/coral_b200.h."""
    text = open(path).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(coral_\w+)\s*\(", text)))


def load() -> C.CDLL:
    """Loads the library (once) and declares every signature."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(
            f"{LIB_PATH} is missing: build it with `python -m coral_b200.build` "
            "(there is no CPU fallback)")
    lib = C.CDLL(LIB_PATH)
    for name, args in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = _RESTYPE.get(name, _st)
    _lib = lib
    return lib
