"""ctypes binding of libpofd_b200.so (the C ABI in include/pofd_b200.h).

The library is built in-tree (pofd_affine_b200/_lib/libpofd_b200.so) by
``python -m pofd_affine_b200.build``.  There is no CPU fallback: if the
library is missing or cannot be loaded, every use raises.
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIBPATH = os.path.join(HERE, "_lib", "libpofd_b200.so")
HEADER = os.path.join(HERE, "..", "include", "pofd_b200.h")
SUPPORT_LIBPATH = os.path.join(HERE, "_lib", "libpofd_b200_support.so")
SUPPORT_HEADER = os.path.join(HERE, "..", "include", "pofd_b200_support.h")

_dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_fp = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")
_ip = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_up = np.ctypeslib.ndpointer(dtype=np.uint32, flags="C_CONTIGUOUS")
V, I, U, D, S = C.c_void_p, C.c_int, C.c_uint, C.c_double, C.c_size_t
PV = C.POINTER(C.c_void_p)

# name -> (restype, argtypes); pointer-typed outputs that may be NULL are
# declared as c_void_p.
SIGNATURES = {
    "pofd_last_error": (C.c_char_p, []),
    "pofd_version": (C.c_char_p, []),
    "pofd_ctx_create": (I, [I, PV]),
    "pofd_ctx_destroy": (I, [V]),
    "pofd_ctx_stream": (I, [V, PV]),
    "pofd_ctx_synchronize": (I, [V]),
    "pofd_fits_read_data": (I, [C.c_char_p, I, I, V, S, C.POINTER(S)]),
    "pofd_fits_read_beam": (I, [C.c_char_p, V, S, C.POINTER(S), C.POINTER(S),
                                C.POINTER(D)]),
    "pofd_fits_read_data2": (I, [C.c_char_p, C.c_char_p, I, I, V, V, S,
                                 C.POINTER(S)]),
    "pofd_ensemble_get_counter": (I, [V, C.POINTER(C.c_ulonglong),
                                      C.POINTER(C.c_ulonglong)]),
    "pofd_ensemble_set_counter": (I, [V, C.c_ulonglong]),
    "pofd_ensemble_set_naccept": (I, [V, _up]),
    "pofd_beam1_create": (I, [_dp, S, D, D, U, PV]),
    "pofd_beam1_destroy": (I, [V]),
    "pofd_beam1_info": (I, [V, _dp]),
    "pofd_beam1_terms": (I, [V, I, C.POINTER(S), V, V]),
    "pofd_pdfactory1_create": (I, [V, U, PV]),
    "pofd_pdfactory1_destroy": (I, [V]),
    "pofd_pdfactory1_initpd": (I, [V, U, D, D, U, _dp, _fp, V]),
    "pofd_pdfactory1_getpd": (I, [V, D, I, _dp, C.POINTER(D),
                                  C.POINTER(D)]),
    "pofd_pdfactory1_get_r": (I, [V, _dp]),
    "pofd_like1_create": (I, [V, U, _dp, U, U, I, U, PV]),
    "pofd_like1_destroy": (I, [V]),
    "pofd_like1_add_beamset": (I, [V, V, D]),
    "pofd_like1_add_dataset": (I, [V, I, _dp, S, I, D, D]),
    "pofd_like1_add_dataset_device": (I, [V, I, V, S, I, D, D]),
    "pofd_data_bin_device": (I, [V, S, I, U, V, _dp, V]),
    "pofd_data2_bin_device": (I, [V, V, S, I, U, U, V, _dp, V]),
    "pofd_like2_add_dataset_device": (I, [V, I, V, V, S, I, D, D, D]),
    "pofd_like1_set_rranges": (I, [V, _fp, U]),
    "pofd_like1_get_rrange": (I, [V, I, _dp]),
    "pofd_like1_get_r": (I, [V, I, _fp, U, _dp]),
    "pofd_like1_dataset_info": (I, [V, I, I, _dp, V]),
    "pofd_like1_reserve": (I, [V, U]),
    "pofd_like1_loglike": (I, [V, _fp, U, C.POINTER(D), C.POINTER(I)]),
    # the batch calls take raw pointers: the arrays are made contiguous and
    # typed by the caller, and ndpointer's checks cost microseconds per call
    "pofd_like1_eval_batch": (I, [V, U, V, U, V, V]),
    "pofd_like1_eval_batch_device": (I, [V, U, V, U, V, V, V]),
    "pofd_like1_pd": (I, [V, I, I, _fp, U, I, _dp, V]),
    "pofd_like1_rnodes": (I, [V, I, I, _fp, U, _dp, _dp]),
    "pofd_like1_kernels_per_eval": (I, [V, C.POINTER(I)]),
    "pofd_like1_profile": (I, [V, U, _fp, U, I, _dp, C.POINTER(I)]),
    "pofd_like1_stage_name": (C.c_char_p, [V, I]),
    "pofd_like1_set_fft": (I, [V, I]),
    "pofd_like1_fft_info": (I, [V, C.POINTER(I)]),
    "pofd_like1_set_sigma_prior": (I, [V, I, D]),
    "pofd_like1_autotune": (I, [V, U, _fp, U, I, V]),
    "pofd_like1_get_tuning": (I, [V, _ip]),
    "pofd_like1_set_tuning": (I, [V, _ip]),
    "pofd_like2_set_sigma_prior": (I, [V, I, I, D]),
    "pofd_like2_set_cfirb_prior": (I, [V, I, I, D, D]),
    "pofd_like2_set_poisson_prior": (I, [V, I, I, D, D]),
    "pofd_like2_set_regularization": (I, [V, D]),
    "pofd_like2_bonus": (I, [V, U, _fp, U, _dp]),
    "pofd_like2_fill_bonus_device": (I, [V, U, V, U, V]),
    "pofd_like1_set_cfirb_prior": (I, [V, I, D, D]),
    "pofd_like1_set_poisson_prior": (I, [V, I, D, D]),
    "pofd_like1_set_regularization": (I, [V, D]),
    "pofd_like1_bonus": (I, [V, U, _fp, U, _dp]),
    "pofd_like1_fill_bonus_device": (I, [V, U, V, U, V]),
    "pofd_beam2_create": (I, [_dp, _dp, S, D, D, U, PV]),
    "pofd_beam2_destroy": (I, [V]),
    "pofd_beam2_info": (I, [V, _dp]),
    "pofd_like2_create": (I, [V, U, _dp, U, _dp, U, _dp, U, U, I, I, U, PV]),
    "pofd_like2_destroy": (I, [V]),
    "pofd_like2_add_beamset": (I, [V, V, D, D]),
    "pofd_like2_add_dataset": (I, [V, I, _dp, _dp, S, I, D, D, D]),
    "pofd_like2_set_rranges": (I, [V, _fp, U]),
    "pofd_like2_get_rrange": (I, [V, I, _dp]),
    "pofd_like2_dataset_info": (I, [V, I, I, _dp, V]),
    "pofd_like2_reserve": (I, [V, U]),
    "pofd_like2_loglike": (I, [V, _fp, U, C.POINTER(D), C.POINTER(I)]),
    "pofd_like2_eval_batch": (I, [V, U, V, U, V, V]),
    "pofd_like2_eval_batch_device": (I, [V, U, V, U, V, V, V]),
    "pofd_like2_pd": (I, [V, I, I, _fp, U, I, _dp, V]),
    "pofd_like2_get_r": (I, [V, I, _fp, U, _dp]),
    "pofd_like2_kernels_per_eval": (I, [V, C.POINTER(I)]),
    "pofd_like2_profile": (I, [V, U, _fp, U, I, _dp, C.POINTER(I)]),
    "pofd_like2_stage_name": (C.c_char_p, [I]),
    "pofd_like2_stage_name_now": (C.c_char_p, [V, I]),
    "pofd_like2_set_fft": (I, [V, I]),
    "pofd_like2_set_reference_sums": (I, [V, I]),
    "pofd_like2_active_terms": (I, [V, _fp, U, C.POINTER(C.c_longlong)]),
    "pofd_like2_autotune": (I, [V, U, _fp, U, I, V]),
    "pofd_like2_get_tuning": (I, [V, _ip]),
    "pofd_like2_set_tuning": (I, [V, _ip]),
    "pofd_like2_fft_info": (I, [V, C.POINTER(I)]),
    "pofd_pd1_loglike_noalloc": (I, [V, U, D, D, U, D, D, V, V, U, D, D, D, D,
                                     V, V, V]),
    "pofd_ensemble_create": (I, [V, U, U, D, C.c_ulonglong, PV]),
    "pofd_ensemble_destroy": (I, [V]),
    "pofd_ensemble_set_likelihood": (I, [V, V, V]),
    "pofd_ensemble_use_like1": (I, [V, V]),
    "pofd_ensemble_prepare_da": (I, [V]),
    "pofd_ensemble_set_bonus": (I, [V, V, V]),
    "pofd_ensemble_use_like2": (I, [V, V]),
    "pofd_ensemble_set_param_state": (I, [V, U, I]),
    "pofd_ensemble_set_param_limits": (I, [V, U, C.c_float, C.c_float]),
    "pofd_ensemble_set_temperature": (I, [V, D]),
    "pofd_ensemble_init": (I, [V, _fp, V]),
    "pofd_ensemble_reserve_chain": (I, [V, U]),
    "pofd_ensemble_clear_chain": (I, [V]),
    "pofd_ensemble_do_steps": (I, [V, U, I]),
    "pofd_ensemble_nrecorded": (I, [V, C.POINTER(U)]),
    "pofd_ensemble_chain": (I, [V, V, V]),
    "pofd_ensemble_last": (I, [V, V, V]),
    "pofd_ensemble_naccept": (I, [V, _up]),
    "pofd_ensemble_acor": (I, [V, _dp]),
    "pofd_surrogate_create": (I, [V, U, _ip, U, U, U, C.c_ulonglong, PV]),
    "pofd_surrogate_destroy": (I, [V]),
    "pofd_surrogate_add_pairs": (I, [V, U, V, U, V, V, V]),
    "pofd_surrogate_npairs": (I, [V, C.POINTER(U)]),
    "pofd_surrogate_get_pairs": (I, [V, U, V, V]),
    "pofd_surrogate_train": (I, [V, U, U, C.c_float, C.POINTER(C.c_float)]),
    "pofd_surrogate_predict_device": (I, [V, U, V, U, V, V, V]),
    "pofd_surrogate_get_params": (I, [V, I, V, C.POINTER(S)]),
    "pofd_surrogate_set_params": (I, [V, C.POINTER(C.c_void_p)]),
    "pofd_surrogate_gradients": (I, [V, U, C.POINTER(C.c_void_p),
                                     C.POINTER(C.c_float)]),
    "pofd_surrogate_scaling": (I, [V, _dp]),
    "pofd_bf16_gemm": (I, [I, I, I, V, I, V, I, V, I, V]),
    "pofd_ensemble_set_surrogate": (I, [V, V, V]),
    "pofd_ensemble_collect_pairs": (I, [V, V]),
    "pofd_ensemble_set_da_scale": (I, [V, D]),
    "pofd_ensemble_do_steps_da": (I, [V, U, I]),
    "pofd_ensemble_da_stats": (I, [V, C.POINTER(C.c_ulonglong)]),
    "pofd_likesum_create": (I, [V, PV]),
    "pofd_likesum_destroy": (I, [V]),
    "pofd_likesum_add": (I, [V, V, V]),
    "pofd_likesum_add_like1": (I, [V, V]),
    "pofd_likesum_add_like2": (I, [V, V]),
    "pofd_likesum_eval_batch_device": (I, [V, U, V, U, V, V, V]),
    "pofd_ensemble_set_error_policy": (I, [V, I]),
    "pofd_ensemble_set_limit_policy": (I, [V, I]),
    "pofd_ensemble_failures": (I, [V, C.POINTER(C.c_ulonglong)]),
    "pofd_pdfactory2_create": (I, [V, U, PV]),
    "pofd_pdfactory2_destroy": (I, [V]),
    "pofd_pdfactory2_initpd": (I, [V, U, D, D, D, D, U, _dp, U, _dp, U, _dp, _fp, V, I]),
    "pofd_pdfactory2_getpd": (I, [V, D, D, I, _dp, _dp]),
    "pofd_pdfactory2_get_r": (I, [V, _dp]),
    "pofd_acor": (I, [_fp, S, C.POINTER(D), C.POINTER(D), C.POINTER(D)]),
    "pofd_shard_rows": (I, [U, I, I, C.POINTER(U), C.POINTER(U)]),
    "pofd_nccl_unique_id": (I, [C.c_char_p]),
    "pofd_shard_create": (I, [V, C.c_char_p, I, I, V, V, PV]),
    "pofd_shard_destroy": (I, [V]),
    "pofd_shard_eval_batch_device": (I, [V, U, V, U, V, V, V]),
}

# libpofd_b200_support.so (include/pofd_b200_support.h): measurement and
# test helpers outside the likelihood's ABI
SUPPORT_SIGNATURES = {
    "pofd_fp64_peak": (I, [I, C.POINTER(D)]),
    "pofd_exp2_check": (I, [I, I, D, D, C.POINTER(D)]),
    "pofd_wait_check": (I, [I, U, I, C.POINTER(I)]),
    "pofd_gauss_create": (I, [I, U, _dp, _dp, PV]),
    "pofd_gauss_destroy": (I, [V]),
    "pofd_gauss_eval_batch_device": (I, [V, U, V, U, V, V, V]),
}

_lib = None
_support = None


class PofdError(RuntimeError):
    """Raised for a negative status; .code is the POFD_E_* value."""

    def __init__(self, code, msg):
        super().__init__("pofd error %d: %s" % (code, msg))
        self.code = code


def lib():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIBPATH):
        raise RuntimeError(
            "libpofd_b200.so is not built (%s); run python -m "
            "pofd_affine_b200.build" % LIBPATH)
    L = C.CDLL(LIBPATH)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


def support_lib():
    """The measurement / test helper library (FP64 peak, exp2 self-check,
    Gaussian test target)."""
    global _support
    if _support is not None:
        return _support
    if not os.path.exists(SUPPORT_LIBPATH):
        raise RuntimeError(
            "libpofd_b200_support.so is not built (%s); run python -m "
            "pofd_affine_b200.build" % SUPPORT_LIBPATH)
    L = C.CDLL(SUPPORT_LIBPATH)
    for name, (res, args) in SUPPORT_SIGNATURES.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _support = L
    return L


def check(st):
    if st < 0:
        raise PofdError(st, lib().pofd_last_error().decode())
    return st


def declared_functions(header=HEADER):
    """Function names declared in a header (default include/pofd_b200.h)."""
    import re
    txt = open(header).read()
    return sorted(set(re.findall(r"\b(pofd_[a-z0-9_]+)\s*\(", txt)))


def ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)
