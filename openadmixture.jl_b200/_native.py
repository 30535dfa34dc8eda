"""ctypes binding of libadmix.so (include/admix.h) and libadmix_synth.so.

The libraries are built in-tree (``lib/``) by ``build.py``.  Loading fails loudly when they
are missing; there is no pure-Python stand-in for the engine.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

LIB_DIR = Path(__file__).resolve().parent / "lib"

ADMIX_OK = 0
ADMIX_ERR_ARG = 1
ADMIX_ERR_CUDA = 2
ADMIX_ERR_NOMEM = 3
ADMIX_ERR_UNSUPPORTED = 4
ADMIX_ERR_STATE = 5

ADMIX_X, ADMIX_X_NEXT, ADMIX_X_NEXT2, ADMIX_X_TMP = 0, 1, 2, 3
ADMIX_FLAG_MU_GERSHGORIN = 1
ADMIX_FLAG_MIXED = 2
ADMIX_FLAG_MEAN_IMPUTE = 4
ADMIX_MAX_K = 16
ADMIX_MAX_Q = 8

ADMIX_QN_ZAL, ADMIX_QN_LBQN = 0, 1
ADMIX_SKFR_GLOBAL, ADMIX_SKFR_LOCAL = 0, 1
ADMIX_PASS_LOGLIK, ADMIX_PASS_QSWEEP, ADMIX_PASS_PSWEEP, ADMIX_PASS_QQP, ADMIX_PASS_PQP, ADMIX_PASS_EM = range(6)


class AdmixError(RuntimeError):
    """A libadmix call returned a non-zero status."""

    def __init__(self, code: int, msg: str):
        super().__init__(f"libadmix error {code}: {msg}")
        self.code = code


class IterInfo(C.Structure):
    _fields_ = [
        ("ll_prev", C.c_double), ("ll_basic", C.c_double), ("ll_qn", C.c_double),
        ("ll_new", C.c_double), ("reldiff", C.c_double),
        ("iter", C.c_int32), ("accepted_qn", C.c_int32),
        ("qp_fail_q", C.c_int32), ("qp_fail_p", C.c_int32),
    ]

    def as_dict(self) -> dict:
        return {f: getattr(self, f) for f, _ in self._fields_}


class MLPNet(C.Structure):
    _fields_ = [("S", C.c_int32), ("R", C.c_int32), ("H", C.c_int32), ("K", C.c_int32),
                ("w1", C.c_void_p), ("b1", C.c_void_p), ("w2", C.c_void_p), ("b2", C.c_void_p),
                ("w3", C.c_void_p), ("b3", C.c_void_p)]


class MLPGrads(C.Structure):
    _fields_ = [("w1", C.c_void_p), ("b1", C.c_void_p), ("w2", C.c_void_p), ("b2", C.c_void_p),
                ("w3", C.c_void_p), ("b3", C.c_void_p)]


_P = C.c_void_p
_D = C.POINTER(C.c_double)
_I32 = C.POINTER(C.c_int32)
_I64 = C.POINTER(C.c_int64)
_U8 = C.POINTER(C.c_uint8)

# name -> (restype, argtypes); every symbol include/admix.h declares
ADMIX_SIGNATURES = {
    "admix_create": (C.c_int, [C.c_int64, C.c_int64, C.c_int32, C.c_int32, _U8, C.c_uint32, C.POINTER(_P)]),
    "admix_create_device": (C.c_int, [C.c_int64, C.c_int64, C.c_int32, C.c_int32, _P, C.c_int64, C.c_uint32, C.POINTER(_P)]),
    "admix_create_streamed": (C.c_int, [C.c_int64, C.c_int64, C.c_int32, C.c_int32, _U8, C.c_int64, C.c_uint32,
                                        C.POINTER(_P)]),
    "admix_destroy": (C.c_int, [_P]),
    "admix_last_error": (C.c_char_p, [_P]),
    "admix_device_bytes": (C.c_int, [_P, _I64]),
    "admix_set_x": (C.c_int, [_P, C.c_int32, _D, _D]),
    "admix_get_x": (C.c_int, [_P, C.c_int32, _D, _D]),
    "admix_set_ll": (C.c_int, [_P, C.c_double]),
    "admix_set_qn_mode": (C.c_int, [_P, C.c_int32]),
    "admix_get_ll": (C.c_int, [_P, _D]),
    "admix_loglik": (C.c_int, [_P, C.c_int32, _D]),
    "admix_em_q": (C.c_int, [_P]),
    "admix_em_p": (C.c_int, [_P]),
    "admix_init_em": (C.c_int, [_P, C.c_int32, _D]),
    "admix_grad_hess_q": (C.c_int, [_P, C.c_int32, C.c_int32, _D, _D]),
    "admix_grad_hess_p": (C.c_int, [_P, C.c_int32, C.c_int32, _D, _D]),
    "admix_update_q": (C.c_int, [_P, C.c_int32, _I32]),
    "admix_update_p": (C.c_int, [_P, C.c_int32, _I32]),
    "admix_set_fixed": (C.c_int, [_P, C.c_int32, C.c_int32]),
    "admix_selftest_wait_timeout": (C.c_int, [_P]),
    "admix_tc_probe": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32, C.c_int32]),
    "admix_skfr": (C.c_int, [_P, C.c_int32, C.c_int64, C.c_int32, C.c_int32, C.c_int32, C.c_uint64, _I32, _I32, C.c_int64, _I64, _D, _I32]),
    "admix_qn_iteration": (C.c_int, [_P, C.c_int32, C.POINTER(IterInfo)]),
    "admix_run_qn": (C.c_int, [_P, C.c_int32, C.c_double, C.c_int32, C.POINTER(IterInfo), _I32, _I32]),
    "admix_decode_counts": (C.c_int, [_P, _I64, _I64]),
    "admix_stream": (C.c_int, [_P, C.POINTER(_P)]),
    "admix_time_pass": (C.c_int, [_P, C.c_int32, C.c_int32, _D]),
    "admix_iteration_kernels": (C.c_int, [_P, _I32]),
    "admix_loglik_dev_workspace": (C.c_size_t, [C.c_int64, C.c_int64, C.c_int32]),
    "admix_loglik_dev": (C.c_int, [_P, C.c_int64, C.c_int64, C.c_int32, _P, _P, _P, _P, C.c_size_t, _P]),
    "admix_loglik_dev_noalloc": (C.c_int, [_P, C.c_int64, C.c_int64, C.c_int32, _P, _P, _P, _P]),
    "admix_sketch": (C.c_int, [_P, C.c_int64, C.c_int64, _P, C.c_int32, C.c_int32, C.c_uint64, _P, _P, _P, _P]),
    "admix_mlp_forward": (C.c_int, [C.POINTER(MLPNet), C.c_int64, _P, _P, _P, _P, _P, _P, _P, _P]),
    "admix_mlp_backward": (C.c_int, [C.POINTER(MLPNet), C.POINTER(MLPGrads), C.c_int64, _P, _P, _P, _P, _P, _P,
                                     _P, _P, _P, _P, _P, _P, _P]),
    "admix_mlp_adam": (C.c_int, [_P, _P, _P, _P, C.c_int64, C.c_float, C.c_float, C.c_float, C.c_float,
                                 C.c_int32, _P]),
    "admix_warm_p": (C.c_int, [_P, C.c_int64, C.c_int64, C.c_int64, C.c_int32, _P, _P, _P]),
    "admix_noalloc_last_error": (C.c_char_p, []),
    "admix_batch_create": (C.c_int, [C.c_int64, C.c_int64, _U8, C.c_int32, _I32, C.c_int32, C.c_uint32,
                                     C.POINTER(_P)]),
    "admix_batch_create_device": (C.c_int, [C.c_int64, C.c_int64, _P, C.c_int64, C.c_int32, _I32, C.c_int32,
                                            C.c_uint32, C.POINTER(_P)]),
    "admix_batch_destroy": (C.c_int, [_P]),
    "admix_batch_last_error": (C.c_char_p, [_P]),
    "admix_batch_size": (C.c_int, [_P, _I32]),
    "admix_batch_member": (C.c_int, [_P, C.c_int32, C.POINTER(_P)]),
    "admix_batch_init_em": (C.c_int, [_P, C.c_int32, _D]),
    "admix_batch_set_split": (C.c_int, [_P, C.c_int32]),
    "admix_batch_autotune": (C.c_int, [_P, _I32, _D]),
    "admix_batch_run_qn": (C.c_int, [_P, C.c_int32, C.c_double, _I32, _I32, C.POINTER(IterInfo), _D]),
}

SYNTH_SIGNATURES = {
    "syn_truth": (C.c_int, [C.c_int64, C.c_int64, C.c_int32, C.c_uint64, C.c_int32, C.c_double,
                            C.c_double, C.c_double, C.c_double, _D, _D]),
    "syn_bed_host": (C.c_int, [C.c_int64, C.c_int64, C.c_int32, C.c_uint64, C.c_double, _D, _D, _U8]),
    "syn_bed_device": (C.c_int, [C.c_int64, C.c_int64, C.c_int32, C.c_uint64, C.c_double, _P, _P, _P, _P]),
    "syn_init_x": (C.c_int, [C.c_int64, C.c_int64, C.c_int32, C.c_uint64, _D]),
}

_admix = None
_synth = None


def _load(name: str, sigs: dict) -> C.CDLL:
    path = LIB_DIR / name
    if not path.exists():
        raise ImportError(
            f"{path} is missing: build the native libraries first "
            f"(python -c 'import __graft_entry__ as g; g.build()')")
    lib = C.CDLL(str(path))
    for fn, (res, args) in sigs.items():
        f = getattr(lib, fn)
        f.restype = res
        f.argtypes = args
    return lib


def admix_lib() -> C.CDLL:
    global _admix
    if _admix is None:
        _admix = _load("libadmix.so", ADMIX_SIGNATURES)
    return _admix


def synth_lib() -> C.CDLL:
    global _synth
    if _synth is None:
        _synth = _load("libadmix_synth.so", SYNTH_SIGNATURES)
    return _synth


def dptr(a: np.ndarray | None):
    if a is None:
        return None
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(_D)


def i32ptr(a: np.ndarray | None):
    if a is None:
        return None
    assert a.dtype == np.int32 and a.flags.c_contiguous
    return a.ctypes.data_as(_I32)


def i64ptr(a: np.ndarray | None):
    if a is None:
        return None
    assert a.dtype == np.int64 and a.flags.c_contiguous
    return a.ctypes.data_as(_I64)


def u8ptr(a: np.ndarray):
    assert a.dtype == np.uint8 and a.flags.c_contiguous
    return a.ctypes.data_as(_U8)


def check(rc: int, handle=None) -> None:
    if rc != ADMIX_OK:
        msg = admix_lib().admix_last_error(handle)
        raise AdmixError(rc, msg.decode() if msg else "unknown error")
