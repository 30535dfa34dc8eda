"""ctypes binding of liboracle.so -- the CPU restatement of the reference (admix_oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and bench.py's CPU
baseline leg, as the checker.  Parity unpinned (see admix_oracle.c's header).
"""
from __future__ import annotations

import ctypes as C
import math
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "liboracle.so"

MU_AS_EXECUTED = 0
MU_GERSHGORIN = 1

_D = C.POINTER(C.c_double)
_I32 = C.POINTER(C.c_int32)
_I64 = C.POINTER(C.c_int64)
_U8 = C.POINTER(C.c_uint8)


class OrcState(C.Structure):
    _fields_ = [
        ("I", C.c_int64), ("J", C.c_int64), ("K", C.c_int32), ("Q", C.c_int32),
        ("bed", _U8),
        ("x", _D), ("x_next", _D), ("x_next2", _D), ("x_tmp", _D),
        ("XtX_q", _D), ("Xtz_q", _D), ("XtX_p", _D), ("Xtz_p", _D),
        ("U", _D), ("V", _D), ("vt", _D),
        ("ll_prev", C.c_double), ("ll_new", C.c_double),
        ("mu_mode", C.c_int32), ("fix", C.c_int32),
        ("mode", C.c_int32), ("x_q", _D), ("x_r", _D),
    ]


_lib = None


def build() -> Path:
    r = subprocess.run(["make", "-C", str(HERE)], capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"oracle build failed:\n{r.stdout}\n{r.stderr}")
    return LIB_PATH


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            build()
        L = C.CDLL(str(LIB_PATH))
        sig = {
            "orc_decode_counts": (None, [_U8, C.c_int64, C.c_int64, _I64, _I64]),
            "orc_loglik": (C.c_double, [_U8, C.c_int64, C.c_int64, C.c_int, _D, _D]),
            "orc_em_q": (None, [_U8, C.c_int64, C.c_int64, C.c_int, _D, _D, _D]),
            "orc_em_p": (None, [_U8, C.c_int64, C.c_int64, C.c_int, _D, _D, _D]),
            "orc_grad_hess_q": (None, [_U8, C.c_int64, C.c_int64, C.c_int, _D, _D, _D, _D]),
            "orc_grad_hess_p": (None, [_U8, C.c_int64, C.c_int64, C.c_int, _D, _D, _D, _D]),
            "orc_vt_ones": (None, [C.c_int, _D]),
            "orc_sweep": (None, [_D, C.c_int, C.c_int, _D, C.c_int]),
            "orc_create_tableau": (None, [_D, _D, _D, _D, _D, C.c_int, C.c_int, C.c_int, _D]),
            "orc_quadratic_program": (C.c_int, [_D, _D, _D, _D, _D, C.c_int, C.c_int, _D, _D, C.POINTER(C.c_int)]),
            "orc_project_q1": (None, [_D, C.c_int, C.c_double]),
            "orc_project_q": (None, [_D, C.c_int64, C.c_int]),
            "orc_project_p": (None, [_D, C.c_int64]),
            "orc_qp_batch": (None, [_D, _D, _D, _D, C.c_int, C.c_int64, C.c_int, C.c_int, _D, _I32]),
            "orc_update_q": (None, [C.POINTER(OrcState), C.c_int, _I32]),
            "orc_update_p": (None, [C.POINTER(OrcState), C.c_int, _I32]),
            "orc_loglik_x": (C.c_double, [C.POINTER(OrcState), _D]),
            "orc_init_em": (None, [C.POINTER(OrcState), C.c_int, _D]),
            "orc_qn_step": (None, [C.POINTER(OrcState), C.c_int]),
            "orc_qn_iteration": (C.c_int, [C.POINTER(OrcState), C.c_int, C.c_double, _D, _I32, _I32]),
            "orc_admixture_qn": (C.c_int, [C.POINTER(OrcState), C.c_int, C.c_double, C.c_int, _D, C.POINTER(C.c_int)]),
            "orc_num_threads": (C.c_int, []),
            "orc_set_mean_impute": (None, [_D]),
            "orc_snp_means": (None, [_U8, C.c_int64, C.c_int64, _D]),
        }
        for fn, (res, args) in sig.items():
            f = getattr(L, fn)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def _d(a):
    if a is None:
        return None
    assert a.dtype == np.float64 and a.flags.c_contiguous, (a.dtype, a.flags)
    return a.ctypes.data_as(_D)


def _u8(a):
    assert a.dtype == np.uint8 and a.flags.c_contiguous
    return a.ctypes.data_as(_U8)


# ----------------------------------------------------------------------------- functions
# Arrays follow the numpy mirror of Julia's column-major layout: q is (I, K), p is (J, K),
# XtX_q is (I, K, K) with XtX[i, k, k2] = Julia XtX_q[k2, k, i].

class _impute:
    """Selects the non-skipmissing (mean-imputed) loops for the calls inside the block when mu
    (the SNP means, length J) is given; the skipmissing loops otherwise."""

    def __init__(self, mu):
        self.mu = None if mu is None else np.ascontiguousarray(mu, dtype=np.float64)

    def __enter__(self):
        lib().orc_set_mean_impute(_d(self.mu) if self.mu is not None else None)

    def __exit__(self, *a):
        lib().orc_set_mean_impute(None)


def snp_means(bed: np.ndarray, I: int, J: int) -> np.ndarray:
    """g.mu of the SnpLinAlg (additive model): mean dosage over the non-missing individuals."""
    mu = np.empty(J)
    lib().orc_snp_means(_u8(bed), I, J, _d(mu))
    return mu


def decode_counts(bed: np.ndarray, I: int, J: int):
    snp = np.zeros(J, np.int64); ind = np.zeros(I, np.int64)
    lib().orc_decode_counts(_u8(bed), I, J, snp.ctypes.data_as(_I64), ind.ctypes.data_as(_I64))
    return snp, ind


def loglik(bed, I, J, K, q, p, mu=None) -> float:
    with _impute(mu):
        return lib().orc_loglik(_u8(bed), I, J, K, _d(q), _d(p))


def em_q(bed, I, J, K, q, p, mu=None):
    out = np.empty((I, K))
    with _impute(mu):
        lib().orc_em_q(_u8(bed), I, J, K, _d(q), _d(p), _d(out))
    return out


def em_p(bed, I, J, K, q, p, mu=None):
    out = np.empty((J, K))
    with _impute(mu):
        lib().orc_em_p(_u8(bed), I, J, K, _d(q), _d(p), _d(out))
    return out


def grad_hess_q(bed, I, J, K, q, p, mu=None):
    H = np.empty((I, K, K)); z = np.empty((I, K))
    with _impute(mu):
        lib().orc_grad_hess_q(_u8(bed), I, J, K, _d(q), _d(p), _d(H), _d(z))
    return H, z


def grad_hess_p(bed, I, J, K, q, p, mu=None):
    H = np.empty((J, K, K)); z = np.empty((J, K))
    with _impute(mu):
        lib().orc_grad_hess_p(_u8(bed), I, J, K, _d(q), _d(p), _d(H), _d(z))
    return H, z


def vt_ones(K: int) -> np.ndarray:
    """V' of svd(ones(1,K), full=true), returned as a numpy (K, K) array holding the
    column-major memory, i.e. the transpose of Julia's V'."""
    v = np.empty((K, K)); lib().orc_vt_ones(K, _d(v)); return v


def create_tableau(H, r, x, vt, simplex: bool, mu_mode: int = MU_AS_EXECUTED):
    K = H.shape[0]
    n = K + 2 if simplex else K + 1
    tab = np.empty((n, n)); tmp = np.empty(K + 2)
    lib().orc_create_tableau(_d(tab), _d(np.ascontiguousarray(H)), _d(np.ascontiguousarray(r)),
                             _d(np.ascontiguousarray(x)), _d(np.ascontiguousarray(vt)), K,
                             int(simplex), mu_mode, _d(tmp))
    return tab


def quadratic_program(tab, par, p: int, c: int):
    tab = np.ascontiguousarray(tab.copy())
    n = p + c + 1
    delta = np.empty(p); dd = np.empty(n); tmp = np.empty(n)
    swept = (C.c_int * p)()
    pmin = np.zeros(p); pmax = np.ones(p)
    it = lib().orc_quadratic_program(_d(delta), _d(tab), _d(np.ascontiguousarray(par, dtype=np.float64)),
                                     _d(pmin), _d(pmax), p, c, _d(dd), _d(tmp), swept)
    return it, delta, tab


def qp_batch(XtX, Xtz, x, simplex: bool, mu_mode: int = MU_AS_EXECUTED):
    """The QPs of update_q! (simplex=True) or update_p! (simplex=False) on given sums: XtX (n, K, K),
    Xtz (n, K) as the sweep returns them (negated here, as algorithms_inner.jl:196,272 does), x (n, K)
    the current block.  Returns (status (n,) int32, delta (n, K))."""
    n, K = x.shape
    r = np.ascontiguousarray(-np.asarray(Xtz, dtype=np.float64))
    H = np.ascontiguousarray(XtX, dtype=np.float64)
    xx = np.ascontiguousarray(x, dtype=np.float64)
    st = np.empty(n, np.int32); delta = np.empty((n, K))
    lib().orc_qp_batch(_d(H), _d(r), _d(xx), _d(np.ascontiguousarray(vt_ones(K))), K, n, int(simplex), mu_mode,
                       _d(delta), st.ctypes.data_as(_I32))
    return st, delta


def project_q1(b, pseudocount=1e-5):
    b = np.ascontiguousarray(b, dtype=np.float64).copy()
    lib().orc_project_q1(_d(b), len(b), pseudocount)
    return b


def project_p(b):
    b = np.ascontiguousarray(b, dtype=np.float64).copy()
    lib().orc_project_p(_d(b), b.size)
    return b


class OracleRun:
    """Oracle mirror of AdmixData + the outer loop (structs.jl, algorithms_outer.jl)."""

    def __init__(self, bed: np.ndarray, I: int, J: int, K: int, Q: int, x0: np.ndarray,
                 mu_mode: int = MU_AS_EXECUTED, fix_q: bool = False, fix_p: bool = False, mode: str = "ZAL",
                 skipmissing: bool = True):
        self.bed = np.ascontiguousarray(bed)
        self.I, self.J, self.K, self.Q = I, J, K, Q
        n = I + J
        self.x = np.ascontiguousarray(x0, dtype=np.float64).copy()
        self.x_next = np.zeros((n, K)); self.x_next2 = np.zeros((n, K)); self.x_tmp = np.zeros((n, K))
        self.XtX_q = np.zeros((I, K, K)); self.Xtz_q = np.zeros((I, K))
        self.XtX_p = np.zeros((J, K, K)); self.Xtz_p = np.zeros((J, K))
        self.U = np.zeros((Q, n * K)); self.V = np.zeros((Q, n * K))
        self.vt = vt_ones(K)
        s = OrcState()
        s.I, s.J, s.K, s.Q = I, J, K, Q
        s.bed = _u8(self.bed)
        s.x, s.x_next, s.x_next2, s.x_tmp = _d(self.x), _d(self.x_next), _d(self.x_next2), _d(self.x_tmp)
        s.XtX_q, s.Xtz_q, s.XtX_p, s.Xtz_p = _d(self.XtX_q), _d(self.Xtz_q), _d(self.XtX_p), _d(self.Xtz_p)
        s.U, s.V, s.vt = _d(self.U), _d(self.V), _d(self.vt)
        s.ll_prev = math.nan; s.ll_new = math.nan
        s.mu_mode = mu_mode
        s.fix = (1 if fix_q else 0) | (2 if fix_p else 0)
        if mode not in ("ZAL", "LBQN"):
            raise ValueError(f"Invalid mode {mode!r}")
        s.mode = 1 if mode == "LBQN" else 0
        # AdmixData(...; skipmissing=false): the mean-imputed loops with the SNP means g.mu
        self.mu = None if skipmissing else snp_means(self.bed, I, J)
        self.x_q = np.zeros(n * K); self.x_r = np.zeros(n * K)
        s.x_q, s.x_r = _d(self.x_q), _d(self.x_r)
        self.s = s

    @property
    def ll_new(self) -> float:
        return self.s.ll_new

    @ll_new.setter
    def ll_new(self, v: float) -> None:
        self.s.ll_new = v

    def loglik(self, x: np.ndarray) -> float:
        x = np.ascontiguousarray(x)
        with _impute(self.mu):
            return lib().orc_loglik_x(C.byref(self.s), _d(x))

    def init_em(self, iters: int) -> list[float]:
        hist = np.empty(max(iters, 1))
        with _impute(self.mu):
            lib().orc_init_em(C.byref(self.s), iters, _d(hist))
        return list(hist[:iters])

    def update_q(self, update2: bool) -> np.ndarray:
        st = np.empty(self.I, np.int32)
        with _impute(self.mu):
            lib().orc_update_q(C.byref(self.s), int(update2), st.ctypes.data_as(_I32))
        return st

    def update_p(self, update2: bool) -> np.ndarray:
        st = np.empty(self.J, np.int32)
        with _impute(self.mu):
            lib().orc_update_p(C.byref(self.s), int(update2), st.ctypes.data_as(_I32))
        return st

    def qn_iteration(self, it: int, rtol: float = 1e-7) -> dict:
        info = np.empty(5)
        with _impute(self.mu):
            stop = lib().orc_qn_iteration(C.byref(self.s), it, rtol, _d(info), None, None)
        return dict(ll_prev=info[0], ll_basic=info[1], ll_qn=info[2], ll_new=info[3], reldiff=info[4],
                    stop=bool(stop))

    def admixture_qn(self, n_iter: int = 1000, rtol: float = 1e-7, iter_offset: int = 0):
        hist = np.empty((max(n_iter, 1), 5))
        conv = C.c_int(0)
        with _impute(self.mu):
            n = lib().orc_admixture_qn(C.byref(self.s), n_iter, rtol, iter_offset, _d(hist), C.byref(conv))
        return hist[:n], bool(conv.value)


def num_threads() -> int:
    return lib().orc_num_threads()
