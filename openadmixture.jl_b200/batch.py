"""Restarts and K sweeps over one cohort, advanced together on the device (libadmix batches).

The reference solves one (K, seed) problem per run_admixture call (driver.jl:35-75); choosing K
or guarding against poor local optima means calling it many times.  AdmixBatch holds all those
problems over ONE device copy of the genotypes and advances them together: one batch iteration
is one CUDA graph launch whose independent branches are the members' admixture_qn! iterations,
so their kernels run concurrently, and members drop out as they converge.  Each member is an
ordinary handle (BatchMember, a CuAdmixData) for set / get / loglik calls.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _native as N
from .admixture import X, CuAdmixData
from .bed import DeviceGenotypes, Genotypes
from .synth import init_x


def _bcheck(rc: int, b=None) -> None:
    if rc != N.ADMIX_OK:
        msg = N.admix_lib().admix_batch_last_error(b)
        raise N.AdmixError(rc, msg.decode() if msg else "unknown error")


class BatchMember(CuAdmixData):
    """A member's handle, borrowed from its batch (closing it does not free it)."""

    def __init__(self, batch: "AdmixBatch", handle: C.c_void_p, K: int):
        self._h = handle
        self._batch = batch
        self.I, self.J, self.K, self.Q = batch.I, batch.J, K, batch.Q
        self.flags = batch.flags

    def close(self) -> None:
        self._h = None


class AdmixBatch:
    """n member problems over one cohort: member m has K = Ks[m] (repeat a K for restarts) and
    starts from init_x(I, J, K, seeds[m]) -- the random start of AdmixData (structs.jl:107,128)."""

    def __init__(self, g, Ks, *, Q: int = 3, flags: int = 0, seeds=None):
        self.Ks = [int(k) for k in Ks]
        n = len(self.Ks)
        self.I, self.J, self.Q, self.flags = g.I, g.J, Q, flags
        self.seeds = list(range(n)) if seeds is None else [int(s) for s in seeds]
        if len(self.seeds) != n:
            raise ValueError(f"{len(self.seeds)} seeds for {n} members")
        lib = N.admix_lib()
        ks = (C.c_int32 * max(n, 1))(*self.Ks)
        b = C.c_void_p()
        if isinstance(g, DeviceGenotypes):
            rc = lib.admix_batch_create_device(g.I, g.J, C.c_void_p(g.data.data_ptr()), g.Ib, n, ks, Q, flags,
                                               C.byref(b))
        else:
            rc = lib.admix_batch_create(g.I, g.J, N.u8ptr(g.data), n, ks, Q, flags, C.byref(b))
        _bcheck(rc, None)
        self._b = b
        self.members = []
        for m, K in enumerate(self.Ks):
            h = C.c_void_p()
            _bcheck(lib.admix_batch_member(b, m, C.byref(h)), b)
            mem = BatchMember(self, h, K)
            mem.upload(X, init_x(self.I, self.J, K, self.seeds[m]))
            self.members.append(mem)

    @property
    def handle(self) -> C.c_void_p:
        if self._b is None:
            raise ValueError("AdmixBatch has been closed")
        return self._b

    def __len__(self) -> int:
        return len(self.Ks)

    def close(self) -> None:
        if getattr(self, "_b", None) is not None:
            for mem in self.members:
                mem.close()
            N.admix_lib().admix_batch_destroy(self._b)
            self._b = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def init_em(self, iters: int = 5) -> np.ndarray:
        """init_em! on every member concurrently; returns the (n, iters) log-likelihoods."""
        hist = np.zeros((len(self), max(iters, 1)))
        _bcheck(N.admix_lib().admix_batch_init_em(self.handle, int(iters), N.dptr(hist)), self._b)
        return hist[:, :iters]

    def set_split(self, divisor: int) -> None:
        _bcheck(N.admix_lib().admix_batch_set_split(self.handle, int(divisor)), self._b)

    def autotune(self) -> tuple[int, float]:
        """Pick the work split of the members' passes by timing them concurrently; returns the
        chosen divisor and the milliseconds of one concurrent sweep + sweep + loglik probe."""
        d = C.c_int32()
        ms = C.c_double()
        _bcheck(N.admix_lib().admix_batch_autotune(self.handle, C.byref(d), C.byref(ms)), self._b)
        return d.value, ms.value

    def run_qn(self, n_iter: int = 1000, rtol: float = 1e-7) -> dict:
        """admixture_qn! on every member to convergence (or n_iter).  Returns per-member arrays
        (iterations, converged, ll = last iteration's log-likelihood) and the summed device
        milliseconds of the batch launches."""
        n = len(self)
        done = (C.c_int32 * n)()
        conv = (C.c_int32 * n)()
        last = (N.IterInfo * n)()
        ms = C.c_double()
        _bcheck(N.admix_lib().admix_batch_run_qn(self.handle, int(n_iter), float(rtol), done, conv, last,
                                                 C.byref(ms)), self._b)
        return {"iterations": np.array(done[:], dtype=np.int64), "converged": np.array(conv[:], dtype=bool),
                "ll": np.array([last[m].ll_new for m in range(n)]), "last": [last[m].as_dict() for m in range(n)],
                "ms_device": ms.value}

    def x(self, m: int) -> np.ndarray:
        """member m's current iterate, shape (I+J, K_m)"""
        return self.members[m].download(X)

    def best(self, K: int | None = None) -> int:
        """index of the member with the highest FP64 log-likelihood (among those with this K)"""
        cand = [m for m in range(len(self)) if K is None or self.Ks[m] == K]
        lls = [self.members[m].loglik(X) for m in cand]
        return cand[int(np.argmax(lls))]


def run_restarts(g, K: int, n_restarts: int, *, flags: int = 0, em_iters: int = 5, n_iter: int = 1000,
                 rtol: float = 1e-7, autotune: bool = True, seed0: int = 0):
    """n_restarts random starts of one K, solved together; returns (best x, its FP64 loglik,
    the run_qn record)."""
    with AdmixBatch(g, [K] * n_restarts, flags=flags, seeds=range(seed0, seed0 + n_restarts)) as b:
        if autotune:
            b.autotune()
        b.init_em(em_iters)
        rec = b.run_qn(n_iter, rtol)
        m = b.best()
        return b.x(m), b.members[m].loglik(X), rec


def k_sweep(g, Ks, *, flags: int = 0, em_iters: int = 5, n_iter: int = 1000, rtol: float = 1e-7,
            autotune: bool = True, seed: int = 0):
    """One run per K in Ks, solved together; returns {K: (x, FP64 loglik)} and the run_qn record."""
    with AdmixBatch(g, list(Ks), flags=flags, seeds=[seed] * len(Ks)) as b:
        if autotune:
            b.autotune()
        b.init_em(em_iters)
        rec = b.run_qn(n_iter, rtol)
        return {K: (b.x(m), b.members[m].loglik(X)) for m, K in enumerate(b.Ks)}, rec
