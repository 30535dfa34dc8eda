"""Host API mirroring OpenADMIXTURE.jl's run_admixture / AdmixData / GPU hook, driving libadmix.

Names and argument meanings follow the reference (Julia ``!`` suffixes dropped):

    AdmixData(I, J, K, Q; rng)            structs.jl:105-215
    _cu_admixture_base(d, g, I, J)         cuda/structs.jl:33-39  -> (d_cu, g_cu)
    loglikelihood(d_cu, g_cu)              cuda/runners.jl:13-20
    em_q(d_cu, g_cu), em_p(d_cu, g_cu)     cuda/runners.jl:36-67
    update_q(d, g, update2; d_cu, g_cu)    algorithms_inner.jl:167-231
    update_p(d, g, update2; d_cu, g_cu)    algorithms_inner.jl:245-310
    init_em(d, g, iter; d_cu, g_cu)        algorithms_outer.jl:12-45
    admixture_qn(d, g, iter, rtol; ...)    algorithms_outer.jl:63-193
    run_admixture(filename, K; ...)        driver.jl:35-75

Every numeric step runs in libadmix on the GPU.  The reference's CPU loops (d_cu === nothing)
are the reference itself; asking for them here (use_gpu=False, d_cu=None) raises.
"""
from __future__ import annotations

import ctypes as C
import math
import time

import numpy as np

from . import _native as N
from .bed import DeviceGenotypes, Genotypes, read_bed
from .synth import init_x

X, X_NEXT, X_NEXT2, X_TMP = N.ADMIX_X, N.ADMIX_X_NEXT, N.ADMIX_X_NEXT2, N.ADMIX_X_TMP


class AdmixData:
    """Host state of one run (AdmixData{T}, structs.jl:9-91).

    x, x_next, x_next2, x_tmp are numpy arrays of shape (I+J, K) -- the memory of Julia's
    K x (I+J) column-major matrices.  ``q``/``p`` (and the _next/_next2/_tmp variants) are
    K x I / K x J views, indexed q[k, i] as in the reference.
    """

    def __init__(self, I: int, J: int, K: int, Q: int = 3, *, skipmissing: bool = True, rng: int = 0):
        self.I, self.J, self.K, self.Q = int(I), int(J), int(K), int(Q)
        # skipmissing=False: the mean-imputed loops (ADMIX_FLAG_MEAN_IMPUTE on the handle)
        self.skipmissing = bool(skipmissing)
        self.x = init_x(self.I, self.J, self.K, int(rng))
        self.x_next = np.zeros_like(self.x)
        self.x_next2 = np.zeros_like(self.x)
        self.x_tmp = np.zeros_like(self.x)
        self.ll_prev = math.nan
        self.ll_new = math.nan

    def _qv(self, x):
        return x[: self.I].T

    def _pv(self, x):
        return x[self.I:].T

    q = property(lambda s: s._qv(s.x))
    p = property(lambda s: s._pv(s.x))
    q_next = property(lambda s: s._qv(s.x_next))
    p_next = property(lambda s: s._pv(s.x_next))
    q_next2 = property(lambda s: s._qv(s.x_next2))
    p_next2 = property(lambda s: s._pv(s.x_next2))
    q_tmp = property(lambda s: s._qv(s.x_tmp))
    p_tmp = property(lambda s: s._pv(s.x_tmp))

    def buffer(self, which: int) -> np.ndarray:
        return (self.x, self.x_next, self.x_next2, self.x_tmp)[which]


class CuAdmixData:
    """Device-resident state (the CuAdmixData{T} role, cuda/structs.jl:1-31): the packed
    genotypes, the four iterates, the secant matrices and the sweep workspaces, owned by one
    libadmix handle."""

    def __init__(self, d: AdmixData, g: Genotypes, *, flags: int = 0, stream_block: int | None = None):
        """stream_block: keep the genotypes in host memory and stream them through the device in
        blocks of that many SNPs (a multiple of 32) -- for cohorts larger than device memory."""
        if (g.I, g.J) != (d.I, d.J):
            raise ValueError(f"genotypes are {g.I} x {g.J}, AdmixData is {d.I} x {d.J}")
        if not d.skipmissing:      # AdmixData(...; skipmissing=false): the mean-imputed loops
            flags |= N.ADMIX_FLAG_MEAN_IMPUTE
        lib = N.admix_lib()
        h = C.c_void_p()
        self._host_bed = None
        if stream_block is not None:
            if isinstance(g, DeviceGenotypes):
                raise ValueError("stream_block needs genotypes in host memory")
            self._host_bed = np.ascontiguousarray(g.data)      # must outlive the handle
            N.check(lib.admix_create_streamed(d.I, d.J, d.K, d.Q, N.u8ptr(self._host_bed), int(stream_block), flags,
                                              C.byref(h)), None)
        elif isinstance(g, DeviceGenotypes):
            N.check(lib.admix_create_device(d.I, d.J, d.K, d.Q, C.c_void_p(g.data.data_ptr()), g.Ib, flags,
                                            C.byref(h)), None)
        else:
            N.check(lib.admix_create(d.I, d.J, d.K, d.Q, N.u8ptr(g.data), flags, C.byref(h)), None)
        self._h = h
        self.I, self.J, self.K, self.Q = d.I, d.J, d.K, d.Q
        self.flags = flags

    @property
    def handle(self) -> C.c_void_p:
        if self._h is None:
            raise ValueError("CuAdmixData has been closed")
        return self._h

    def _chk(self, rc: int) -> None:
        N.check(rc, self._h)

    def close(self) -> None:
        if getattr(self, "_h", None) is not None:
            N.admix_lib().admix_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # copyto_sync! (cuda/transfer.jl) in both directions, on whole iterates
    def upload(self, which: int, x: np.ndarray) -> None:
        x = np.ascontiguousarray(x, dtype=np.float64)
        self._chk(N.admix_lib().admix_set_x(self.handle, which, N.dptr(x[: self.I]), N.dptr(x[self.I:])))

    def upload_qp(self, which: int, q: np.ndarray | None = None, p: np.ndarray | None = None) -> None:
        """q is K x I (or (I, K) memory), p is K x J; either may be None."""
        qa = None if q is None else np.ascontiguousarray(np.asarray(q, dtype=np.float64).T if q.shape == (self.K, self.I) else q)
        pa = None if p is None else np.ascontiguousarray(np.asarray(p, dtype=np.float64).T if p.shape == (self.K, self.J) else p)
        self._chk(N.admix_lib().admix_set_x(self.handle, which, N.dptr(qa), N.dptr(pa)))

    def download(self, which: int, out: np.ndarray | None = None) -> np.ndarray:
        if out is None:
            out = np.empty((self.I + self.J, self.K), dtype=np.float64)
        q = np.empty((self.I, self.K)); p = np.empty((self.J, self.K))
        self._chk(N.admix_lib().admix_get_x(self.handle, which, N.dptr(q), N.dptr(p)))
        out[: self.I] = q
        out[self.I:] = p
        return out

    def loglik(self, which: int = X) -> float:
        v = C.c_double()
        self._chk(N.admix_lib().admix_loglik(self.handle, which, C.byref(v)))
        return v.value

    def set_ll(self, ll: float) -> None:
        self._chk(N.admix_lib().admix_set_ll(self.handle, float(ll)))

    def get_ll(self) -> float:
        v = C.c_double()
        self._chk(N.admix_lib().admix_get_ll(self.handle, C.byref(v)))
        return v.value

    def grad_hess_q(self, which_q: int = X, which_p: int = X) -> tuple[np.ndarray, np.ndarray]:
        """(XtX_q, Xtz_q) in the reference layout: arrays of shape (I, K, K) and (I, K) holding
        the memory of Julia's K x K x I and K x I arrays (XtX[i] is XtX_q[:, :, i]')."""
        XtX = np.empty((self.I, self.K, self.K)); Xtz = np.empty((self.I, self.K))
        self._chk(N.admix_lib().admix_grad_hess_q(self.handle, which_q, which_p, N.dptr(XtX), N.dptr(Xtz)))
        return XtX, Xtz

    def grad_hess_p(self, which_q: int = X_NEXT, which_p: int = X) -> tuple[np.ndarray, np.ndarray]:
        XtX = np.empty((self.J, self.K, self.K)); Xtz = np.empty((self.J, self.K))
        self._chk(N.admix_lib().admix_grad_hess_p(self.handle, which_q, which_p, N.dptr(XtX), N.dptr(Xtz)))
        return XtX, Xtz

    def decode_counts(self) -> tuple[np.ndarray, np.ndarray]:
        snp = np.empty(self.J, dtype=np.int64); ind = np.empty(self.I, dtype=np.int64)
        self._chk(N.admix_lib().admix_decode_counts(self.handle, N.i64ptr(snp), N.i64ptr(ind)))
        return snp, ind

    def stream(self) -> int:
        v = C.c_void_p()
        self._chk(N.admix_lib().admix_stream(self.handle, C.byref(v)))
        return v.value or 0

    def time_pass(self, pass_id: int, reps: int = 5) -> float:
        """Mean device milliseconds of one launch of a pass (CUDA events on the handle's stream)."""
        v = C.c_double()
        self._chk(N.admix_lib().admix_time_pass(self.handle, pass_id, reps, C.byref(v)))
        return v.value

    def iteration_kernels(self) -> int:
        v = C.c_int32()
        self._chk(N.admix_lib().admix_iteration_kernels(self.handle, C.byref(v)))
        return v.value

    def device_bytes(self) -> int:
        v = C.c_int64()
        self._chk(N.admix_lib().admix_device_bytes(self.handle, C.byref(v)))
        return v.value


def _require_gpu(d_cu) -> CuAdmixData:
    if d_cu is None:
        raise NotImplementedError(
            "this engine is the GPU drop-in; the CPU loops (d_cu === nothing) are the reference's own "
            "code path -- pass d_cu from _cu_admixture_base(d, g, I, J)")
    return d_cu


def _cu_admixture_base(d: AdmixData, g: Genotypes, I: int, J: int, *, flags: int = 0,
                       stream_block: int | None = None):
    """Allocate the device state and upload the genotype bytes once (cuda/structs.jl:33-39).
    Returns (d_cu, g_cu); the genotypes live inside d_cu, so g_cu is the same object."""
    if (I, J) != (d.I, d.J):
        raise ValueError("I, J disagree with AdmixData")
    d_cu = CuAdmixData(d, g, flags=flags, stream_block=stream_block)
    return d_cu, d_cu


def loglikelihood(d_cu: CuAdmixData, g_cu=None) -> float:
    """loglikelihood(d_cu, g_cu) (cuda/runners.jl:13-20): loglik at the device (q, p)."""
    return _require_gpu(d_cu).loglik(X)


def em_q(d_cu: CuAdmixData, g_cu=None, *, verbose: bool = False) -> None:
    """em_q!(d_cu, g_cu): q_next = EM update of Q at (q, p) (cuda/runners.jl:36-43)."""
    _require_gpu(d_cu)._chk(N.admix_lib().admix_em_q(d_cu.handle))


def em_p(d_cu: CuAdmixData, g_cu=None, *, verbose: bool = False) -> None:
    """em_p!(d_cu, g_cu): p_next = EM update of P at (q, p) (cuda/runners.jl:60-67)."""
    _require_gpu(d_cu)._chk(N.admix_lib().admix_em_p(d_cu.handle))


def update_q(d: AdmixData, g, update2: bool = False, *, d_cu: CuAdmixData | None = None, g_cu=None,
             verbose: bool = False) -> np.ndarray:
    """update_q!(d, g, update2) (algorithms_inner.jl:167-231): q_next (or q_next2) of d from one
    SQP step at (q, p) (or (q_next, p_next)).  Returns quadratic_program!'s status per individual."""
    d_cu = _require_gpu(d_cu)
    if update2:
        d_cu.upload(X_NEXT, d.x_next)
    else:
        d_cu.upload(X, d.x)
    d.ll_prev = d.ll_new
    st = np.empty(d.I, dtype=np.int32)
    d_cu._chk(N.admix_lib().admix_update_q(d_cu.handle, int(bool(update2)), N.i32ptr(st)))
    out = d_cu.download(X_NEXT2 if update2 else X_NEXT)
    (d.x_next2 if update2 else d.x_next)[: d.I] = out[: d.I]
    return st


def update_p(d: AdmixData, g, update2: bool = False, *, d_cu: CuAdmixData | None = None, g_cu=None,
             verbose: bool = False) -> np.ndarray:
    """update_p!(d, g, update2) (algorithms_inner.jl:245-310): p_next from (q_next, p), or p_next2
    from (q_next2, p_next).  Returns quadratic_program!'s status per SNP."""
    d_cu = _require_gpu(d_cu)
    if update2:
        d_cu.upload_qp(X_NEXT2, q=d.x_next2[: d.I])
        d_cu.upload_qp(X_NEXT, p=d.x_next[d.I:])
    else:
        d_cu.upload_qp(X_NEXT, q=d.x_next[: d.I])
        d_cu.upload_qp(X, p=d.x[d.I:])
    d.ll_prev = d.ll_new
    st = np.empty(d.J, dtype=np.int32)
    d_cu._chk(N.admix_lib().admix_update_p(d_cu.handle, int(bool(update2)), N.i32ptr(st)))
    out = d_cu.download(X_NEXT2 if update2 else X_NEXT)
    (d.x_next2 if update2 else d.x_next)[d.I:] = out[d.I:]
    return st


def init_em(d: AdmixData, g, iters: int, *, d_cu: CuAdmixData | None = None, g_cu=None,
            verbose: bool = False, quiet: bool = False) -> list[float]:
    """init_em!(d, g, iter) (algorithms_outer.jl:12-45): `iters` FRAPPE EM steps on the device,
    then d.q, d.p and d.ll_new updated.  Returns the per-iteration log-likelihoods."""
    d_cu = _require_gpu(d_cu)
    d_cu.upload(X, d.x)
    if not quiet:
        print(f"Performing {iters} EM steps for priming")
    hist = np.empty(max(iters, 1))
    t0 = time.perf_counter()
    d_cu._chk(N.admix_lib().admix_init_em(d_cu.handle, int(iters), N.dptr(hist)))
    dt = time.perf_counter() - t0
    if not quiet:
        for i in range(iters):
            print(f"EM Iteration {i + 1} ({dt / max(iters, 1):.6f} sec): Loglikelihood = {hist[i]}")
    d_cu.download(X, d.x)
    d.ll_new = d_cu.get_ll()
    return list(hist[:iters])


def admixture_qn(d: AdmixData, g, iter: int = 1000, rtol: float = 1e-7, *, d_cu: CuAdmixData | None = None,
                 g_cu=None, mode: str = "ZAL", iter_count_offset: int = 0, fix_p: bool = False,
                 fix_q: bool = False, verbose: bool = False, progress_bar: bool = False,
                 quiet: bool = False) -> list[dict]:
    """admixture_qn!(d, g, iter, rtol) (algorithms_outer.jl:63-193), run on the device; mode "ZAL"
    (default) or "LBQN" (quasi_newton.jl:15-58), fix_q / fix_p as the reference's keywords.
    Returns one record per iteration (ll_prev, ll_basic, ll_qn, ll_new, reldiff, ...)."""
    d_cu = _require_gpu(d_cu)
    modes = {"ZAL": N.ADMIX_QN_ZAL, "LBQN": N.ADMIX_QN_LBQN}
    if str(mode).lstrip(":") not in modes:
        raise ValueError(f"Invalid mode {mode!r} (:ZAL or :LBQN)")      # the reference's @assert false
    lib = N.admix_lib()
    d_cu._chk(lib.admix_set_qn_mode(d_cu.handle, modes[str(mode).lstrip(":")]))
    d_cu._chk(lib.admix_set_fixed(d_cu.handle, int(bool(fix_q)), int(bool(fix_p))))
    try:
        return _admixture_qn_loop(d, d_cu, iter, rtol, iter_count_offset, verbose, quiet)
    finally:
        d_cu._chk(lib.admix_set_fixed(d_cu.handle, 0, 0))
        d_cu._chk(lib.admix_set_qn_mode(d_cu.handle, N.ADMIX_QN_ZAL))


def _admixture_qn_loop(d: AdmixData, d_cu: CuAdmixData, iter: int, rtol: float, iter_count_offset: int,
                       verbose: bool, quiet: bool) -> list[dict]:
    d_cu.upload(X, d.x)
    if math.isnan(d.ll_new):
        d.ll_new = d_cu.loglik(X)
    d_cu.set_ll(d.ll_new)
    if not quiet:
        print("initial ll: ", d.ll_new)
        print("Starting main algorithm")
    lib = N.admix_lib()
    recs = []
    converged = False
    i = iter_count_offset
    t_loop = time.perf_counter()
    for i in range(iter_count_offset + 1, iter + 1):
        info = N.IterInfo()
        t0 = time.perf_counter()
        d_cu._chk(lib.admix_qn_iteration(d_cu.handle, i, C.byref(info)))
        dt = time.perf_counter() - t0
        rec = info.as_dict()
        rec["time"] = dt
        recs.append(rec)
        d.ll_prev, d.ll_new = info.ll_prev, info.ll_new
        if not quiet:
            print(f"Iteration {i} ({dt} sec): LogLikelihood = {info.ll_new}, reldiff = {info.reldiff}")
            print(f"    LogLikelihoods: Previous = {info.ll_prev} QN = {info.ll_qn}, Basic = {info.ll_basic}")
        if info.reldiff < rtol:
            converged = True
            break
    total = time.perf_counter() - t_loop
    d_cu.download(X, d.x)
    if not quiet:
        if converged:
            print(f"Main algorithm converged in {i} iterations over {total} sec.")
        else:
            print(f"Main algorithm failed to converge after {i} iterations over {total} sec.")
    return recs


def skfr(g, K: int, sparsity: int, *, mode: str = "global", max_iter: int = 50, tries: int = 1, rng: int = 0):
    """Sparse k-means via feature ranking (the reference's SparseKmeansFeatureRanking.sparsekmeans1
    for mode "global", sparsekmeans2 for "local", sparsekmeans_repeat for tries > 1; driver.jl:56-69,
    80-101) on the device: K clusters of the individuals on the `sparsity` most informative SNPs of
    the imputed, standardised genotypes.  Returns (clusters (I,) in 0..K-1, aims (the selected SNP
    indices, 0-based and increasing), objective, iterations).  ``rng`` seeds the k-means++
    seeding (a splitmix64 stream; the reference's Julia RNG is not reproduced)."""
    modes = {"global": N.ADMIX_SKFR_GLOBAL, "local": N.ADMIX_SKFR_LOCAL}
    mode = str(mode).lstrip(":")
    if mode not in modes:
        raise ValueError("skfr_mode can only be :global or :local")        # driver.jl:63
    d = AdmixData(g.I, g.J, min(K, 16), 1, rng=rng)
    with CuAdmixData(d, g) as h:
        clusters = np.empty(g.I, dtype=np.int32)
        cap = min(g.J, sparsity * (K if mode == "local" else 1))
        aims = np.empty(max(cap, 1), dtype=np.int32)
        n_aims = C.c_int64(0)
        obj = C.c_double(0.0)
        iters = C.c_int32(0)
        h._chk(N.admix_lib().admix_skfr(h.handle, int(K), int(sparsity), modes[mode], int(max_iter), int(tries),
                                        int(rng) & ((1 << 64) - 1), N.i32ptr(clusters), N.i32ptr(aims), cap,
                                        C.byref(n_aims), C.byref(obj), C.byref(iters)))
    return clusters, aims[: n_aims.value].copy(), obj.value, iters.value


def _filter_skfr(g, K: int, sparsity: int, *, rng: int = 0, prefix=None, tries: int = 1, max_inner_iter: int = 50,
                 mode: str = "global", source=None, quiet: bool = False):
    """_filter_SKFR (driver.jl:80-101): SKFR, then the genotypes of the selected SNPs only --
    written as `{prefix}_{K}_{sparsity}aims.bed` (.bim / .fam beside it, copied from the source's
    where it has them) when a prefix is given -- returned with clusters and aims."""
    clusters, aims, _, _ = skfr(g, K, sparsity, mode=mode, max_iter=max_inner_iter, tries=tries, rng=rng)
    if isinstance(g, DeviceGenotypes):
        import torch
        sub = DeviceGenotypes(g.data.index_select(0, torch.as_tensor(aims, dtype=torch.long, device=g.data.device)),
                              g.I, len(aims))
    else:
        sub = Genotypes(np.ascontiguousarray(np.asarray(g.data)[aims]), g.I, len(aims))
    if prefix is not None:
        from pathlib import Path
        from .bed import write_bed
        des = Path(f"{prefix}_{K}_{sparsity}aims.bed")
        if not quiet:
            print(des.with_suffix(""))
        host = sub.to_host() if isinstance(sub, DeviceGenotypes) else sub
        write_bed(des, host, write_sidecars=True)
        if source is not None:                      # keep the source's identifiers
            src = Path(source).with_suffix("")
            if src.with_suffix(".fam").exists():
                des.with_suffix(".fam").write_text(src.with_suffix(".fam").read_text())
            if src.with_suffix(".bim").exists():
                lines = src.with_suffix(".bim").read_text().splitlines()
                des.with_suffix(".bim").write_text("".join(lines[j] + "\n" for j in aims))
    return sub, clusters, aims


def run_admixture(filename, K: int, *, rng: int = 0, sparsity=None, prefix=None, skfr_tries: int = 1,
                  skfr_max_inner_iter: int = 50, skfr_mode: str = "global", admix_n_iter: int = 1000,
                  admix_rtol: float = 1e-7, admix_n_em_iters: int = 5, T=np.float64, Q: int = 3,
                  use_gpu: bool = True, verbose: bool = False, progress_bar: bool = False,
                  fix_q: bool = False, fix_p: bool = False, init_q=None, init_p=None,
                  quiet: bool = False, flags: int = 0, warm_start=None, stream_block: int | None = None):
    """run_admixture(filename, K; ...) (driver.jl:35-75) -> (d, clusters, aims).

    ``filename`` is a .bed path, an in-memory Genotypes or a DeviceGenotypes.  ``rng`` is an
    integer seed of this engine's generator (the reference's Julia RNG streams are not
    reproduced).  sparsity (an integer) first selects that many ancestry-informative SNPs with
    SKFR on the device (`skfr`; skfr_mode, skfr_tries and skfr_max_inner_iter as the reference's
    keywords) and runs the engine on them; the filtered genotypes are written as
    `{prefix}_{K}_{sparsity}aims.bed` (prefix defaults to the .bed path without its suffix; no
    file for in-memory genotypes without a prefix), and clusters and aims are returned.

    init_q (K x I) / init_p (K x J): as in the reference, EM priming runs unless both are given
    (driver.jl:180); a given one overwrites the primed value.  warm_start ("learned", a model
    path or a WarmStartMLP) starts from the learned encoder's Q and the closed-form P instead
    of the random start, followed by warmstart.LEARNED_EM EM iterations instead of
    admix_n_em_iters; where no model applies it falls back to the random start + EM.  Explicit
    init_q / init_p take precedence over the warm start.  stream_block keeps the genotypes in host
    memory and streams them in blocks of that many SNPs (cohorts larger than device memory).

    T = Float32 (np.float32 or "Float32"): the reference then holds and computes every array in
    Float32 (AdmixData{T}, structs.jl:9-91) for speed.  Here it selects the mixed form
    (ADMIX_FLAG_MIXED: FP32 cells and tensor-core Hessians with FP64 sums, QPs and state), which
    is faster than the FP64 form and more accurate than an all-Float32 run; the returned
    AdmixData holds Float32 arrays."""
    if T in (np.float32, "Float32"):
        flags |= N.ADMIX_FLAG_MIXED
    elif T not in (np.float64, float, "Float64"):
        raise NotImplementedError(f"T = {T!r}: Float64 and Float32 are supported")
    if not use_gpu:
        raise NotImplementedError("use_gpu=False is the reference's CPU path; this engine runs on the GPU")
    g = filename if isinstance(filename, (Genotypes, DeviceGenotypes)) else read_bed(filename)
    clusters = aims = None
    if sparsity is not None:
        if not isinstance(sparsity, (int, np.integer)):
            raise NotImplementedError("sparsity: an integer (the reference's vector of sparsities writes one file per "
                                      "value and does not run the likelihood engine)")
        in_memory = isinstance(filename, (Genotypes, DeviceGenotypes))
        if prefix is None and not in_memory:
            prefix = str(filename)[:-4]
        g, clusters, aims = _filter_skfr(g, K, int(sparsity), rng=rng, prefix=prefix, tries=skfr_tries,
                                         max_inner_iter=skfr_max_inner_iter, mode=skfr_mode,
                                         source=None if in_memory else filename, quiet=quiet)
    if not quiet:
        print(f"Loaded {g.I} samples and {g.J} SNPs")
    d = AdmixData(g.I, g.J, K, Q, rng=rng)
    d_cu, g_cu = _cu_admixture_base(d, g, g.I, g.J, flags=flags, stream_block=stream_block)
    try:
        learned = False
        if warm_start is not None and (init_q is None or init_p is None):
            from . import warmstart
            info = {}
            start = warmstart.learned_start(g, K, None if warm_start == "learned" else warm_start, info=info)
            if start is not None:
                if not quiet:
                    print("Starting from the learned warm start")
                learned = init_q is None and init_p is None
                init_q = start[0].T if init_q is None else init_q
                init_p = start[1].T if init_p is None else init_p
            elif not quiet:
                print(f"No warm start ({info.get('fallback')}); random start + EM")
        if init_q is None or init_p is None:
            init_em(d, g, admix_n_em_iters, d_cu=d_cu, g_cu=g_cu, quiet=quiet)
        if init_q is not None:
            d.q[:] = init_q
        if init_p is not None:
            d.p[:] = init_p
        if learned:   # the learned start's P is a closed-form step behind its Q: EM to pair them
            init_em(d, g, warmstart.LEARNED_EM, d_cu=d_cu, g_cu=g_cu, quiet=quiet)
        admixture_qn(d, g, admix_n_iter, admix_rtol, d_cu=d_cu, g_cu=g_cu, fix_q=fix_q, fix_p=fix_p,
                     verbose=verbose, progress_bar=progress_bar, quiet=quiet)
    finally:
        d_cu.close()
    if T in (np.float32, "Float32"):
        for name in ("x", "x_next", "x_next2", "x_tmp"):
            setattr(d, name, getattr(d, name).astype(np.float32))
    return d, clusters, aims
