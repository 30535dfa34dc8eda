"""Learned warm start: an MLP encoder that maps each individual's genotype sketch to a starting
Q on the simplex, and the closed-form P step that completes the start (csrc/mlp.cu).

It plugs into run_admixture's init_q / init_p (driver.jl:52-53,161-166,183-188): the predicted
Q and the derived P replace the random start and the EM priming.  The network is trained by
train() on (sketch, converged Q) pairs that this engine produced on cohorts drawn from the same
ancestral populations; the converged Q of each training cohort is relabelled to the
populations' order first (cluster labels of a solve are arbitrary).  All arithmetic runs in
libadmix kernels; torch only holds the device buffers.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from pathlib import Path

import numpy as np

from . import _native as N
from .bed import DeviceGenotypes, Genotypes
from .synth import WARMSTART_WORLD

MODEL_DIR = Path(__file__).resolve().parent / "models"
# ancestral-frequency seed (CohortSpec.p_seed) of the cohorts the shipped models were trained on
WORLD_SEED = WARMSTART_WORLD
# EM iterations run from the learned start before the QN loop.  The start's P is the closed-form
# frequency step of its Q, one half-step behind it; one EM iteration pairs them and, at
# I=200k, J=500k, K=8, saved one QN iteration (9 -> 8; 7.0 -> 6.75 s to convergence).
LEARNED_EM = 1


def _torch():
    import torch
    return torch


def _ptr(t) -> C.c_void_p:
    return C.c_void_p(t.data_ptr()) if t is not None else None


def _chk(rc: int) -> None:
    if rc != 0:
        raise N.AdmixError(rc, "warm-start kernel call failed")


def sketch_snps(J_panel: int, S: int = 4096, seed: int = 20240) -> np.ndarray:
    """The fixed sketch: S SNP indices drawn (sorted) from the first J_panel SNPs."""
    rng = np.random.default_rng(seed)
    return np.sort(rng.choice(J_panel, size=S, replace=False)).astype(np.int32)


@dataclass
class Sketch:
    dos: object      # int8 (n, S) device tensor, 3 = missing
    freq: object     # float32 (S,)
    proj: object     # float32 (n, R)

    @property
    def center(self):
        return 2.0 * self.freq


def sketch(g, snps: np.ndarray, R: int = 32, seed: int = 7) -> Sketch:
    """Sketch features of every individual of g (Genotypes or DeviceGenotypes)."""
    torch = _torch()
    dev = torch.device("cuda", torch.cuda.current_device())
    bed = g.data if isinstance(g, DeviceGenotypes) else torch.from_numpy(g.data).to(dev)
    S = int(len(snps))
    if S < 1 or int(np.min(snps)) < 0 or int(np.max(snps)) >= g.J:
        raise ValueError(f"sketch SNP indices must lie in [0, {g.J})")
    d_snps = torch.from_numpy(np.ascontiguousarray(snps, dtype=np.int32)).to(dev)
    freq = torch.empty(S, dtype=torch.float32, device=dev)
    dos = torch.empty((g.I, S), dtype=torch.int8, device=dev)
    proj = torch.empty((g.I, R), dtype=torch.float32, device=dev)
    _chk(N.admix_lib().admix_sketch(_ptr(bed), g.Ib, g.I, _ptr(d_snps), S, R, seed, _ptr(freq), _ptr(dos),
                                    _ptr(proj), C.c_void_p(torch.cuda.current_stream().cuda_stream)))
    torch.cuda.synchronize()
    return Sketch(dos, freq, proj)


class WarmStartMLP:
    """(S + R) -> H -> H -> K encoder; FP32 parameters on the device (stored as FP16)."""

    NAMES = ("w1", "b1", "w2", "b2", "w3", "b3")

    def __init__(self, S: int, R: int, K: int, H: int = 256, seed: int = 0, params: dict | None = None,
                 snps: np.ndarray | None = None, freq: np.ndarray | None = None):
        torch = _torch()
        self.S, self.R, self.K, self.H = S, R, K, H
        self.snps = None if snps is None else np.ascontiguousarray(snps, dtype=np.int32)
        # allele frequencies of the training cohorts at the sketch SNPs: the populations the model knows
        self.freq = None if freq is None else np.ascontiguousarray(freq, dtype=np.float32)
        if self.snps is not None and len(self.snps) != S:
            raise ValueError(f"{len(self.snps)} sketch SNPs for an input of S={S}")
        dev = torch.device("cuda", torch.cuda.current_device())
        if params is None:
            rng = np.random.default_rng(seed)
            D = S + R
            params = {"w1": rng.normal(0, np.sqrt(2.0 / D), (D, H)), "b1": np.zeros(H),
                      "w2": rng.normal(0, np.sqrt(2.0 / H), (H, H)), "b2": np.zeros(H),
                      "w3": rng.normal(0, np.sqrt(1.0 / H), (H, K)), "b3": np.zeros(K)}
        self.p = {k: torch.tensor(np.asarray(params[k], dtype=np.float32), device=dev) for k in self.NAMES}

    def net(self) -> N.MLPNet:
        p = self.p
        return N.MLPNet(self.S, self.R, self.H, self.K, p["w1"].data_ptr(), p["b1"].data_ptr(),
                        p["w2"].data_ptr(), p["b2"].data_ptr(), p["w3"].data_ptr(), p["b3"].data_ptr())

    def numpy_params(self) -> dict:
        return {k: v.detach().cpu().numpy().astype(np.float64) for k, v in self.p.items()}

    def save(self, path) -> None:
        """FP16 weights on disk (the deployed precision); the sketch definition alongside."""
        extra = {} if self.snps is None else {"snps": np.ascontiguousarray(self.snps, dtype=np.int32)}
        if self.freq is not None:
            extra["freq"] = np.ascontiguousarray(self.freq, dtype=np.float32)
        np.savez_compressed(path, S=self.S, R=self.R, K=self.K, H=self.H, **extra,
                            **{k: v.detach().cpu().numpy().astype(np.float16) for k, v in self.p.items()})

    @classmethod
    def load(cls, path) -> "WarmStartMLP":
        z = np.load(path)
        params = {k: z[k].astype(np.float32) for k in cls.NAMES}
        return cls(int(z["S"]), int(z["R"]), int(z["K"]), int(z["H"]), params=params,
                   snps=z["snps"] if "snps" in z.files else None,
                   freq=z["freq"] if "freq" in z.files else None)

    def forward(self, sk: Sketch, batch: int = 65536):
        """Class probabilities (n x K) of every individual of the sketch, as a device tensor."""
        torch = _torch()
        n = sk.dos.shape[0]
        dev = sk.dos.device
        out = torch.empty((n, self.K), dtype=torch.float32, device=dev)
        center = sk.center.contiguous()
        net = self.net()
        st = C.c_void_p(torch.cuda.current_stream().cuda_stream)
        for a in range(0, n, batch):
            b = min(n, a + batch)
            m = b - a
            h1 = torch.empty((m, self.H), dtype=torch.float32, device=dev)
            h2 = torch.empty_like(h1)
            logits = torch.empty((m, self.K), dtype=torch.float32, device=dev)
            _chk(N.admix_lib().admix_mlp_forward(C.byref(net), m, _ptr(sk.dos[a:b]), _ptr(center), _ptr(sk.proj[a:b]),
                                                 _ptr(h1), _ptr(h2), _ptr(logits), _ptr(out[a:b]), st))
        torch.cuda.synchronize()
        return out


def align_to_populations(q: np.ndarray, p: np.ndarray, p_ref: np.ndarray) -> np.ndarray:
    """Relabel a solve's clusters to the reference populations: the permutation maximising the
    summed correlation between its P columns and p_ref's (Hungarian assignment).  q is (I, K),
    p and p_ref (J, K); returns q with columns in the reference order."""
    from scipy.optimize import linear_sum_assignment
    K = q.shape[1]
    a = (p - p.mean(0)) / (p.std(0) + 1e-12)
    b = (p_ref - p_ref.mean(0)) / (p_ref.std(0) + 1e-12)
    corr = a.T @ b / p.shape[0]                      # corr[k_solve, k_ref]
    rows, cols = linear_sum_assignment(-corr)
    perm = np.empty(K, dtype=np.int64)
    perm[cols] = rows                                # reference column c <- solve column perm[c]
    return np.ascontiguousarray(q[:, perm])          # fancy indexing can return a column-major copy


def train(model: WarmStartMLP, data: list, epochs: int = 8, batch: int = 4096, lr: float = 1e-3,
          seed: int = 0, log=None) -> list[float]:
    """Adam on the mean cross-entropy between predicted and target Q.  `data` holds
    (Sketch, target) pairs, one per cohort, target an (n, K) device tensor.  Returns the mean
    loss of each epoch."""
    torch = _torch()
    lib = N.admix_lib()
    dev = model.p["w1"].device
    st = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    grads = {k: torch.zeros_like(v) for k, v in model.p.items()}
    m1 = {k: torch.zeros_like(v) for k, v in model.p.items()}
    m2 = {k: torch.zeros_like(v) for k, v in model.p.items()}
    G = N.MLPGrads(*[grads[k].data_ptr() for k in WarmStartMLP.NAMES])
    H, K = model.H, model.K
    h1 = torch.empty((batch, H), dtype=torch.float32, device=dev)
    h2, dh1, dh2 = torch.empty_like(h1), torch.empty_like(h1), torch.empty_like(h1)
    logits = torch.empty((batch, K), dtype=torch.float32, device=dev)
    probs, dl = torch.empty_like(logits), torch.empty_like(logits)
    loss = torch.zeros(1, dtype=torch.float32, device=dev)
    # the kernels take row-major rows through raw pointers
    data = [(Sketch(sk.dos.contiguous(), sk.freq.contiguous(), sk.proj.contiguous()),
             tgt.to(dtype=torch.float32).contiguous()) for sk, tgt in data]
    for sk, tgt in data:
        if tuple(tgt.shape) != (sk.dos.shape[0], K):
            raise ValueError(f"target shape {tuple(tgt.shape)} != ({sk.dos.shape[0]}, {K})")
    rng = np.random.default_rng(seed)
    step, hist = 0, []
    for ep in range(epochs):
        loss.zero_()
        seen = 0
        jobs = [(c, a) for c, (sk, _) in enumerate(data) for a in range(0, sk.dos.shape[0], batch)]
        for ji in rng.permutation(len(jobs)):
            c, a = jobs[ji]
            sk, tgt = data[c]
            b = min(sk.dos.shape[0], a + batch)
            n = b - a
            net = model.net()
            center = sk.center.contiguous()
            _chk(lib.admix_mlp_forward(C.byref(net), n, _ptr(sk.dos[a:b]), _ptr(center), _ptr(sk.proj[a:b]),
                                       _ptr(h1), _ptr(h2), _ptr(logits), _ptr(probs), st))
            _chk(lib.admix_mlp_backward(C.byref(net), C.byref(G), n, _ptr(sk.dos[a:b]), _ptr(center),
                                        _ptr(sk.proj[a:b]), _ptr(h1), _ptr(h2), _ptr(logits), _ptr(tgt[a:b]),
                                        _ptr(probs), _ptr(dl), _ptr(dh2), _ptr(dh1), _ptr(loss), st))
            step += 1
            for k in WarmStartMLP.NAMES:
                _chk(lib.admix_mlp_adam(_ptr(model.p[k]), _ptr(grads[k]), _ptr(m1[k]), _ptr(m2[k]),
                                        model.p[k].numel(), lr, 0.9, 0.999, 1e-8, step, st))
            seen += n
        torch.cuda.synchronize()
        hist.append(float(loss.item()) / seen)
        if log:
            log(f"epoch {ep + 1}: mean cross-entropy {hist[-1]:.4f}")
    return hist


def warm_p(g, q: np.ndarray) -> np.ndarray:
    """Closed-form starting P (J, K) from Q (I, K) on g's genotypes (csrc/mlp.cu k_warm_p)."""
    torch = _torch()
    dev = torch.device("cuda", torch.cuda.current_device())
    bed = g.data if isinstance(g, DeviceGenotypes) else torch.from_numpy(g.data).to(dev)
    dq = torch.from_numpy(np.ascontiguousarray(q, dtype=np.float64)).to(dev)
    dp = torch.empty((g.J, q.shape[1]), dtype=torch.float64, device=dev)
    _chk(N.admix_lib().admix_warm_p(_ptr(bed), g.Ib, g.I, g.J, q.shape[1], _ptr(dq), _ptr(dp),
                                    C.c_void_p(torch.cuda.current_stream().cuda_stream)))
    torch.cuda.synchronize()
    return dp.cpu().numpy()


# a cohort whose sketch-SNP allele frequencies correlate less than this with the training
# cohorts' comes from other ancestral populations than the model was trained on
MIN_FREQ_CORR = 0.9


def freq_corr(model: WarmStartMLP, sk: Sketch) -> float | None:
    """Pearson correlation of the cohort's sketch-SNP allele frequencies with the training
    cohorts' (None when the model does not record them)."""
    if model.freq is None:
        return None
    a = sk.freq.detach().cpu().numpy().astype(np.float64)
    b = model.freq.astype(np.float64)
    a, b = a - a.mean(), b - b.mean()
    den = np.sqrt((a * a).sum() * (b * b).sum())
    return float((a * b).sum() / den) if den > 0 else 0.0


def predict_start(model: WarmStartMLP, g, snps: np.ndarray | None = None, R: int = 32, seed: int = 7,
                  info: dict | None = None, check: bool = False):
    """(q, p) starting point for run_admixture's init_q / init_p: Q (I, K) from the encoder (rows
    floored at the projection's pseudocount 1e-5 and renormalised), P (J, K) from the closed-form
    step.  snps defaults to the sketch stored with the model.  With check=True the start is
    refused (None) when the cohort's sketch-SNP allele frequencies correlate less than
    MIN_FREQ_CORR with the training cohorts' (populations the model was not trained on); `info`
    receives the correlation and the decision."""
    if snps is None:
        snps = model.snps
    if snps is None:
        raise ValueError("the model carries no sketch SNP list; pass snps")
    sk = sketch(g, snps, R, seed)
    corr = freq_corr(model, sk)
    if info is not None:
        info["freq_corr"] = corr
        info["fallback"] = None
    if check and corr is not None and corr < MIN_FREQ_CORR:
        if info is not None:
            info["fallback"] = (f"sketch allele frequencies correlate {corr:.3f} with the training cohorts' "
                                f"(< {MIN_FREQ_CORR}): other ancestral populations")
        return None
    q = model.forward(sk).cpu().numpy().astype(np.float64)
    q = np.maximum(q, 1e-5)
    q /= q.sum(1, keepdims=True)
    return q, warm_p(g, q)


def default_model_path(K: int) -> Path:
    return MODEL_DIR / f"warmstart_k{K}.npz"


def load_default(K: int) -> WarmStartMLP | None:
    """The shipped model for K clusters, or None if there is none."""
    path = default_model_path(K)
    return WarmStartMLP.load(path) if path.exists() else None


def learned_start(g, K: int, model=None, info: dict | None = None):
    """(q, p) from the learned encoder, or None when no model applies -- none for K, the cohort
    has fewer SNPs than the sketch reaches, or its sketch-SNP allele frequencies do not match the
    populations the model was trained on: the caller then falls back to the random start + EM.
    `model` is a WarmStartMLP, a path to one, or None for the shipped model of K; `info` (a dict)
    receives the reason for a fallback and the frequency correlation."""
    if info is None:
        info = {}
    if model is None:
        model = load_default(K)
    elif not isinstance(model, WarmStartMLP):
        model = WarmStartMLP.load(model)
    if model is None or model.K != K:
        info["fallback"] = f"no model for K={K}"
        return None
    if model.snps is None or int(model.snps.max()) >= g.J:
        info["fallback"] = f"the model's sketch reaches beyond the cohort's {g.J} SNPs"
        return None
    return predict_start(model, g, info=info, check=True)


def run_to_target(g, K: int, *, flags: int = 0, start=None, em: int = 5, rtol: float = 1e-7, target=None,
                  max_iter: int = 1000, extra_iter: int = 10, rng: int = 1, em_after_start: int | None = None) -> dict:
    """Solve g from the random start + `em` EM iterations (start=None) or from start=(q, p) +
    em_after_start EM iterations (default LEARNED_EM), and
    record when the iteration log-likelihood first reached `target`.  Returns x (I+J, K), the
    FP64 log-likelihood of the result, the QN iterations run, the seconds from the start
    (initialisation included) and, when target is given, iterations_to_target /
    seconds_to_target (None if never reached), and the trace (iteration, log-likelihood, seconds)
    of every QN iteration.  The run stops at relative change < rtol once
    the target (if any) has been reached, or extra_iter iterations after that."""
    import time
    from . import admixture as A
    torch = _torch()
    lib = N.admix_lib()
    d = A.AdmixData(g.I, g.J, K, 3, rng=rng)
    with A.CuAdmixData(d, g, flags=flags) as h:
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        if start is None:
            h.upload(A.X, d.x)
            hist = (C.c_double * max(em, 1))()
            h._chk(lib.admix_init_em(h.handle, em, hist))
        else:
            h.upload_qp(A.X, q=start[0], p=start[1])
            n_em = LEARNED_EM if em_after_start is None else em_after_start
            if n_em > 0:
                hist = (C.c_double * n_em)()
                h._chk(lib.admix_init_em(h.handle, n_em, hist))
            else:
                h.set_ll(h.loglik(A.X))
        info = N.IterInfo()
        t_hit = it_hit = conv_at = None
        trace = []
        it = 0
        for it in range(1, max_iter + 1):
            h._chk(lib.admix_qn_iteration(h.handle, it, C.byref(info)))
            trace.append((it, info.ll_new, time.perf_counter() - t0))
            if target is not None and t_hit is None and info.ll_new >= target:
                t_hit, it_hit = time.perf_counter() - t0, it
            if info.reldiff < rtol:
                conv_at = conv_at or it
                # past convergence, keep going a little while the target is still unreached
                if target is None or t_hit is not None or it >= conv_at + extra_iter:
                    break
        secs = time.perf_counter() - t0
        x = h.download(A.X)
        ll = h.loglik(A.X)
    return {"x": x, "ll": ll, "iterations": it, "seconds": secs, "iterations_to_target": it_hit,
            "seconds_to_target": t_hit, "trace": trace}
