"""Seeded synthetic admixed cohorts (the benchmark and test inputs).

Generator model: P_kj ~ Uniform(lo, hi) or Beta(a, a) clipped to [lo, hi];
Q_i ~ Dirichlet(alpha 1_K) (normalised Gamma draws); g_ij ~ Binomial(2, sum_k q_ki p_kj);
each cell missing (code 01) with probability ``miss``.  No public dataset is involved: the
cohort sizes and distributions below stand in for real data of the same shape.
"""
from __future__ import annotations

from dataclasses import dataclass, replace

import numpy as np

from . import _native as N
from .bed import DeviceGenotypes, Genotypes


@dataclass(frozen=True)
class CohortSpec:
    name: str
    I: int
    J: int
    K: int
    alpha: float = 0.5
    p_dist: str = "uniform"        # "uniform" or "beta"
    p_lo: float = 0.05
    p_hi: float = 0.95
    beta_a: float = 0.5
    miss: float = 0.01
    seed: int = 0
    p_seed: int = -1               # seed of P; -1: the cohort seed.  Cohorts sharing a p_seed share
                                   # their ancestral allele frequencies SNP by SNP (one "world").

    def scaled(self, I: int | None = None, J: int | None = None, K: int | None = None, **kw) -> "CohortSpec":
        return replace(self, I=I or self.I, J=J or self.J, K=K or self.K, **kw)


# p_seed of the synthetic "world" (shared ancestral allele frequencies) of the warm-start models
WARMSTART_WORLD = 777

COHORTS = {
    # plain method, CPU-runnable
    "c1": CohortSpec("c1", 1_000, 10_000, 3, alpha=0.5, miss=0.01),
    # plain method on GPU, drop-in (packed genotypes 250 MB)
    "c2": CohortSpec("c2", 10_000, 100_000, 5, alpha=0.5, miss=0.005),
    # precision form: extreme frequencies (packed genotypes 5 GB)
    "c3": CohortSpec("c3", 100_000, 200_000, 12, alpha=0.5, p_dist="beta", p_lo=1e-3, p_hi=1 - 1e-3,
                     beta_a=0.5, miss=0.01),
    # batching form
    "c4": CohortSpec("c4", 20_000, 50_000, 6, alpha=0.3, miss=0.01),
    # learned warm-start form (packed genotypes 25 GB); drawn from the ancestral frequencies the
    # shipped warm-start model was trained on (its training cohorts: I=20k, J=100k, seeds 1000-1049)
    "c5": CohortSpec("c5", 200_000, 500_000, 8, alpha=0.2, miss=0.01, p_seed=WARMSTART_WORLD),
}


def truth(spec: CohortSpec) -> tuple[np.ndarray, np.ndarray]:
    """Ground-truth (q_true, p_true) as numpy arrays of shape (I, K) and (J, K)
    (the memory of Julia's K x I and K x J column-major matrices)."""
    q = np.empty((spec.I, spec.K), dtype=np.float64)
    p = np.empty((spec.J, spec.K), dtype=np.float64)
    rc = N.synth_lib().syn_truth(spec.I, spec.J, spec.K, spec.seed, 0 if spec.p_dist == "uniform" else 1,
                                 spec.p_lo, spec.p_hi, spec.beta_a, spec.alpha, N.dptr(q), N.dptr(p))
    if rc != 0:
        raise ValueError(f"syn_truth failed for {spec}")
    if spec.p_seed >= 0 and spec.p_seed != spec.seed:
        q2 = np.empty((1, spec.K))
        rc = N.synth_lib().syn_truth(1, spec.J, spec.K, spec.p_seed, 0 if spec.p_dist == "uniform" else 1,
                                     spec.p_lo, spec.p_hi, spec.beta_a, spec.alpha, N.dptr(q2), N.dptr(p))
        if rc != 0:
            raise ValueError(f"syn_truth failed for {spec}")
    return q, p


def genotypes(spec: CohortSpec, q: np.ndarray, p: np.ndarray) -> Genotypes:
    """Packed SNP-major genotype bytes drawn on the host (OpenMP)."""
    Ib = (spec.I + 3) // 4
    data = np.empty((spec.J, Ib), dtype=np.uint8)
    rc = N.synth_lib().syn_bed_host(spec.I, spec.J, spec.K, spec.seed, spec.miss, N.dptr(q), N.dptr(p),
                                    N.u8ptr(data))
    if rc != 0:
        raise ValueError(f"syn_bed_host failed for {spec}")
    return Genotypes(data, spec.I, spec.J)


def genotypes_device(spec: CohortSpec, q: np.ndarray, p: np.ndarray) -> DeviceGenotypes:
    """The same genotype bytes as genotypes(), drawn on the current CUDA device (for cohorts too
    large to draw on the host quickly, e.g. 25 GB of packed genotypes)."""
    import torch
    dev = torch.device("cuda", torch.cuda.current_device())
    dq = torch.from_numpy(np.ascontiguousarray(q)).to(dev)
    dp = torch.from_numpy(np.ascontiguousarray(p)).to(dev)
    bed = torch.empty((spec.J, (spec.I + 3) // 4), dtype=torch.uint8, device=dev)
    rc = N.synth_lib().syn_bed_device(spec.I, spec.J, spec.K, spec.seed, spec.miss, dq.data_ptr(), dp.data_ptr(),
                                      bed.data_ptr(), torch.cuda.current_stream().cuda_stream)
    if rc != 0:
        raise RuntimeError(f"syn_bed_device failed for {spec}")
    torch.cuda.synchronize()
    return DeviceGenotypes(bed, spec.I, spec.J)


def make_cohort(spec: CohortSpec) -> tuple[Genotypes, np.ndarray, np.ndarray]:
    q, p = truth(spec)
    return genotypes(spec, q, p), q, p


def init_x(I: int, J: int, K: int, seed: int) -> np.ndarray:
    """Random starting point of AdmixData (structs.jl:107,128): shape (I+J, K), rows of the
    first I (the Q block) summing to one, the P block uniform on [0, 1)."""
    x = np.empty((I + J, K), dtype=np.float64)
    rc = N.synth_lib().syn_init_x(I, J, K, seed, N.dptr(x))
    if rc != 0:
        raise ValueError("syn_init_x failed")
    return x
