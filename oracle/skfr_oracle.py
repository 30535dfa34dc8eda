"""CPU oracle of the SKFR AIM pre-selection (test infrastructure: only tests/ and the checker may
import it).

The reference selects ancestry-informative markers before run_admixture with sparse k-means via
feature ranking (driver.jl:56-69, _filter_SKFR driver.jl:80-101), calling the third-party package
SparseKmeansFeatureRanking.jl (Project.toml: compat "0.1", source not vendored with the
reference).  This is a restatement of the published method (Zhang, Lange and Xu, "Simple and
scalable sparse k-means clustering via feature ranking", NeurIPS 2020) with this project's own
choices where the package's are not available, stated here and used identically by the device
implementation (csrc/skfr.cu), which this oracle checks exactly:

- data: the genotype matrix imputed and standardised per SNP l (the package's ImputedSnpMatrix):
  mu_l, sigma_l = mean and population standard deviation of the non-missing dosages g in {0,1,2};
  x_il = (g_il - mu_l) / sigma_l, and 0 where g_il is missing or sigma_l = 0;
- seeding: k-means++ from a splitmix64 stream (seed): the first centre is individual
  floor(u I); each next one is drawn with probability proportional to the squared distance
  D_i to the nearest chosen centre (the first i whose running sum exceeds u * sum D); distances
  over all SNPs, summed in FP64 per slice of SLICE SNPs and then across slices in order; the
  starting clusters are the nearest centres (ties to the lower cluster);
- iteration ("global" mode): cluster means theta_kl over all SNPs (from exact integer sums),
  scores r_l = sum_k n_k theta_kl^2, the `sparsity` SNPs of largest score kept (ties to the lower
  index), centres zero elsewhere, each individual reassigned to
  argmin_k sum_{l kept} theta_kl^2 - 2 x_il theta_kl (ties to the lower cluster), the sum in FP64
  over each ASLICE kept SNPs in SNP order, two SNPs at a time (the terms of list positions 2r and
  2r+1 added first, an odd last position alone), the slice sums then added in order; stop when no
  assignment changes or after max_iter iterations;
- "local" mode: each cluster keeps its own `sparsity` SNPs by n_k theta_kl^2 and is scored on
  them; the AIMs are the union of the kept sets;
- objective: the within-cluster sum of squares with the sparse centres,
  sum_i ||x_i - theta_{c_i}||^2 over all SNPs; with tries > 1 the run of least objective wins
  (seeds continue the same splitmix64 stream).
"""
from __future__ import annotations

import numpy as np

SLICE = 1024          # SNPs per partial sum of the seeding distances
ASLICE = 1024         # kept SNPs per partial sum of the reassignment scores
MASK64 = (1 << 64) - 1


class SplitMix64:
    def __init__(self, seed: int):
        self.s = seed & MASK64

    def next(self) -> int:
        self.s = (self.s + 0x9E3779B97F4A7C15) & MASK64
        z = self.s
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & MASK64
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & MASK64
        return z ^ (z >> 31)

    def uniform(self) -> float:
        return (self.next() >> 11) * (2.0 ** -53)


def codes_of(data: np.ndarray, I: int) -> np.ndarray:
    """(J, ceil(I/4)) packed PLINK bytes -> (I, J) codes 0..3 (01 = missing)."""
    c = np.stack([(data >> (2 * s)) & 3 for s in range(4)], axis=2).reshape(data.shape[0], -1)[:, :I]
    return np.ascontiguousarray(c.T.astype(np.int8))


def snp_stats(codes: np.ndarray):
    """mu, a = 1/sigma, b = mu/sigma per SNP (a = b = 0 for sigma = 0 or no data) and the count of
    non-missing dosages, from the class counts."""
    n1 = (codes == 2).sum(0).astype(np.float64)   # code 10: dosage 1
    n2 = (codes == 3).sum(0).astype(np.float64)   # code 11: dosage 2
    n0 = (codes == 0).sum(0).astype(np.float64)
    n = n0 + n1 + n2
    with np.errstate(invalid="ignore", divide="ignore"):
        mu = (n1 + 2.0 * n2) / n
        var = (n1 + 4.0 * n2) / n - mu * mu
    ok = (n > 0) & (var > 0)
    sd = np.sqrt(np.where(ok, var, 1.0))
    a = np.where(ok, 1.0 / sd, 0.0)
    b = np.where(ok, mu * a, 0.0)
    return a, b, n


def x_table(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    """(J, 4) standardised value of each code: 00 -> -b, 01 (missing) -> 0, 10 -> a - b, 11 -> 2a - b."""
    t = np.zeros((a.shape[0], 4))
    t[:, 0] = -b
    t[:, 2] = a - b
    t[:, 3] = 2.0 * a - b
    return t


def dist_to(codes: np.ndarray, xt: np.ndarray, c: int) -> np.ndarray:
    """||x_i - x_c||^2 over all SNPs for every individual i, summed per SLICE SNPs in FP64 (SNP
    order), slices added in order."""
    I, J = codes.shape
    cols = np.arange(J)
    xc = xt[cols, codes[c]]
    total = np.zeros(I)
    for s0 in range(0, J, SLICE):
        part = np.zeros(I)
        for l in range(s0, min(J, s0 + SLICE)):
            d = xt[l, codes[:, l]] - xc[l]
            part += d * d
        total += part
    return total


def seed_clusters(codes: np.ndarray, xt: np.ndarray, K: int, rng: SplitMix64) -> np.ndarray:
    I = codes.shape[0]
    centers = [min(int(rng.uniform() * I), I - 1)]
    dk = [dist_to(codes, xt, centers[0])]
    D = dk[0].copy()
    for _ in range(1, K):
        tot = 0.0                   # FP64, in individual order
        for v in D:
            tot += v
        u = rng.uniform()
        if tot > 0.0:
            r = u * tot
            acc, pick = 0.0, I - 1
            for i in range(I):
                acc += D[i]
                if acc > r:
                    pick = i
                    break
        else:
            pick = min(int(u * I), I - 1)
        centers.append(pick)
        dk.append(dist_to(codes, xt, pick))
        D = np.minimum(D, dk[-1])
    return np.argmin(np.stack(dk, axis=1), axis=1).astype(np.int32)


def cluster_means(codes: np.ndarray, a, b, c: np.ndarray, K: int):
    """theta (K, J) from exact integer sums; n_k (K)."""
    I, J = codes.shape
    theta = np.zeros((K, J))
    nk = np.bincount(c, minlength=K).astype(np.float64)
    g = np.where(codes == 3, 2, np.where(codes == 2, 1, 0)).astype(np.int64)
    nm = (codes != 1).astype(np.int64)
    for k in range(K):
        m = c == k
        if nk[k] == 0:
            continue
        S = g[m].sum(0).astype(np.float64)         # sum of dosages of the non-missing members
        n = nm[m].sum(0).astype(np.float64)        # non-missing members
        theta[k] = (a * S - b * n) / nk[k]
    return theta, nk


def top_s(score: np.ndarray, s: int) -> np.ndarray:
    """indices of the s largest scores, ties to the lower index, returned in increasing order"""
    order = np.lexsort((np.arange(score.shape[0]), -score))
    return np.sort(order[: min(s, score.shape[0])])


def scores(codes: np.ndarray, xt: np.ndarray, theta: np.ndarray, kept: list[np.ndarray]) -> np.ndarray:
    """sc[i, k] = sum_{l in kept[k]} theta_kl^2 - 2 x_il theta_kl: FP64 sums over each ASLICE kept
    SNPs in SNP order, two list positions at a time (their terms added first), the slice sums
    added in order"""
    I = codes.shape[0]
    K = theta.shape[0]
    sc = np.zeros((I, K))

    def term(k, l):
        t = theta[k, l]
        return t * t - 2.0 * xt[l, codes[:, l]] * t

    for k in range(K):
        lst = kept[k]
        total = np.zeros(I)
        for p0 in range(0, len(lst), ASLICE):
            part = np.zeros(I)
            sl = lst[p0:p0 + ASLICE]
            for q in range(0, len(sl), 2):
                t = term(k, sl[q])
                if q + 1 < len(sl):
                    t = t + term(k, sl[q + 1])
                part += t
            total += part
        sc[:, k] = total
    return sc


def reassign(codes: np.ndarray, xt: np.ndarray, theta: np.ndarray, kept: list[np.ndarray]):
    """argmin_k of the scores (ties to the lower cluster) and the minimum"""
    sc = scores(codes, xt, theta, kept)
    c = np.argmin(sc, axis=1).astype(np.int32)
    return c, sc[np.arange(codes.shape[0]), c]


def skfr(data: np.ndarray, I: int, K: int, sparsity: int, *, mode: str = "global", max_iter: int = 50,
         tries: int = 1, seed: int = 0):
    """SKFR on packed genotypes (J, ceil(I/4)).  Returns (clusters (I,), aims (sorted), objective,
    iterations of the winning try)."""
    codes = codes_of(data, I)
    J = codes.shape[1]
    a, b, n = snp_stats(codes)
    xt = x_table(a, b)
    x2_total = float(np.sum(np.where(a > 0, n, 0.0)))     # sum_il x_il^2 (n_l per informative SNP)
    rng = SplitMix64(seed)
    best = None
    for _ in range(tries):
        c = seed_clusters(codes, xt, K, rng)
        it = 0
        for it in range(1, max_iter + 1):
            theta, nk = cluster_means(codes, a, b, c, K)
            if mode == "global":
                S = top_s((nk[:, None] * theta * theta).sum(0), sparsity)
                kept = [S] * K
            else:
                kept = [top_s(nk[k] * theta[k] * theta[k], sparsity) for k in range(K)]
            c_new, smin = reassign(codes, xt, theta, kept)
            if np.array_equal(c_new, c):
                break
            c = c_new
        # objective of the final assignment with its sparse centres
        theta, nk = cluster_means(codes, a, b, c, K)
        if mode == "global":
            kept = [top_s((nk[:, None] * theta * theta).sum(0), sparsity)] * K
        else:
            kept = [top_s(nk[k] * theta[k] * theta[k], sparsity) for k in range(K)]
        sc = scores(codes, xt, theta, kept)[np.arange(I), c]
        obj = x2_total
        for v in sc:
            obj += v
        aims = np.unique(np.concatenate(kept)) if mode != "global" else kept[0]
        if best is None or obj < best[2]:
            best = (c.copy(), aims, obj, it)
    return best
