"""CPU tests of the SKFR oracle (oracle/skfr_oracle.py), the checker of the device's SKFR AIM
pre-selection: the splitmix64 stream against its published test vector, recovery of the
populations of a well-separated cohort, informative AIMs, the objective's bookkeeping against a
dense computation, and the fixed point at convergence."""
import sys
from pathlib import Path

import numpy as np
import pytest

sys.path.insert(0, str(Path(__file__).resolve().parents[1] / "oracle"))
import skfr_oracle as S  # noqa: E402


def _cohort(oa, I, J, K, seed, alpha=0.05):
    spec = oa.COHORTS["c1"].scaled(I=I, J=J, K=K, seed=seed, alpha=alpha)
    g, q, p = oa.make_cohort(spec)
    return g, q, p


def _purity(c, true, K):
    return sum(np.bincount(true[c == k], minlength=K).max() for k in range(K) if (c == k).any()) / len(c)


def test_splitmix64_matches_its_published_vector():
    r = S.SplitMix64(0)
    assert [r.next() for _ in range(3)] == [0xE220A8397B1DCDAF, 0x6E789E6AA1B965F4, 0x06C45D188009454F]
    u = S.SplitMix64(7).uniform()
    assert 0.0 <= u < 1.0


@pytest.mark.parametrize("mode", ["global", "local"])
def test_recovers_the_populations_of_a_separated_cohort(oa, mode):
    K = 3
    g, q, p = _cohort(oa, 300, 2000, K, seed=5)
    c, aims, obj, it = S.skfr(g.data, g.I, K, 200, mode=mode, tries=4, seed=11)
    assert _purity(c, np.argmax(q, axis=1), K) >= 0.94
    assert np.all(np.diff(aims) > 0) and aims.min() >= 0 and aims.max() < g.J
    if mode == "global":
        assert len(aims) == 200
    else:
        assert 200 <= len(aims) <= K * 200
    # the selected SNPs separate the populations better than the average SNP
    spread = p.max(1) - p.min(1)
    assert spread[aims].mean() > 1.3 * spread.mean()


def test_objective_is_the_sparse_within_cluster_sum_of_squares(oa):
    K = 3
    g, _, _ = _cohort(oa, 120, 900, K, seed=9, alpha=0.3)
    c, aims, obj, _ = S.skfr(g.data, g.I, K, 60, seed=3)
    codes = S.codes_of(g.data, g.I)
    a, b, _ = S.snp_stats(codes)
    X = S.x_table(a, b)[np.arange(g.J)[None, :], codes]          # dense (I, J) standardised
    theta = np.zeros((K, g.J))
    for k in range(K):
        theta[k, aims] = X[c == k][:, aims].mean(0)
    direct = float(((X - theta[c]) ** 2).sum())
    assert abs(obj - direct) <= 1e-9 * direct


def test_converged_assignment_is_a_fixed_point(oa):
    K = 4
    g, _, _ = _cohort(oa, 200, 1500, K, seed=13)
    c, aims, _, it = S.skfr(g.data, g.I, K, 150, seed=2, max_iter=100)
    assert it < 100
    codes = S.codes_of(g.data, g.I)
    a, b, _ = S.snp_stats(codes)
    xt = S.x_table(a, b)
    theta, nk = S.cluster_means(codes, a, b, c, K)
    kept = S.top_s((nk[:, None] * theta * theta).sum(0), 150)
    assert np.array_equal(kept, aims)
    c2, _ = S.reassign(codes, xt, theta, [kept] * K)
    assert np.array_equal(c2, c)


def test_standardisation_of_missing_and_monomorphic_snps():
    # SNP 0: dosages 0, 1, 2, missing; SNP 1: all 2 (monomorphic); 4 individuals
    codes = np.array([[0, 3], [2, 3], [3, 3], [1, 3]], dtype=np.int8)
    a, b, n = S.snp_stats(codes)
    assert n.tolist() == [3.0, 4.0]
    assert a[1] == 0.0 and b[1] == 0.0                       # no variance: the column is zero
    mu, sd = 1.0, np.sqrt(2.0 / 3.0)
    assert np.isclose(a[0], 1 / sd) and np.isclose(b[0], mu / sd)
    xt = S.x_table(a, b)
    assert xt[0, 1] == 0.0                                  # missing -> the (zero) mean
    assert np.allclose([xt[0, 0], xt[0, 2], xt[0, 3]], [-mu / sd, 0.0, mu / sd])
