"""CPU tests of the warm start's checker (oracle/mlp_oracle.py) and host logic: the analytic
gradients against central finite differences, the sketch's definition, the closed-form P step
and the relabelling of a solve's clusters."""
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT / "oracle"))
import mlp_oracle as mo  # noqa: E402


def _tiny_net(rng, S, R, H, K):
    D = S + R
    return {"w1": rng.normal(0, 0.5, (D, H)), "b1": rng.normal(0, 0.1, H),
            "w2": rng.normal(0, 0.5, (H, H)), "b2": rng.normal(0, 0.1, H),
            "w3": rng.normal(0, 0.5, (H, K)), "b3": rng.normal(0, 0.1, K)}


def test_mlp_oracle_gradients_match_finite_differences():
    rng = np.random.default_rng(0)
    n, S, R, H, K = 7, 6, 3, 5, 4
    dos = rng.integers(0, 4, (n, S)).astype(np.int8)
    center = rng.uniform(0.2, 1.8, S)
    proj = rng.normal(0, 1, (n, R))
    tgt = rng.dirichlet(np.ones(K), n)
    params = _tiny_net(rng, S, R, H, K)
    loss, g = mo.loss_and_grads(params, dos, center, proj, tgt)
    assert np.isfinite(loss) and loss > 0
    eps = 1e-6
    for name, w in params.items():
        num = np.zeros_like(w)
        flat, nflat = w.reshape(-1), num.reshape(-1)
        for t in range(flat.size):
            old = flat[t]
            flat[t] = old + eps
            lp, _ = mo.loss_and_grads(params, dos, center, proj, tgt)
            flat[t] = old - eps
            lm, _ = mo.loss_and_grads(params, dos, center, proj, tgt)
            flat[t] = old
            nflat[t] = (lp - lm) / (2 * eps)
        # ReLU kinks are measure-zero for these draws; central differences are O(eps^2)
        assert np.allclose(g[name], num, rtol=1e-5, atol=1e-7), name


def test_softmax_output_is_on_the_simplex():
    rng = np.random.default_rng(1)
    params = _tiny_net(rng, 4, 2, 3, 5)
    dos = rng.integers(0, 4, (9, 4)).astype(np.int8)
    *_, p = mo.forward(params, dos, np.full(4, 1.0), rng.normal(0, 1, (9, 2)))
    assert np.allclose(p.sum(1), 1.0) and np.all(p > 0)


def test_sketch_definition(oa):
    spec = oa.COHORTS["c1"].scaled(I=203, J=300, seed=3)
    g, _, _ = oa.make_cohort(spec)
    snps = np.array([0, 5, 17, 150, 299], np.int32)
    freq, dos, proj = mo.sketch(g.data, g.I, snps, 8, 7)
    gg, nm = g.decode()                       # I x J
    assert np.array_equal(dos == 3, nm[:, snps] == 0)
    assert np.array_equal(np.where(dos == 3, 0, dos), (gg * nm)[:, snps].astype(np.int8))
    f = (gg * nm)[:, snps].sum(0) / (2 * nm[:, snps].sum(0))
    assert np.allclose(freq, f, rtol=1e-6)
    # the projection is linear in the standardised dosages: a sign flip of every hash bit negates it
    assert proj.shape == (203, 8) and np.isfinite(proj).all()
    assert abs(proj.mean()) < 0.5


def test_hash_matches_generator_constants():
    # splitmix-style finaliser: distinct, deterministic, full 64-bit outputs
    hs = {mo.hash3(7, s, 0) for s in range(1000)}
    assert len(hs) == 1000 and max(hs) < 1 << 64
    assert mo.hash3(7, 3, 0) == mo.hash3(7, 3, 0) != mo.hash3(8, 3, 0)


def test_warm_p_oracle_recovers_frequencies_from_the_true_q(oa):
    spec = oa.COHORTS["c1"].scaled(I=4000, J=50, K=2, seed=5, alpha=0.05)
    g, q, p = oa.make_cohort(spec)
    pw = mo.warm_p(g.data, g.I, 2, q)
    assert pw.shape == (50, 2)
    assert np.all((pw >= 1e-5) & (pw <= 1 - 1e-5))
    # with nearly unadmixed individuals the weighted allele frequency is close to the truth
    assert np.abs(pw - p).mean() < 0.05


def test_align_to_populations_undoes_a_label_permutation():
    pytest.importorskip("scipy")
    sys.path.insert(0, str(ROOT))
    from openadmixture_b200.warmstart import align_to_populations
    rng = np.random.default_rng(4)
    p_ref = rng.uniform(0.05, 0.95, (500, 5))
    q = rng.dirichlet(np.ones(5), 40)
    perm = np.array([3, 0, 4, 1, 2])
    q_solve, p_solve = q[:, perm], p_ref[:, perm] + rng.normal(0, 0.02, (500, 5))
    assert np.allclose(align_to_populations(q_solve, p_solve, p_ref), q)


def test_aligned_targets_are_row_major():
    from openadmixture_b200.warmstart import align_to_populations
    rng = np.random.default_rng(5)
    p_ref = rng.uniform(0.05, 0.95, (300, 4))
    q = rng.dirichlet(np.ones(4), 50)
    out = align_to_populations(q[:, [2, 0, 3, 1]], p_ref[:, [2, 0, 3, 1]], p_ref)
    assert out.flags["C_CONTIGUOUS"]
