"""Parity at the full sizes of the three correctness cohorts.

- C1 (I=1000, J=10000, K=3): the plain FP64 engine runs to convergence from the oracle's start
  (same random init + 5 EM) and ends on the oracle's optimum; its first QN iterations match the
  oracle's record by record.
- C2 (I=10000, J=100000, K=5, 0.5 % missing): at identical initial Q/P every pass of one
  iteration -- decode counts, log-likelihood, Q- and P-side gradient / Hessian, both EM
  half-steps, both SQP half-steps and one whole QN iteration -- against the oracle.
- C3 (I=100000, J=200000, K=12, P ~ Beta(0.5, 0.5) clipped to [1e-3, 1-1e-3]): the FP64 engine
  against the oracle on a subset of rows (512 individuals x all SNPs for the Q side, 256 SNPs x
  all individuals for the P side: each row of a sweep is independent of the others, so the
  subset runs the full reduction), and the mixed form against the FP64 engine at the full size,
  within the bounds the precision statement gives (Hessian 1.1e-2 of the row maximum, diagonal
  unbiased to 1e-6).

Tolerances as in test_gpu_parity: FP64 passes 1e-10 relative (row-wise for sums with
cancellation), SQP steps 1e-9 absolute with QP statuses equal to the oracle's QPs run on the
same sums, QN iteration log-likelihoods 1e-9 relative, converged log-likelihood 1e-6."""
import json

import numpy as np
import pytest

from conftest import rel_err

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-10


def _row_rel(a, b):
    a = a.reshape(a.shape[0], -1); b = b.reshape(b.shape[0], -1)
    scale = np.abs(b).max(axis=1, keepdims=True)
    return np.max(np.abs(a - b) / np.maximum(scale, 1e-300), axis=1)


def test_c1_full_size_converges_to_the_oracle_optimum(oa, orc):
    spec = oa.COHORTS["c1"]
    g, _, _ = oa.make_cohort(spec)
    x0 = oa.init_x(g.I, g.J, spec.K, 11)
    r = orc.OracleRun(g.data, g.I, g.J, spec.K, 3, x0)
    ll_em_o = r.init_em(5)
    d = oa.AdmixData(g.I, g.J, spec.K, 3, rng=11)
    assert np.array_equal(d.x, x0)
    with oa.CuAdmixData(d, g) as h:
        ll_em = oa.init_em(d, g, 5, d_cu=h, quiet=True)
        assert rel_err(np.array(ll_em), np.array(ll_em_o)) < 1e-10
        recs = oa.admixture_qn(d, g, 1000, 1e-7, d_cu=h, quiet=True)
    hist, conv = r.admixture_qn(1000, 1e-7)
    assert conv and recs[-1]["reldiff"] < 1e-7
    # the first iterations record for record (later ones drift apart at the rounding level of
    # the FP64 sums, amplified by the accept/reject test near convergence)
    for it in range(min(5, len(recs), len(hist))):
        got = [recs[it][k] for k in ("ll_prev", "ll_basic", "ll_qn", "ll_new")]
        assert rel_err(np.array(got), hist[it, :4]) < 1e-9, it
    assert rel_err(d.ll_new, r.ll_new) < 1e-6
    assert abs(len(recs) - len(hist)) <= max(3, len(hist) // 5), (len(recs), len(hist))


def test_c2_full_size_passes_match_oracle(oa, orc):
    spec = oa.COHORTS["c2"]
    g, _, _ = oa.make_cohort(spec)
    I, J, K = g.I, g.J, spec.K
    x0 = oa.init_x(I, J, K, 21)
    q, p = np.ascontiguousarray(x0[:I]), np.ascontiguousarray(x0[I:])
    d = oa.AdmixData(I, J, K, 3, rng=21)
    with oa.CuAdmixData(d, g) as h:
        h.upload(oa.X, x0)
        snp, ind = h.decode_counts()
        snp_o, ind_o = orc.decode_counts(g.data, I, J)
        assert np.array_equal(snp, snp_o) and np.array_equal(ind, ind_o)
        assert rel_err(h.loglik(oa.X), orc.loglik(g.data, I, J, K, q, p)) < FP64_TOL
        H, z = h.grad_hess_q(oa.X, oa.X)
        Ho, zo = orc.grad_hess_q(g.data, I, J, K, q, p)
        assert _row_rel(H, Ho).max() < FP64_TOL and _row_rel(z, zo).max() < FP64_TOL
        del H, Ho
        H, z = h.grad_hess_p(oa.X, oa.X)
        Hp, zp = orc.grad_hess_p(g.data, I, J, K, q, p)
        assert _row_rel(H, Hp).max() < FP64_TOL and _row_rel(z, zp).max() < FP64_TOL
        del H, Hp
        oa.em_q(h); oa.em_p(h)
        xn = h.download(oa.X_NEXT)
        assert rel_err(xn[:I], orc.em_q(g.data, I, J, K, q, p)) < FP64_TOL
        assert rel_err(xn[I:], orc.em_p(g.data, I, J, K, q, p)) < FP64_TOL
        # one EM-primed QN iteration: its four log-likelihoods and the iterate
        r = orc.OracleRun(g.data, I, J, K, 3, x0)
        r.init_em(2)
        d.x[:] = r.x
        d.ll_new = r.ll_new
        recs = oa.admixture_qn(d, g, 1, 0.0, d_cu=h, quiet=True)
        o = r.qn_iteration(1)
        for k in ("ll_prev", "ll_basic", "ll_qn", "ll_new"):
            assert rel_err(recs[0][k], o[k]) < 1e-9, (k, recs[0][k], o[k])
        assert np.max(np.abs(d.x - r.x)) < 1e-8


def test_c3_full_size_fp64_rows_match_oracle_and_mixed_within_bounds(oa, orc):
    import torch
    torch.cuda.set_device(0)
    spec = oa.COHORTS["c3"]
    qt, pt = oa.truth(spec)
    g = oa.genotypes_device(spec, qt, pt)
    I, J, K = g.I, g.J, spec.K
    d = oa.AdmixData(I, J, K, 3, rng=31)
    with oa.CuAdmixData(d, g) as h64:
        oa.init_em(d, g, 2, d_cu=h64, quiet=True)          # an EM-primed point, off the simplex
    x = d.x.copy()
    q, p = np.ascontiguousarray(x[:I]), np.ascontiguousarray(x[I:])
    report = {}
    h64 = oa.CuAdmixData(d, g)
    hmx = oa.CuAdmixData(d, g, flags=oa.ADMIX_FLAG_MIXED)
    try:
        for h in (h64, hmx):
            h.upload(oa.X, x)
        # --- Q side: FP64 rows vs the oracle on 512 individuals, mixed vs FP64 at full size
        H0, z0 = h64.grad_hess_q(oa.X, oa.X)
        nI = 512
        sub = np.ascontiguousarray(g.data[:, : nI // 4].cpu().numpy())
        Ho, zo = orc.grad_hess_q(sub, nI, J, K, np.ascontiguousarray(q[:nI]), p)
        assert _row_rel(H0[:nI], Ho).max() < FP64_TOL and _row_rel(z0[:nI], zo).max() < FP64_TOL
        H1, z1 = hmx.grad_hess_q(oa.X, oa.X)
        gq, hq = _row_rel(z1, z0), _row_rel(H1, H0)
        bq = (np.diagonal(H1, axis1=1, axis2=2) - np.diagonal(H0, axis1=1, axis2=2)) / np.diagonal(H0, axis1=1, axis2=2)
        report["q"] = {"grad_max": float(gq.max()), "hess_max": float(hq.max()),
                       "diag_bias_mean": float(bq.mean()), "diag_bias_maxabs": float(np.abs(bq).max())}
        del H0, H1, Ho
        # --- P side: FP64 rows vs the oracle on 256 SNPs, mixed vs FP64 at full size
        H0, z0 = h64.grad_hess_p(oa.X, oa.X)
        nJ = 256
        sub = np.ascontiguousarray(g.data[:nJ].cpu().numpy())
        Ho, zo = orc.grad_hess_p(sub, I, nJ, K, q, np.ascontiguousarray(p[:nJ]))
        assert _row_rel(H0[:nJ], Ho).max() < FP64_TOL and _row_rel(z0[:nJ], zo).max() < FP64_TOL
        H1, z1 = hmx.grad_hess_p(oa.X, oa.X)
        gp, hp = _row_rel(z1, z0), _row_rel(H1, H0)
        bp = (np.diagonal(H1, axis1=1, axis2=2) - np.diagonal(H0, axis1=1, axis2=2)) / np.diagonal(H0, axis1=1, axis2=2)
        report["p"] = {"grad_max": float(gp.max()), "hess_max": float(hp.max()),
                       "diag_bias_mean": float(bp.mean()), "diag_bias_maxabs": float(np.abs(bp).max())}
        del H0, H1, Ho
        # --- the mixed form's in-iteration log-likelihoods against the FP64 pass
        d.x[:] = x
        d.ll_new = h64.loglik(oa.X)
        recs = oa.admixture_qn(d, g, 2, 0.0, d_cu=hmx, quiet=True)
        lb, lq = hmx.loglik(oa.X_NEXT2), hmx.loglik(oa.X_TMP)
        report["loglik"] = {"basic_rel": (recs[-1]["ll_basic"] - lb) / abs(lb),
                            "qn_rel": (recs[-1]["ll_qn"] - lq) / abs(lq)}
    finally:
        h64.close(); hmx.close()
    print("C3_PRECISION " + json.dumps(report))
    assert report["q"]["grad_max"] < 1e-5 and report["p"]["grad_max"] < 1e-4
    assert report["q"]["hess_max"] < 1.1e-2 and report["p"]["hess_max"] < 1.1e-2
    assert abs(report["q"]["diag_bias_mean"]) < 1e-6 and abs(report["p"]["diag_bias_mean"]) < 1e-6
    assert abs(report["loglik"]["basic_rel"]) < 1e-8 and abs(report["loglik"]["qn_rel"]) < 1e-8
