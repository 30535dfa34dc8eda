"""GPU tests of the mixed-precision form (ADMIX_FLAG_MIXED): tensor-core BF16 Hessian with FP32
accumulation, gradients from two-part BF16 products, sums carried in FP64.  Tolerances against
the FP64 form on the same inputs: gradient 1e-5 and Hessian HESS_TOL, both relative to the largest
entry of each problem's row; Hessian diagonal unbiased to 1e-6; converged log-likelihood within
1e-6 relative of the FP64 solve."""
import numpy as np
import pytest

from conftest import rel_err

pytestmark = pytest.mark.gpu

GRAD_TOL = 1e-5
P_GRAD_TOL = 1e-5       # of sum_i |dz q_k|, the P-side gradient's term magnitude
# Every Hessian entry is a sum of non-negative terms (weights >= 0, factors in [0, 1]), so its
# relative error is at most the per-term one: the dithered BF16 weight (< 1 ulp, 2^-7), the
# BF16 pair product (2^-9; the diagonal's is corrected by its residual row) and the truncating
# FP32 accumulation (< 2^-23 per step, at most 4 * 256 steps per drained block): 2^-7 + 2^-9 +
# 1024 * 2^-23 = 1.0e-2.  Measured maxima at the sizes below: 3e-3.
HESS_TOL = 1.1e-2
DIAG_BIAS_TOL = 1e-6


def _row_rel(a, b):
    a = a.reshape(a.shape[0], -1); b = b.reshape(b.shape[0], -1)
    scale = np.abs(b).max(axis=1, keepdims=True)
    return float(np.max(np.abs(a - b) / np.maximum(scale, 1e-300)))


def _pair(oa, I, J, K, seed, cfg="c1"):
    spec = oa.COHORTS[cfg].scaled(I=I, J=J, K=K, seed=seed)
    g, _, _ = oa.make_cohort(spec)
    d = oa.AdmixData(I, J, K, 3, rng=seed + 1)
    h64 = oa.CuAdmixData(d, g)
    hmx = oa.CuAdmixData(d, g, flags=oa.ADMIX_FLAG_MIXED)
    for h in (h64, hmx):
        h.upload(oa.X, d.x)
    return g, d, h64, hmx


@pytest.mark.parametrize("K", [1, 2, 3, 5, 8, 9, 12, 16])
def test_mixed_q_sweep_matches_fp64(oa, K):
    g, d, h64, hmx = _pair(oa, I=389, J=3001, K=K, seed=40 + K)   # partial tile and partial chunk
    H0, z0 = h64.grad_hess_q(oa.X, oa.X)
    H1, z1 = hmx.grad_hess_q(oa.X, oa.X)
    assert np.all(np.isfinite(H1)) and np.all(np.isfinite(z1))
    assert _row_rel(z1, z0) < GRAD_TOL
    assert _row_rel(H1, H0) < HESS_TOL
    h64.close(); hmx.close()


def test_mixed_q_sweep_c2_size(oa):
    g, d, h64, hmx = _pair(oa, I=10_000, J=100_000, K=5, seed=2, cfg="c2")
    H0, z0 = h64.grad_hess_q(oa.X, oa.X)
    H1, z1 = hmx.grad_hess_q(oa.X, oa.X)
    assert _row_rel(z1, z0) < GRAD_TOL
    assert _row_rel(H1, H0) < HESS_TOL
    h64.close(); hmx.close()


@pytest.mark.parametrize("K", [3, 6])
def test_mixed_run_reaches_fp64_optimum(oa, K):
    spec = oa.COHORTS["c1"].scaled(I=800, J=6000, K=K, seed=70 + K)
    g, _, _ = oa.make_cohort(spec)
    finals = []
    for flags in (0, oa.ADMIX_FLAG_MIXED):
        d = oa.AdmixData(g.I, g.J, K, 3, rng=9)
        with oa.CuAdmixData(d, g, flags=flags) as h:
            oa.init_em(d, g, 5, d_cu=h, quiet=True)
            recs = oa.admixture_qn(d, g, 500, 1e-7, d_cu=h, quiet=True)
            assert recs[-1]["reldiff"] < 1e-7
            h.upload(oa.X, d.x)
            finals.append(h.loglik(oa.X))     # FP64 verifier
    assert rel_err(finals[1], finals[0]) < 1e-6


def _p_grad_scale(g, q, p):
    """sum_i |d l_ij / d p_jk| = sum_i nm |g/qp - (2-g)/(1-qp)| q_ik, the magnitude of the terms the
    P-side gradient adds up (J, K): the scale its rounding error is measured against, since the sum
    cancels and can be far smaller than its terms."""
    codes = np.stack([(g.data >> (2 * s)) & 3 for s in range(4)], axis=2).reshape(g.J, -1)[:, : g.I]
    gv = np.where(codes == 3, 2.0, np.where(codes == 2, 1.0, 0.0))
    nm = codes != 1
    qp = p @ q.T                                              # (J, I)
    dz = np.where(nm, gv / qp - (2 - gv) / (1 - qp), 0.0)
    return np.abs(dz) @ q                                     # (J, K)


@pytest.mark.parametrize("K", [1, 2, 3, 5, 8, 12, 16])
def test_mixed_p_sweep_matches_fp64(oa, K):
    """The P-side gradient is a cancelling sum (dz changes sign with the genotype): its error is
    bounded against the magnitude of its terms, P_GRAD_TOL * sum_i |dz q_k| (each term carries about
    2^-17 relative from the two-part BF16 split); the Hessian against each row's largest entry."""
    g, d, h64, hmx = _pair(oa, I=1037, J=517, K=K, seed=80 + K)   # partial individual chunk and SNP tile
    H0, z0 = h64.grad_hess_p(oa.X, oa.X)
    H1, z1 = hmx.grad_hess_p(oa.X, oa.X)
    assert np.all(np.isfinite(H1)) and np.all(np.isfinite(z1))
    scale = _p_grad_scale(g, d.x[: g.I], d.x[g.I:])
    assert np.max(np.abs(z1 - z0) / scale) < P_GRAD_TOL
    if K > 1:
        assert _row_rel(z1, z0) < 1e-4
    assert _row_rel(H1, H0) < HESS_TOL
    h64.close(); hmx.close()


def test_mixed_p_sweep_c2_size(oa):
    g, d, h64, hmx = _pair(oa, I=10_000, J=100_000, K=5, seed=3, cfg="c2")
    H0, z0 = h64.grad_hess_p(oa.X, oa.X)
    H1, z1 = hmx.grad_hess_p(oa.X, oa.X)
    assert _row_rel(z1, z0) < 1e-4
    assert _row_rel(H1, H0) < HESS_TOL
    h64.close(); hmx.close()


@pytest.mark.parametrize("side", ["q", "p"])
def test_mixed_hessian_diagonal_is_unbiased(oa, side):
    """The compensated diagonal.  The tensor core's FP32 accumulation truncates, so each chunk's
    diagonal is a fresh FP32 sum carried on in FP64; the B operand's diagonal products carry their
    BF16 rounding residual in extra rows; the A operand's weights are rounded to BF16 with dither
    (unbiased; round to nearest biased the diagonal by -3e-6 on the Q side and -4.5e-5 on the P
    side).  The mean signed relative error of all diagonal entries stays below 1e-6."""
    g, d, h64, hmx = _pair(oa, I=20_000, J=20_000, K=8, seed=5)
    H0, _ = getattr(h64, f"grad_hess_{side}")(oa.X, oa.X)
    H1, _ = getattr(hmx, f"grad_hess_{side}")(oa.X, oa.X)
    d0 = np.diagonal(H0, axis1=1, axis2=2); d1 = np.diagonal(H1, axis1=1, axis2=2)
    bias = float(np.mean((d1 - d0) / d0))
    assert abs(bias) < DIAG_BIAS_TOL, bias
    assert _row_rel(H1, H0) < HESS_TOL
    h64.close(); hmx.close()


@pytest.mark.parametrize("K,I,J", [(3, 777, 2001), (8, 1000, 3000), (12, 333, 1500)])
def test_mixed_loglik_in_iteration_matches_fp64_verifier(oa, K, I, J):
    """In the mixed form the iteration's log-likelihoods use FP32 cells with an FP64 reduction;
    they agree with the FP64 verifier (admix_loglik) to 1e-8 relative (FP32 rounding of q and p
    moves each cell's log by ~1e-7 relative, correlated along rows and columns)."""
    spec = oa.COHORTS["c1"].scaled(I=I, J=J, K=K, seed=90 + K)
    g, _, _ = oa.make_cohort(spec)
    d = oa.AdmixData(I, J, K, 3, rng=4)
    with oa.CuAdmixData(d, g, flags=oa.ADMIX_FLAG_MIXED) as h:
        oa.init_em(d, g, 2, d_cu=h, quiet=True)
        recs = oa.admixture_qn(d, g, 2, 0.0, d_cu=h, quiet=True)
        ll_basic = recs[-1]["ll_basic"]
        ll_qn = recs[-1]["ll_qn"]
        assert rel_err(ll_basic, h.loglik(oa.X_NEXT2)) < 1e-8
        assert rel_err(ll_qn, h.loglik(oa.X_TMP)) < 1e-8


@pytest.mark.parametrize("K", [3, 8])
def test_mixed_sweeps_match_fp64_after_em_priming(oa, K):
    """After EM priming sum_k q_k < 1 where genotypes are missing (the reference's EM Q-step
    divides by 2J); the mixed sweeps must still use the reference's 1 - qp, not sum_k q_k (1-p_k)."""
    spec = oa.COHORTS["c1"].scaled(I=700, J=5000, K=K, seed=60 + K, miss=0.05)
    g, _, _ = oa.make_cohort(spec)
    d = oa.AdmixData(g.I, g.J, K, 3, rng=2)
    with oa.CuAdmixData(d, g) as h:
        oa.init_em(d, g, 2, d_cu=h, quiet=True)
    assert np.abs(d.q.sum(0) - 1).max() > 1e-3          # the primed Q is off the simplex
    h64 = oa.CuAdmixData(d, g)
    hmx = oa.CuAdmixData(d, g, flags=oa.ADMIX_FLAG_MIXED)
    for h in (h64, hmx):
        h.upload(oa.X, d.x)
    for side in ("q", "p"):
        H0, z0 = getattr(h64, f"grad_hess_{side}")(oa.X, oa.X)
        H1, z1 = getattr(hmx, f"grad_hess_{side}")(oa.X, oa.X)
        assert _row_rel(z1, z0) < (GRAD_TOL if side == "q" else 1e-4), side
        assert _row_rel(H1, H0) < HESS_TOL, side
    h64.close(); hmx.close()


@pytest.mark.parametrize("K,I,J,miss", [(1, 100, 700, 0.0), (3, 777, 2001, 0.0), (8, 1000, 3000, 0.05),
                                        (12, 333, 1500, 0.02), (16, 515, 900, 0.01)])
def test_mixed_em_matches_fp64(oa, K, I, J, miss):
    """init_em! in the mixed form takes both EM half-steps' sums from FP32 cells added in FP64
    across chunks (the Q half from the tensor-core gradient sweep, the P half from the EM mode
    of the mixed P sweep); after 5 steps its iterates are within 1e-5 of the FP64 EM's and
    the FP64 log-likelihood of the result within 1e-6 relative."""
    spec = oa.COHORTS["c1"].scaled(I=I, J=J, K=K, seed=110 + K, miss=miss)
    g, _, _ = oa.make_cohort(spec)
    runs = []
    for flags in (0, oa.ADMIX_FLAG_MIXED):
        d = oa.AdmixData(I, J, K, 3, rng=7)
        with oa.CuAdmixData(d, g, flags=flags) as h:
            hist = oa.init_em(d, g, 5, d_cu=h, quiet=True)
        runs.append((d.x.copy(), d.ll_new, hist))
    (x0, ll0, h0), (x1, ll1, h1) = runs
    assert np.all(np.isfinite(x1))
    dx = float(np.abs(x1 - x0).max())
    assert dx < 1e-5, dx
    assert rel_err(ll1, ll0) < 1e-6, (ll1, ll0)
    assert rel_err(h1[-1], h0[-1]) < 1e-6, (h1[-1], h0[-1])


def test_run_admixture_float32_runs_the_mixed_form(oa):
    """run_admixture(T=Float32) selects the mixed form and returns Float32 arrays; from the same
    start it reaches the FP64 run's optimum (FP64 log-likelihood within 1e-6 relative; the
    stopping rule, reldiff < 1e-7 on the log-likelihood, resolves Q at I=600, J=4000 to a few
    1e-3, measured 2.4e-3)."""
    spec = oa.COHORTS["c1"].scaled(I=600, J=4000, K=3, seed=31)
    g, _, _ = oa.make_cohort(spec)
    d64, _, _ = oa.run_admixture(g, 3, rng=2, quiet=True)
    d32, _, _ = oa.run_admixture(g, 3, rng=2, quiet=True, T=np.float32)
    assert d32.q.dtype == np.float32 and d32.p.dtype == np.float32
    assert d32.q.shape == d64.q.shape and d32.p.shape == d64.p.shape
    assert rel_err(d32.ll_new, d64.ll_new) < 1e-6
    assert np.abs(d32.q - d64.q).max() < 1e-2


def test_timed_out_pipeline_wait_is_reported_and_the_handle_recovers(oa):
    """A bounded pipeline wait that runs out (admix_selftest_wait_timeout: an mbarrier that
    nothing completes, 1024 polls) fails the call with ADMIX_ERR_CUDA and clears the flag: the
    same handle's next EM and QN iterations succeed and equal a fresh handle's bit for bit."""
    from openadmixture_b200 import _native as N
    lib = N.admix_lib()
    spec = oa.COHORTS["c1"].scaled(I=300, J=1200, K=3, seed=5)
    g, _, _ = oa.make_cohort(spec)
    with oa.CuAdmixData(oa.AdmixData(g.I, g.J, 3, 3, rng=3), g) as h64:
        assert lib.admix_selftest_wait_timeout(h64.handle) == N.ADMIX_ERR_STATE
    lls = []
    for probe in (True, False):
        d = oa.AdmixData(g.I, g.J, 3, 3, rng=3)
        with oa.CuAdmixData(d, g, flags=oa.ADMIX_FLAG_MIXED) as h:
            if probe:
                assert lib.admix_selftest_wait_timeout(h.handle) == N.ADMIX_ERR_CUDA
                assert b"gave up" in lib.admix_last_error(h.handle)
            oa.init_em(d, g, 2, d_cu=h, quiet=True)
            recs = oa.admixture_qn(d, g, 3, 0.0, d_cu=h, quiet=True)
            lls.append(recs[-1]["ll_new"])
    assert lls[0] == lls[1]
