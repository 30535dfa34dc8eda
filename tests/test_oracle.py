"""CPU tests of the oracle (oracle/admix_oracle.c): against the golden fixtures of the
independent numpy restatement, and against mathematical known answers (derivatives, KKT,
projection optimality, EM monotonicity)."""
import itertools
import math

import numpy as np
import pytest

from conftest import rel_err


def _qp_split(x, I):
    return np.ascontiguousarray(x[:I]), np.ascontiguousarray(x[I:])


def test_decode_counts_bit_exact(orc, golden):
    I, J = int(golden["I"]), int(golden["J"])
    snp, ind = orc.decode_counts(golden["bed"], I, J)
    assert np.array_equal(snp, golden["miss_snp"])
    assert np.array_equal(ind, golden["miss_ind"])


def test_loglik_matches_golden(orc, golden):
    I, J, K = int(golden["I"]), int(golden["J"]), int(golden["K"])
    q, p = _qp_split(golden["x0"], I)
    ll = orc.loglik(golden["bed"], I, J, K, q, p)
    assert rel_err(ll, golden["ll_x0"]) < 1e-12


def test_em_matches_golden(orc, golden):
    I, J, K = int(golden["I"]), int(golden["J"]), int(golden["K"])
    q, p = _qp_split(golden["x0"], I)
    assert rel_err(orc.em_q(golden["bed"], I, J, K, q, p), golden["q_em"]) < 1e-12
    assert rel_err(orc.em_p(golden["bed"], I, J, K, q, p), golden["p_em"]) < 1e-12


def test_grad_hess_matches_golden(orc, golden):
    I, J, K = int(golden["I"]), int(golden["J"]), int(golden["K"])
    q, p = np.ascontiguousarray(golden["q_em"]), np.ascontiguousarray(golden["p_em"])
    H, z = orc.grad_hess_q(golden["bed"], I, J, K, q, p)
    assert rel_err(H, golden["XtX_q"]) < 1e-12
    assert rel_err(z, golden["Xtz_q"], scale=np.abs(golden["Xtz_q"]).max()) < 1e-12
    H, z = orc.grad_hess_p(golden["bed"], I, J, K, q, p)
    assert rel_err(H, golden["XtX_p"]) < 1e-12
    assert rel_err(z, golden["Xtz_p"], scale=np.abs(golden["Xtz_p"]).max()) < 1e-12


def test_sqp_updates_match_golden(orc, golden):
    I, J, K = int(golden["I"]), int(golden["J"]), int(golden["K"])
    x = np.vstack([golden["q_em"], golden["p_em"]])
    r = orc.OracleRun(golden["bed"], I, J, K, 3, x)
    stq = r.update_q(False)
    assert np.array_equal(stq, golden["st_q"])
    assert rel_err(r.x_next[:I], golden["q_sqp"], scale=1.0) < 1e-12
    stp = r.update_p(False)
    assert np.array_equal(stp, golden["st_p"])
    assert rel_err(r.x_next[I:], golden["p_sqp"], scale=1.0) < 1e-12


def test_qn_iterations_match_golden(orc, golden):
    I, J, K = int(golden["I"]), int(golden["J"]), int(golden["K"])
    x = np.vstack([golden["q_em"], golden["p_em"]])
    r = orc.OracleRun(golden["bed"], I, J, K, 3, x)
    r.ll_new = float(golden["ll_em"])
    for it in range(1, 5):
        info = r.qn_iteration(it)
        want = golden["qn_info"][it - 1]
        got = [info[k] for k in ("ll_prev", "ll_basic", "ll_qn", "ll_new")]
        assert rel_err(got, want[:4]) < 1e-9, (it, got, want)
    assert rel_err(r.x, golden["x_qn4"], scale=1.0) < 1e-7


# ---------------------------------------------------------------- known-answer properties

def _tiny(oa, I=61, J=83, K=3, seed=5):
    spec = oa.COHORTS["c1"].scaled(I=I, J=J, K=K, seed=seed)
    g, _, _ = oa.make_cohort(spec)
    x = oa.init_x(I, J, K, seed + 1)
    return g, x


def test_p_gradient_and_hessian_are_derivatives(oa, orc):
    """Xtz_p = dL/dp and XtX_p = -d2L/dp2 (loops.jl:923-950 are the exact derivatives)."""
    g, x = _tiny(oa)
    I, J, K = g.I, g.J, 3
    q, p = _qp_split(x, I)
    p = np.clip(p, 0.1, 0.9)
    H, z = orc.grad_hess_p(g.data, I, J, K, q, p)
    h = 1e-6
    for j, k in [(0, 0), (5, 2), (40, 1)]:
        pp, pm = p.copy(), p.copy()
        pp[j, k] += h; pm[j, k] -= h
        fd = (orc.loglik(g.data, I, J, K, q, pp) - orc.loglik(g.data, I, J, K, q, pm)) / (2 * h)
        assert abs(fd - z[j, k]) < 1e-5 * max(1.0, abs(z[j, k]))
        _, zp = orc.grad_hess_p(g.data, I, J, K, q, pp)
        _, zm = orc.grad_hess_p(g.data, I, J, K, q, pm)
        fd2 = (zp[j] - zm[j]) / (2 * h)
        assert np.allclose(-fd2, H[j, :, k], rtol=1e-5, atol=1e-5)


def test_q_gradient_is_derivative_up_to_a_constant(oa, orc):
    """Xtz_q differs from dL/dq by sum_j nm (2-g)/(1-qp) in every component (loops.jl:885-886),
    so both give the same directional derivative along the simplex."""
    g, x = _tiny(oa)
    I, J, K = g.I, g.J, 3
    q, p = _qp_split(x, I)
    H, z = orc.grad_hess_q(g.data, I, J, K, q, p)
    h = 1e-6
    for i in (0, 7, 60):
        fd = np.empty(K)
        for k in range(K):
            qp_, qm = q.copy(), q.copy()
            qp_[i, k] += h; qm[i, k] -= h
            fd[k] = (orc.loglik(g.data, I, J, K, qp_, p) - orc.loglik(g.data, I, J, K, qm, p)) / (2 * h)
        diff = z[i] - fd
        assert np.ptp(diff) < 1e-5 * max(1.0, np.abs(z[i]).max())
        # Hessian identity on the simplex: XtX_q q_i = Xtz_q when sum(q_i) = 1
        assert np.allclose(H[i] @ q[i], z[i], rtol=1e-12)


def test_em_is_monotone(oa, orc):
    g, x = _tiny(oa, I=120, J=300, K=4)
    r = orc.OracleRun(g.data, g.I, g.J, 4, 3, x)
    hist = [r.loglik(r.x)] + r.init_em(6)
    assert all(b > a for a, b in zip(hist, hist[1:]))


def _brute_qp(H, z, x, simplex):
    """min 1/2 d'Hd - z'd  s.t. 0 <= x+d <= 1 (and sum(x+d) = 1): enumerate active sets."""
    K = len(x)
    best, bestv = None, math.inf
    for act in itertools.product((0, 1, 2), repeat=K):   # 0 free, 1 at lower, 2 at upper
        fixed = {k: (-x[k] if a == 1 else 1 - x[k]) for k, a in enumerate(act) if a}
        free = [k for k in range(K) if not act[k]]
        d = np.zeros(K)
        for k, v in fixed.items():
            d[k] = v
        if free:
            Hf = H[np.ix_(free, free)]
            rhs = z[free] - H[np.ix_(free, list(fixed))] @ np.array(list(fixed.values())) if fixed else z[free]
            if simplex:
                n = len(free)
                M = np.zeros((n + 1, n + 1)); M[:n, :n] = Hf; M[:n, n] = 1; M[n, :n] = 1
                b = np.append(rhs, 1 - x.sum() - sum(fixed.values()))
                try:
                    sol = np.linalg.solve(M, b)
                except np.linalg.LinAlgError:
                    continue
                d[free] = sol[:n]
            else:
                d[free] = np.linalg.solve(Hf, rhs)
        elif simplex and abs(x.sum() + d.sum() - 1) > 1e-9:
            continue
        if np.any(x + d < -1e-9) or np.any(x + d > 1 + 1e-9):
            continue
        if simplex and abs((x + d).sum() - 1) > 1e-9:
            continue
        v = 0.5 * d @ H @ d - z @ d
        if v < bestv:
            best, bestv = d, v
    return best


@pytest.mark.parametrize("simplex", [False, True])
@pytest.mark.parametrize("seed", range(6))
def test_qp_matches_brute_force_active_set(orc, simplex, seed):
    rng = np.random.default_rng(seed)
    K = 3
    A = rng.normal(size=(K, K)); H = A @ A.T + 0.5 * np.eye(K)
    x = rng.dirichlet(np.ones(K)) if simplex else rng.uniform(0.05, 0.95, K)
    z = rng.normal(scale=2.0, size=K)
    vt = orc.vt_ones(K)
    tab = orc.create_tableau(H, -z, x, vt, simplex)
    it, delta, _ = orc.quadratic_program(tab, x, K, 1 if simplex else 0)
    assert it > 0
    want = _brute_qp(H, z, x, simplex)
    # the solver's bound slack is 1e-5 (qp.jl:184)
    assert np.allclose(delta, want, atol=2e-5), (delta, want)


def test_qp_interior_is_newton_step(orc):
    K = 4
    rng = np.random.default_rng(1)
    A = rng.normal(size=(K, K)); H = A @ A.T + K * np.eye(K)
    x = np.full(K, 0.5)
    z = 0.01 * rng.normal(size=K)
    tab = orc.create_tableau(H, -z, x, orc.vt_ones(K), False)
    it, delta, _ = orc.quadratic_program(tab, x, K, 0)
    assert it == 1
    assert np.allclose(delta, np.linalg.solve(H, z), rtol=1e-12, atol=1e-15)


def test_qp_fails_on_non_positive_pivot(orc):
    K = 3
    H = np.diag([1.0, -1.0, 1.0])
    tab = orc.create_tableau(H, np.zeros(K), np.full(K, 0.5), orc.vt_ones(K), False)
    it, delta, _ = orc.quadratic_program(tab, np.full(K, 0.5), K, 0)
    assert it == 0 and np.all(delta == 0)


@pytest.mark.parametrize("mu_mode", [0, 1])
def test_qp_mu_mode_does_not_change_solution(orc, mu_mode):
    """Adding mu 1 1' to H leaves the simplex-constrained solution unchanged (qp.jl:46-66)."""
    rng = np.random.default_rng(3)
    K = 5
    A = rng.normal(size=(K, K)); H = A @ A.T + np.eye(K)
    x = rng.dirichlet(np.ones(K)); z = rng.normal(size=K)
    vt = orc.vt_ones(K)
    d0 = orc.quadratic_program(orc.create_tableau(H, -z, x, vt, True, 0), x, K, 1)[1]
    d1 = orc.quadratic_program(orc.create_tableau(H, -z, x, vt, True, mu_mode), x, K, 1)[1]
    assert np.allclose(d0, d1, atol=1e-10)


@pytest.mark.parametrize("K", [1, 2, 3, 4, 7, 12, 16])
def test_vt_is_orthogonal_with_constant_first_row(orc, K):
    v = orc.vt_ones(K).T          # Julia V'
    assert np.allclose(v @ v.T, np.eye(K), atol=1e-14)
    assert np.allclose(np.abs(v[0]), 1 / math.sqrt(K), atol=1e-15)


@pytest.mark.parametrize("K", [2, 3, 5, 8, 12])
def test_project_q_is_euclidean_projection(orc, K):
    rng = np.random.default_rng(K)
    pc = 1e-5
    for _ in range(20):
        b = rng.normal(scale=0.7, size=K) + 1.0 / K
        out = orc.project_q1(b)
        assert abs(out.sum() - 1.0) < 1e-14
        assert np.all(out >= pc - 1e-18)
        # bisection on the threshold of the shifted problem
        lo, hi = -10.0, 10.0
        for _ in range(200):
            t = 0.5 * (lo + hi)
            s = np.maximum(b - pc - t, 0).sum()
            lo, hi = (t, hi) if s > 1 - K * pc else (lo, t)
        assert np.allclose(out, np.maximum(b - pc - lo, 0) + pc, atol=1e-12)


def test_project_p_clamps(orc):
    b = np.array([-1.0, 0.0, 1e-6, 0.5, 1.0, 2.0])
    assert np.array_equal(orc.project_p(b), np.array([1e-5, 1e-5, 1e-5, 0.5, 1 - 1e-5, 1 - 1e-5]))


def test_oracle_run_converges(oa, orc):
    g, x = _tiny(oa, I=150, J=900, K=3, seed=9)
    r = orc.OracleRun(g.data, g.I, g.J, 3, 3, x)
    em = r.init_em(5)
    hist, conv = r.admixture_qn(300, 1e-7)
    assert conv
    assert r.ll_new > em[-1]
    assert hist[-1, 4] < 1e-7


def test_loglik_tiling_matches_plain_sum(oa, orc):
    """The reference's tile tree (loops.jl:223-258) only changes the summation order."""
    g, x = _tiny(oa, I=333, J=250, K=4, seed=2)
    q, p = _qp_split(x, g.I)
    gg, nm = g.decode()
    qp = q @ p.T
    want = np.sum(nm * (gg * np.log(qp) + (2 - gg) * np.log(1 - qp)))
    assert rel_err(orc.loglik(g.data, g.I, g.J, 4, q, p), want) < 1e-12


def test_oracle_fix_p_keeps_p_and_raises_loglik(oa, orc):
    """fix_p (supervised projection analysis): P is carried over unchanged, Q is fitted, and the
    log-likelihood never decreases (algorithms_outer.jl:98-116)."""
    spec = oa.COHORTS["c1"].scaled(I=150, J=600, K=3, seed=17)
    g, q, p = oa.make_cohort(spec)
    x0 = oa.init_x(g.I, g.J, 3, 2)
    x0[g.I:] = p                                       # the true P, fixed
    r = orc.OracleRun(g.data, g.I, g.J, 3, 3, x0, fix_p=True)
    r.ll_new = float("nan")
    lls = []
    for it in range(1, 8):
        lls.append(r.qn_iteration(it)["ll_new"])
    assert np.all(np.diff(lls) >= -1e-9 * abs(lls[0]))
    assert np.max(np.abs(r.x[g.I:] - np.clip(p, 1e-5, 1 - 1e-5))) < 1e-12
    assert np.max(np.abs(r.x[: g.I] - x0[: g.I])) > 1e-2


def test_qp_batch_reproduces_update_q_and_update_p(oa, orc):
    """oracle.qp_batch (the QP loop of update_q! / update_p! on given sums) returns the statuses
    and steps of the oracle's own updates when given the oracle's own sums."""
    spec = oa.COHORTS["c1"].scaled(I=120, J=700, K=4, seed=5)
    g, _, _ = oa.make_cohort(spec)
    x0 = oa.init_x(g.I, g.J, 4, 9)
    r = orc.OracleRun(g.data, g.I, g.J, 4, 3, x0)
    r.init_em(2)
    q, p = np.ascontiguousarray(r.x[: g.I]), np.ascontiguousarray(r.x[g.I:])
    st = r.update_q(False)
    H, z = orc.grad_hess_q(g.data, g.I, g.J, 4, q, p)
    st2, dq = orc.qp_batch(H, z, q, True)
    assert np.array_equal(st, st2)
    assert np.array_equal(dq, r.x_tmp[: g.I])
    st = r.update_p(False)
    qn = np.ascontiguousarray(r.x_next[: g.I])
    H, z = orc.grad_hess_p(g.data, g.I, g.J, 4, qn, p)
    st2, dp = orc.qp_batch(H, z, p, False)
    assert np.array_equal(st, st2)
    assert np.array_equal(dp, r.x_tmp[g.I:])


def _lbqn_numpy(U, V, x, x1, x2, it, Q):
    """update_UV_LBQN! + update_QN_LBQN! (quasi_newton.jl:15-58) in numpy, columns of U, V as rows."""
    for i in range(min(it, Q) - 1, 0, -1):
        U[i] = U[i - 1]; V[i] = V[i - 1]
    U[0] = x1 - x
    V[0] = (x2 - x1) - U[0]
    m = min(it, Q)
    u, v = U[0], V[0]
    gamma = np.dot(u, v) / np.dot(v, v)
    xq = u.copy()
    alpha = np.zeros(m)
    for i in range(m):
        rho = 1.0 / np.dot(V[i], V[i])
        alpha[i] = rho * np.dot(V[i], xq)
        xq = xq - alpha[i] * V[i]
    xr = gamma * xq
    for i in range(m):
        xr = xr + alpha[i] * U[i]
    return x - xr


def test_lbqn_step_matches_numpy_restatement_and_converges(oa, orc):
    """mode = :LBQN in the oracle: each iteration's QN point (before projection) is the numpy
    restatement's, and the run reaches the :ZAL run's optimum."""
    spec = oa.COHORTS["c1"].scaled(I=150, J=800, K=3, seed=12)
    g, _, _ = oa.make_cohort(spec)
    x0 = oa.init_x(g.I, g.J, 3, 4)
    Q = 3
    r = orc.OracleRun(g.data, g.I, g.J, 3, Q, x0, mode="LBQN")
    r.init_em(3)
    n = (g.I + g.J) * 3
    U = np.zeros((Q, n)); V = np.zeros((Q, n))
    for it in range(1, 7):
        xb = r.x.copy().ravel()
        r.qn_iteration(it)
        want = _lbqn_numpy(U, V, xb, r.x_next.ravel(), r.x_next2.ravel(), it, Q).reshape(-1, 3)
        want[: g.I] = np.array([orc.project_q1(row) for row in want[: g.I]])
        want[g.I:] = orc.project_p(want[g.I:])
        assert np.max(np.abs(r.x_tmp - want)) < 1e-12, it
    hist, conv = r.admixture_qn(1000, 1e-7, iter_offset=6)
    assert conv
    rz = orc.OracleRun(g.data, g.I, g.J, 3, Q, x0)
    rz.init_em(3)
    hz, cz = rz.admixture_qn(1000, 1e-7)
    assert cz and abs(r.ll_new - rz.ll_new) < 1e-6 * abs(rz.ll_new)


def test_mean_imputed_loops(oa, orc):
    """AdmixData(...; skipmissing=false): the missing genotype is the SNP's mean dosage g.mu[j]
    (loops.jl:365-383,589-608,679-698,840-865,896-921).  Known answers: mu is the mean over the
    non-missing genotypes; without missing genotypes the two loop families agree; the imputed
    loglik equals the plain formula evaluated on the imputed dosage matrix; Xtz_p / XtX_p are its
    first / negated second p-derivatives; EM stays monotone."""
    g, x = _tiny(oa)
    I, J, K = g.I, g.J, 3
    q, p = _qp_split(x, I)
    codes = np.stack([(g.data >> (2 * s)) & 3 for s in range(4)], axis=2).reshape(J, -1)[:, :I]
    dose = np.where(codes == 3, 2.0, np.where(codes == 2, 1.0, 0.0))
    nm = codes != 1
    mu = orc.snp_means(g.data, I, J)
    assert np.allclose(mu, (dose * nm).sum(1) / nm.sum(1), rtol=1e-14)
    gi = np.where(nm, dose, mu[:, None])                      # (J, I) imputed dosages
    qp = p @ q.T                                              # (J, I)
    want = float(np.sum(gi * np.log(qp) + (2 - gi) * np.log(1 - qp)))
    assert rel_err(orc.loglik(g.data, I, J, K, q, p, mu=mu), want) < 1e-11
    full = g.data.copy()                                      # every missing code 01 replaced by 00
    for s in range(4):
        c = (full >> (2 * s)) & 3
        full = np.where(c == 1, full & ~np.uint8(3 << (2 * s)), full).astype(np.uint8)
    mu_f = orc.snp_means(full, I, J)
    assert rel_err(orc.loglik(full, I, J, K, q, p, mu=mu_f), orc.loglik(full, I, J, K, q, p)) < 1e-13
    H0, z0 = orc.grad_hess_q(full, I, J, K, q, p)
    H1, z1 = orc.grad_hess_q(full, I, J, K, q, p, mu=mu_f)
    assert np.array_equal(H0, H1) and np.array_equal(z0, z1)
    p2 = np.clip(p, 0.1, 0.9)
    H, z = orc.grad_hess_p(g.data, I, J, K, q, p2, mu=mu)
    h = 1e-6
    for j, k in [(0, 0), (5, 2), (40, 1)]:
        pp, pm = p2.copy(), p2.copy()
        pp[j, k] += h; pm[j, k] -= h
        fd = (orc.loglik(g.data, I, J, K, q, pp, mu=mu) - orc.loglik(g.data, I, J, K, q, pm, mu=mu)) / (2 * h)
        assert abs(fd - z[j, k]) < 1e-5 * max(1.0, abs(z[j, k]))
        _, zp = orc.grad_hess_p(g.data, I, J, K, q, pp, mu=mu)
        _, zm = orc.grad_hess_p(g.data, I, J, K, q, pm, mu=mu)
        assert np.allclose(-(zp[j] - zm[j]) / (2 * h), H[j, :, k], rtol=1e-5, atol=1e-5)
    r = orc.OracleRun(g.data, I, J, K, 3, x, skipmissing=False)
    hist = [r.loglik(r.x)] + r.init_em(5)
    assert all(b > a for a, b in zip(hist, hist[1:]))
