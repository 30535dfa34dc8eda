"""GPU parity: every libadmix entry point against the oracle (and the golden fixtures) on the
same inputs.  Tolerances: integer decode bit-exact; FP64 sweeps 1e-10 relative (per entry,
relative to the entry or, for sums with cancellation, to the largest entry of its row);
SQP updates 1e-9 absolute on Q/P in [0, 1]; full runs 1e-6 relative on the final
log-likelihood."""
import ctypes as C

import numpy as np
import pytest

from conftest import load_golden, rel_err

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-10


def _cohort(oa, I, J, K, seed=1, cfg="c1", **kw):
    spec = oa.COHORTS[cfg].scaled(I=I, J=J, K=K, seed=seed, **kw)
    g, qt, pt = oa.make_cohort(spec)
    return g


def _handle(oa, g, K, Q=3, x=None, seed=3, flags=0):
    d = oa.AdmixData(g.I, g.J, K, Q, rng=seed)
    if x is not None:
        d.x[:] = x
    d_cu = oa.CuAdmixData(d, g, flags=flags)
    d_cu.upload(oa.X, d.x)
    return d, d_cu


def _row_rel(a, b):
    """max |a-b| / max(|b| row-wise max): relative error against each problem's own scale."""
    a = a.reshape(a.shape[0], -1); b = b.reshape(b.shape[0], -1)
    scale = np.abs(b).max(axis=1, keepdims=True)
    return float(np.max(np.abs(a - b) / np.maximum(scale, 1e-300)))


# ------------------------------------------------------------------ golden fixtures

def test_golden_decode_and_loglik(oa):
    for name in ("small_k3", "small_k5"):
        z = load_golden(name)
        I, J, K = int(z["I"]), int(z["J"]), int(z["K"])
        g = oa.Genotypes(z["bed"], I, J)
        d, d_cu = _handle(oa, g, K, x=z["x0"])
        snp, ind = d_cu.decode_counts()
        assert np.array_equal(snp, z["miss_snp"]) and np.array_equal(ind, z["miss_ind"])
        assert rel_err(d_cu.loglik(oa.X), z["ll_x0"]) < FP64_TOL
        d_cu.close()


def test_golden_em_sweeps_and_sqp(oa):
    for name in ("small_k3", "small_k5"):
        z = load_golden(name)
        I, J, K = int(z["I"]), int(z["J"]), int(z["K"])
        g = oa.Genotypes(z["bed"], I, J)
        d, d_cu = _handle(oa, g, K, x=z["x0"])
        oa.em_q(d_cu); oa.em_p(d_cu)
        xn = d_cu.download(oa.X_NEXT)
        assert rel_err(xn[:I], z["q_em"]) < FP64_TOL
        assert rel_err(xn[I:], z["p_em"]) < FP64_TOL
        xe = np.vstack([z["q_em"], z["p_em"]])
        d_cu.upload(oa.X, xe)
        H, zz = d_cu.grad_hess_q(oa.X, oa.X)
        assert _row_rel(H, z["XtX_q"]) < FP64_TOL and _row_rel(zz, z["Xtz_q"]) < FP64_TOL
        H, zz = d_cu.grad_hess_p(oa.X, oa.X)
        assert _row_rel(H, z["XtX_p"]) < FP64_TOL and _row_rel(zz, z["Xtz_p"]) < FP64_TOL
        d.x[:] = xe
        st = oa.update_q(d, g, False, d_cu=d_cu)
        assert np.array_equal(st, z["st_q"])
        assert np.max(np.abs(d.x_next[:I] - z["q_sqp"])) < 1e-9
        st = oa.update_p(d, g, False, d_cu=d_cu)
        assert np.array_equal(st, z["st_p"])
        assert np.max(np.abs(d.x_next[I:] - z["p_sqp"])) < 1e-9
        # four QN iterations
        d.x[:] = xe
        d.ll_new = float(z["ll_em"])
        recs = oa.admixture_qn(d, g, 4, 0.0, d_cu=d_cu, quiet=True)
        got = np.array([[r[k] for k in ("ll_prev", "ll_basic", "ll_qn", "ll_new")] for r in recs])
        assert rel_err(got, z["qn_info"][:, :4]) < 1e-9
        assert np.max(np.abs(d.x - z["x_qn4"])) < 1e-7
        d_cu.close()


# ------------------------------------------------------------------ vs oracle, many K

@pytest.mark.parametrize("K", [1, 2, 3, 5, 8, 9, 12, 16])
def test_sweeps_match_oracle(oa, orc, K):
    g = _cohort(oa, I=523, J=1031, K=K, seed=K)          # ragged last byte (523 % 4 = 3)
    d, d_cu = _handle(oa, g, K, seed=K + 10)
    I, J = g.I, g.J
    q, p = np.ascontiguousarray(d.x[:I]), np.ascontiguousarray(d.x[I:])
    assert rel_err(d_cu.loglik(oa.X), orc.loglik(g.data, I, J, K, q, p)) < FP64_TOL
    H, z = d_cu.grad_hess_q(oa.X, oa.X)
    Ho, zo = orc.grad_hess_q(g.data, I, J, K, q, p)
    assert _row_rel(H, Ho) < FP64_TOL and _row_rel(z, zo) < FP64_TOL
    H, z = d_cu.grad_hess_p(oa.X, oa.X)
    Ho, zo = orc.grad_hess_p(g.data, I, J, K, q, p)
    assert _row_rel(H, Ho) < FP64_TOL and _row_rel(z, zo) < FP64_TOL
    oa.em_q(d_cu); oa.em_p(d_cu)
    xn = d_cu.download(oa.X_NEXT)
    assert rel_err(xn[:I], orc.em_q(g.data, I, J, K, q, p)) < FP64_TOL
    assert rel_err(xn[I:], orc.em_p(g.data, I, J, K, q, p)) < FP64_TOL
    snp, ind = d_cu.decode_counts()
    snp_o, ind_o = orc.decode_counts(g.data, I, J)
    assert np.array_equal(snp, snp_o) and np.array_equal(ind, ind_o)
    d_cu.close()


@pytest.mark.parametrize("K,flags", [(3, 0), (6, 0), (6, 1), (12, 0)])
def test_init_em_and_sqp_updates_match_oracle(oa, orc, K, flags):
    g = _cohort(oa, I=401, J=2003, K=K, seed=20 + K)
    d, d_cu = _handle(oa, g, K, seed=4, flags=flags)
    r = orc.OracleRun(g.data, g.I, g.J, K, 3, d.x, mu_mode=flags & 1)
    ll_o = r.init_em(5)
    ll_g = oa.init_em(d, g, 5, d_cu=d_cu, quiet=True)
    assert rel_err(ll_g, ll_o) < 1e-9
    assert np.max(np.abs(d.x - r.x)) < 1e-9
    # one SQP half-step each way from identical inputs
    d.x[:] = r.x
    st_q = oa.update_q(d, g, False, d_cu=d_cu)
    st_qo = r.update_q(False)
    assert np.max(np.abs(d.x_next[: g.I] - r.x_next[: g.I])) < 1e-9
    # The device QPs are the oracle's QPs: run on the sums the device update used, the oracle's
    # quadratic_program! returns the device's status for every problem; and the statuses equal
    # the oracle's own run (the two FP64 sweeps' sums differ only at ~1e-15, which moved no
    # problem across an active-set test here).
    H, z = d_cu.grad_hess_q(oa.X, oa.X)
    st_chk, _ = orc.qp_batch(H, z, d.x[: g.I], True, mu_mode=flags & 1)
    assert np.array_equal(st_q, st_chk), np.flatnonzero(st_q != st_chk)
    assert np.array_equal(st_q, st_qo), np.flatnonzero(st_q != st_qo)
    st_p = oa.update_p(d, g, False, d_cu=d_cu)
    st_po = r.update_p(False)
    assert np.max(np.abs(d.x_next[g.I:] - r.x_next[g.I:])) < 1e-9
    H, z = d_cu.grad_hess_p(oa.X_NEXT, oa.X)
    st_chk, _ = orc.qp_batch(H, z, d.x[g.I:], False, mu_mode=flags & 1)
    assert np.array_equal(st_p, st_chk), np.flatnonzero(st_p != st_chk)
    assert np.array_equal(st_p, st_po), np.flatnonzero(st_p != st_po)
    d_cu.close()


@pytest.mark.parametrize("K,Q", [(3, 3), (4, 1), (5, 5)])
def test_qn_iterations_match_oracle(oa, orc, K, Q):
    g = _cohort(oa, I=300, J=1500, K=K, seed=30 + K)
    d, d_cu = _handle(oa, g, K, Q=Q, seed=5)
    r = orc.OracleRun(g.data, g.I, g.J, K, Q, d.x)
    r.init_em(3)
    d.x[:] = r.x
    d.ll_new = r.ll_new
    recs = oa.admixture_qn(d, g, 6, 0.0, d_cu=d_cu, quiet=True)
    for it, rec in enumerate(recs, start=1):
        o = r.qn_iteration(it)
        for k in ("ll_prev", "ll_basic", "ll_qn", "ll_new"):
            assert rel_err(rec[k], o[k]) < 1e-8, (it, k, rec[k], o[k])
    assert np.max(np.abs(d.x - r.x)) < 1e-6
    d_cu.close()


@pytest.mark.parametrize("K,Q", [(3, 3), (4, 1), (5, 5)])
def test_lbqn_iterations_match_oracle(oa, orc, K, Q):
    """admixture_qn!(...; mode=:LBQN) (quasi_newton.jl:15-58): the device's limited-memory
    Broyden step (one pass for all dot products, the alpha recurrence on the Gram matrix) against
    the oracle's literal vector updates, iteration by iteration, then both converge to the ZAL
    optimum."""
    g = _cohort(oa, I=300, J=1500, K=K, seed=130 + K)
    d, d_cu = _handle(oa, g, K, Q=Q, seed=7)
    r = orc.OracleRun(g.data, g.I, g.J, K, Q, d.x, mode="LBQN")
    r.init_em(3)
    d.x[:] = r.x
    d.ll_new = r.ll_new
    recs = oa.admixture_qn(d, g, 8, 0.0, d_cu=d_cu, quiet=True, mode="LBQN")
    for it, rec in enumerate(recs, start=1):
        o = r.qn_iteration(it)
        for k in ("ll_prev", "ll_basic", "ll_qn", "ll_new"):
            assert rel_err(rec[k], o[k]) < 1e-8, (it, k, rec[k], o[k])
    assert np.max(np.abs(d.x - r.x)) < 1e-6
    recs = oa.admixture_qn(d, g, 2000, 1e-7, d_cu=d_cu, quiet=True, mode=":LBQN", iter_count_offset=8)
    assert recs[-1]["reldiff"] < 1e-7
    dz = oa.AdmixData(g.I, g.J, K, Q, rng=7)
    with oa.CuAdmixData(dz, g) as hz:
        oa.init_em(dz, g, 3, d_cu=hz, quiet=True)
        oa.admixture_qn(dz, g, 2000, 1e-7, d_cu=hz, quiet=True)
    assert rel_err(d.ll_new, dz.ll_new) < 1e-6
    with pytest.raises(ValueError):
        oa.admixture_qn(d, g, 1, 0.0, d_cu=d_cu, quiet=True, mode="BFGS")
    d_cu.close()


def test_run_admixture_converges_like_oracle(oa, orc, tmp_path):
    spec = oa.COHORTS["c1"].scaled(I=600, J=4000, seed=8)
    g, _, _ = oa.make_cohort(spec)
    path = oa.write_bed(tmp_path / "c1s.bed", g)
    d, _, _ = oa.run_admixture(str(path), 3, rng=11, quiet=True)
    x0 = oa.init_x(g.I, g.J, 3, 11)
    r = orc.OracleRun(g.data, g.I, g.J, 3, 3, x0)
    r.init_em(5)
    hist, conv = r.admixture_qn(1000, 1e-7)
    assert conv
    assert rel_err(d.ll_new, r.ll_new) < 1e-6


def test_loglik_dev_entry_matches_handle(oa):
    import torch
    from openadmixture_b200 import _native as N
    g = _cohort(oa, I=777, J=3001, K=4, seed=2)
    d, d_cu = _handle(oa, g, 4)
    want = d_cu.loglik(oa.X)
    dev = torch.device("cuda:0")
    bed = torch.from_numpy(g.data).to(dev)
    q = torch.from_numpy(np.ascontiguousarray(d.x[: g.I])).to(dev)
    p = torch.from_numpy(np.ascontiguousarray(d.x[g.I:])).to(dev)
    out = torch.zeros(1, dtype=torch.float64, device=dev)
    lib = N.admix_lib()
    nbytes = lib.admix_loglik_dev_workspace(g.I, g.J, 4)
    work = torch.empty(nbytes, dtype=torch.uint8, device=dev)
    stream = torch.cuda.current_stream().cuda_stream
    rc = lib.admix_loglik_dev(C.c_void_p(bed.data_ptr()), g.I, g.J, 4, C.c_void_p(q.data_ptr()),
                              C.c_void_p(p.data_ptr()), C.c_void_p(out.data_ptr()),
                              C.c_void_p(work.data_ptr()), nbytes, C.c_void_p(stream))
    assert rc == 0
    torch.cuda.synchronize()
    assert out.item() == want          # same kernel, same plan: bit-identical
    rc = lib.admix_loglik_dev(C.c_void_p(bed.data_ptr()), g.I, g.J, 4, C.c_void_p(q.data_ptr()),
                              C.c_void_p(p.data_ptr()), C.c_void_p(out.data_ptr()),
                              C.c_void_p(work.data_ptr()), 8, C.c_void_p(stream))
    assert rc == N.ADMIX_ERR_ARG
    d_cu.close()


def test_error_paths(oa):
    from openadmixture_b200 import _native as N
    g = _cohort(oa, I=40, J=50, K=2)
    d, d_cu = _handle(oa, g, 2)
    lib = N.admix_lib()
    v = C.c_double()
    assert lib.admix_loglik(d_cu.handle, 7, C.byref(v)) == N.ADMIX_ERR_ARG
    assert b"selector" in lib.admix_last_error(d_cu.handle)
    assert lib.admix_qn_iteration(d_cu.handle, 0, None) == N.ADMIX_ERR_ARG
    with pytest.raises(oa.AdmixError):
        d_cu.loglik(9)
    d_cu.close()


def test_deterministic_across_runs(oa):
    g = _cohort(oa, I=1000, J=5000, K=5, seed=3)
    outs = []
    for _ in range(2):
        d, d_cu = _handle(oa, g, 5, seed=1)
        oa.init_em(d, g, 2, d_cu=d_cu, quiet=True)
        oa.admixture_qn(d, g, 3, 0.0, d_cu=d_cu, quiet=True)
        outs.append((d.ll_new, d.x.copy()))
        d_cu.close()
    assert outs[0][0] == outs[1][0] and np.array_equal(outs[0][1], outs[1][1])


# ------------------------------------------------------------------ full-size properties

def test_c2_size_properties(oa):
    """At the drop-in cohort's full size (I=10k, J=100k, K=5): missing counts equal a numpy
    popcount of the bytes, the log-likelihood is additive over SNP blocks, EM increases it,
    and the Q-side Hessian maps q to the gradient (XtX_q q = Xtz_q when sum q = 1)."""
    import torch
    from openadmixture_b200 import _native as N
    spec = oa.COHORTS["c2"]
    g, _, _ = oa.make_cohort(spec)
    d, d_cu = _handle(oa, g, spec.K, seed=2)
    snp, ind = d_cu.decode_counts()
    b = g.data
    miss = (b & ~(b >> 1) & 0x55)
    lut = np.array([bin(v).count("1") for v in range(256)], dtype=np.uint8)
    pc = lut[miss].sum(axis=1, dtype=np.int64)
    assert np.array_equal(snp, pc.astype(np.int64))
    assert ind.sum() == snp.sum()
    ll = d_cu.loglik(oa.X)
    lib = N.admix_lib()
    dev = torch.device("cuda:0")
    qd = torch.from_numpy(np.ascontiguousarray(d.x[: g.I])).to(dev)
    parts = []
    for j0, j1 in ((0, 37_000), (37_000, spec.J)):
        bed = torch.from_numpy(np.ascontiguousarray(g.data[j0:j1])).to(dev)
        pd = torch.from_numpy(np.ascontiguousarray(d.x[g.I + j0: g.I + j1])).to(dev)
        out = torch.zeros(1, dtype=torch.float64, device=dev)
        nb = lib.admix_loglik_dev_workspace(g.I, j1 - j0, spec.K)
        work = torch.empty(nb, dtype=torch.uint8, device=dev)
        assert lib.admix_loglik_dev(C.c_void_p(bed.data_ptr()), g.I, j1 - j0, spec.K, C.c_void_p(qd.data_ptr()),
                                    C.c_void_p(pd.data_ptr()), C.c_void_p(out.data_ptr()),
                                    C.c_void_p(work.data_ptr()), nb, None) == 0
        torch.cuda.synchronize()
        parts.append(out.item())
    assert rel_err(sum(parts), ll) < 1e-12
    hist = oa.init_em(d, g, 3, d_cu=d_cu, quiet=True)
    assert hist[0] > ll and hist[1] > hist[0] and hist[2] > hist[1]
    d_cu.upload(oa.X, d.x)
    H, z = d_cu.grad_hess_q(oa.X, oa.X)
    q = d.x[: g.I]
    qn = q / q.sum(1, keepdims=True)
    d.x[: g.I] = qn
    d_cu.upload(oa.X, d.x)
    H, z = d_cu.grad_hess_q(oa.X, oa.X)
    assert _row_rel(np.einsum("ikl,il->ik", H, qn), z) < 1e-10
    d_cu.close()


@pytest.mark.parametrize("flags", [0, 2])
def test_padding_bits_of_the_input_are_ignored(oa, flags):
    """The reference's loops stop at individual I, so whatever the file holds in the padding
    bits of each column's last byte must not change any result (FP64 and mixed forms)."""
    g = _cohort(oa, I=1027, J=700, K=4, seed=6)            # 1027 % 4 = 3: one padding field
    dirty = g.data.copy()
    dirty[:, -1] |= 0xC0                                    # padding field set to code 11
    gd = oa.Genotypes(dirty, g.I, g.J)
    vals = []
    for gg in (g, gd):
        d, d_cu = _handle(oa, gg, 4, seed=8, flags=flags)
        snp, ind = d_cu.decode_counts()
        H, z = d_cu.grad_hess_q(oa.X, oa.X)
        vals.append((d_cu.loglik(oa.X), snp, ind, H, z))
        d_cu.close()
    assert vals[0][0] == vals[1][0]
    assert np.array_equal(vals[0][1], vals[1][1]) and np.array_equal(vals[0][2], vals[1][2])
    assert np.array_equal(vals[0][3], vals[1][3]) and np.array_equal(vals[0][4], vals[1][4])


def test_device_generated_cohort_and_device_create(oa):
    """The device generator draws the host generator's bytes, and a handle created from device
    genotypes (admix_create_device) computes what the host-created one does."""
    spec = oa.COHORTS["c1"].scaled(I=1003, J=2111, K=4, seed=12)
    q, p = oa.truth(spec)
    gh = oa.genotypes(spec, q, p)
    gd = oa.genotypes_device(spec, q, p)
    assert np.array_equal(gd.to_host().data, gh.data)
    lls = []
    for g in (gh, gd):
        d, h = _handle(oa, g, 4, seed=3)
        lls.append((h.loglik(oa.X), h.decode_counts()))
        h.close()
    assert lls[0][0] == lls[1][0]
    assert np.array_equal(lls[0][1][0], lls[1][1][0]) and np.array_equal(lls[0][1][1], lls[1][1][1])


@pytest.mark.parametrize("fix_q,fix_p", [(False, True), (True, False)])
def test_fixed_block_iterations_match_oracle(oa, orc, fix_q, fix_p):
    """admixture_qn!(...; fix_q, fix_p) (algorithms_outer.jl:98-116): the fixed block is copied,
    not updated; the other block and the QN step match the oracle, and the fixed block ends as
    it started (up to the projection the reference applies to the QN point)."""
    K = 4
    g = _cohort(oa, I=300, J=1500, K=K, seed=44)
    d, d_cu = _handle(oa, g, K, Q=3, seed=6)
    r = orc.OracleRun(g.data, g.I, g.J, K, 3, d.x, fix_q=fix_q, fix_p=fix_p)
    r.init_em(3)
    d.x[:] = r.x
    d.ll_new = r.ll_new
    x0 = d.x.copy()
    recs = oa.admixture_qn(d, g, 5, 0.0, d_cu=d_cu, quiet=True, fix_q=fix_q, fix_p=fix_p)
    for it, rec in enumerate(recs, start=1):
        o = r.qn_iteration(it)
        for k in ("ll_prev", "ll_basic", "ll_qn", "ll_new"):
            assert rel_err(rec[k], o[k]) < 1e-8, (it, k, rec[k], o[k])
    assert np.max(np.abs(d.x - r.x)) < 1e-6
    fixed = slice(0, g.I) if fix_q else slice(g.I, None)
    moved = slice(g.I, None) if fix_q else slice(0, g.I)
    diff = d.x[fixed] - x0[fixed]
    if fix_q:   # the QN point's simplex projection: one shift per individual, rows summing to 1
        assert np.max(np.ptp(diff, axis=1)) < 1e-9
        assert np.max(np.abs(d.x[: g.I].sum(1) - 1.0)) < 1e-9
    else:       # P of the EM point is already inside [1e-5, 1 - 1e-5]
        assert np.max(np.abs(diff)) < 1e-12
    assert np.max(np.abs(d.x[moved] - x0[moved])) > 1e-3
    # the mode is per call: the next plain call updates both blocks again
    x1 = d.x.copy()
    oa.admixture_qn(d, g, 1, 0.0, d_cu=d_cu, quiet=True)
    assert np.max(np.abs(d.x[fixed] - x1[fixed])) > 1e-6
    d_cu.close()


@pytest.mark.parametrize("flags", [0, 2])
def test_streamed_handle_matches_resident_handle(oa, flags):
    """admix_create_streamed: the genotypes stay in host memory and every pass streams SNP blocks
    (here 3: 1024 + 1024 + 953 SNPs); results equal the device-resident handle's up to the order
    of the FP64 sums."""
    K = 4
    g = _cohort(oa, I=437, J=3001, K=K, seed=52)
    d = oa.AdmixData(g.I, g.J, K, 3, rng=3)
    hr = oa.CuAdmixData(d, g, flags=flags)
    hs = oa.CuAdmixData(d, g, flags=flags, stream_block=1024)
    for h in (hr, hs):
        h.upload(oa.X, d.x)
    assert rel_err(hs.loglik(oa.X), hr.loglik(oa.X)) < 1e-13
    tol = 1e-12 if flags == 0 else 1e-6
    for side in ("q", "p"):
        H0, z0 = getattr(hr, f"grad_hess_{side}")(oa.X, oa.X)
        H1, z1 = getattr(hs, f"grad_hess_{side}")(oa.X, oa.X)
        assert np.max(np.abs(z1 - z0)) <= tol * np.abs(z0).max(), side
        assert np.max(np.abs(H1 - H0)) <= (tol if flags == 0 else 2e-2) * np.abs(H0).max(), side
    assert all(np.array_equal(a, b) for a, b in zip(hs.decode_counts(), hr.decode_counts()))
    d1, d2 = oa.AdmixData(g.I, g.J, K, 3, rng=3), oa.AdmixData(g.I, g.J, K, 3, rng=3)
    oa.init_em(d1, g, 3, d_cu=hr, quiet=True)
    oa.init_em(d2, g, 3, d_cu=hs, quiet=True)
    assert rel_err(d2.ll_new, d1.ll_new) < 1e-12
    r1 = oa.admixture_qn(d1, g, 4, 0.0, d_cu=hr, quiet=True)
    r2 = oa.admixture_qn(d2, g, 4, 0.0, d_cu=hs, quiet=True)
    # FP64: the same iteration up to the order of FP64 sums.  Mixed: the BF16 Hessian sums restart
    # at every streamed block, so the Hessians differ at ~1e-4 and early iterates drift apart a
    # little (the optimum does not move; test_run_admixture_streamed checks the converged value).
    for a, b in zip(r1, r2):
        assert rel_err(b["ll_new"], a["ll_new"]) < (1e-10 if flags == 0 else 1e-5)
    hr.close(); hs.close()


def test_streamed_handle_matches_oracle(oa, orc):
    """The out-of-core path against the oracle directly (not only against the resident handle):
    genotypes in host memory streamed in 3 SNP blocks (1024 + 1024 + 953), FP64 form -- decode
    counts bit-exact, log-likelihood, Q- and P-side gradient and Hessian at 1e-10, EM priming and
    QN iterations at the tolerances of the resident-handle parity tests."""
    K = 4
    g = _cohort(oa, I=437, J=3001, K=K, seed=54)
    I, J = g.I, g.J
    d = oa.AdmixData(I, J, K, 3, rng=7)
    q, p = np.ascontiguousarray(d.x[:I]), np.ascontiguousarray(d.x[I:])
    with oa.CuAdmixData(d, g, stream_block=1024) as h:
        h.upload(oa.X, d.x)
        snp, ind = h.decode_counts()
        snp_o, ind_o = orc.decode_counts(g.data, I, J)
        assert np.array_equal(snp, snp_o) and np.array_equal(ind, ind_o)
        assert rel_err(h.loglik(oa.X), orc.loglik(g.data, I, J, K, q, p)) < FP64_TOL
        H, z = h.grad_hess_q(oa.X, oa.X)
        Ho, zo = orc.grad_hess_q(g.data, I, J, K, q, p)
        assert _row_rel(H, Ho) < FP64_TOL and _row_rel(z, zo) < FP64_TOL
        H, z = h.grad_hess_p(oa.X, oa.X)
        Ho, zo = orc.grad_hess_p(g.data, I, J, K, q, p)
        assert _row_rel(H, Ho) < FP64_TOL and _row_rel(z, zo) < FP64_TOL
        r = orc.OracleRun(g.data, I, J, K, 3, d.x)
        ll_em_o = r.init_em(3)
        ll_em = oa.init_em(d, g, 3, d_cu=h, quiet=True)
        assert rel_err(np.array(ll_em), np.array(ll_em_o)) < FP64_TOL
        d.x[:] = r.x
        d.ll_new = r.ll_new
        recs = oa.admixture_qn(d, g, 4, 0.0, d_cu=h, quiet=True)
    for it, rec in enumerate(recs, start=1):
        o = r.qn_iteration(it)
        for k in ("ll_prev", "ll_basic", "ll_qn", "ll_new"):
            assert rel_err(rec[k], o[k]) < 1e-8, (it, k, rec[k], o[k])


@pytest.mark.parametrize("flags", [0, 2])
def test_run_admixture_streamed(oa, flags):
    g = _cohort(oa, I=300, J=2000, K=3, seed=53)
    d0, _, _ = oa.run_admixture(g, 3, rng=5, quiet=True)
    d1, _, _ = oa.run_admixture(g, 3, rng=5, quiet=True, stream_block=512, flags=flags)
    assert rel_err(d1.ll_new, d0.ll_new) < (1e-9 if flags == 0 else 1e-6)


@pytest.mark.parametrize("K", [2, 5, 12])
def test_mean_imputed_loops_match_oracle(oa, orc, K):
    """AdmixData(...; skipmissing=false) (ADMIX_FLAG_MEAN_IMPUTE): every pass of the FP64 form with
    missing genotypes imputed by their SNP's mean dosage (loops.jl:493-514,589-608,679-698,
    840-865,896-921) against the oracle's mean-imputed loops, then EM and QN iterations; the
    flag is refused with the mixed form and with a streamed handle."""
    g = _cohort(oa, I=411, J=1703, K=K, seed=150 + K, miss=0.05)
    d = oa.AdmixData(g.I, g.J, K, 3, rng=K, skipmissing=False)
    I, J = g.I, g.J
    mu = orc.snp_means(g.data, I, J)
    q, p = np.ascontiguousarray(d.x[:I]), np.ascontiguousarray(d.x[I:])
    with oa.CuAdmixData(d, g) as h:
        h.upload(oa.X, d.x)
        assert rel_err(h.loglik(oa.X), orc.loglik(g.data, I, J, K, q, p, mu=mu)) < FP64_TOL
        assert rel_err(h.loglik(oa.X), orc.loglik(g.data, I, J, K, q, p)) > 1e-6     # not the skipmissing value
        H, z = h.grad_hess_q(oa.X, oa.X)
        Ho, zo = orc.grad_hess_q(g.data, I, J, K, q, p, mu=mu)
        assert _row_rel(H, Ho) < FP64_TOL and _row_rel(z, zo) < FP64_TOL
        H, z = h.grad_hess_p(oa.X, oa.X)
        Ho, zo = orc.grad_hess_p(g.data, I, J, K, q, p, mu=mu)
        assert _row_rel(H, Ho) < FP64_TOL and _row_rel(z, zo) < FP64_TOL
        oa.em_q(h); oa.em_p(h)
        xn = h.download(oa.X_NEXT)
        assert rel_err(xn[:I], orc.em_q(g.data, I, J, K, q, p, mu=mu)) < FP64_TOL
        assert rel_err(xn[I:], orc.em_p(g.data, I, J, K, q, p, mu=mu)) < FP64_TOL
        r = orc.OracleRun(g.data, I, J, K, 3, d.x, skipmissing=False)
        ll_o = r.init_em(3)
        ll_g = oa.init_em(d, g, 3, d_cu=h, quiet=True)
        assert rel_err(np.array(ll_g), np.array(ll_o)) < 1e-9
        d.x[:] = r.x
        d.ll_new = r.ll_new
        recs = oa.admixture_qn(d, g, 4, 0.0, d_cu=h, quiet=True)
        for it, rec in enumerate(recs, start=1):
            o = r.qn_iteration(it)
            for k in ("ll_prev", "ll_basic", "ll_qn", "ll_new"):
                assert rel_err(rec[k], o[k]) < 1e-8, (it, k, rec[k], o[k])
    with pytest.raises(oa.AdmixError):
        oa.CuAdmixData(d, g, flags=oa.ADMIX_FLAG_MIXED)
    with pytest.raises(oa.AdmixError):
        oa.CuAdmixData(d, g, stream_block=512)
