"""GPU tests of batches (restarts and K sweeps over one cohort): with the single-problem work
split a batch reproduces each member's solo run bit for bit (same kernels, same plans, only
run concurrently); after the autotuner picks another split the EM iterates agree with the solo
runs' and the members at the cohort's own K reach the same optima; converged members leave the
batch while the others continue."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def cohort(oa):
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    spec = oa.COHORTS["c4"].scaled(I=1_500, J=2_500, seed=7)
    g, _, _ = oa.make_cohort(spec)
    return g


def _solo(oa, g, K, seed, flags, em, n_iter, rtol):
    from openadmixture_b200 import _native as N
    d = oa.AdmixData(g.I, g.J, K, 3)
    d.x[:] = oa.init_x(g.I, g.J, K, seed)
    with oa.CuAdmixData(d, g, flags=flags) as h:
        h.upload(oa.X, d.x)
        hist = np.zeros(max(em, 1))
        h._chk(N.admix_lib().admix_init_em(h.handle, em, N.dptr(hist)))
        recs = (N.IterInfo * n_iter)()
        nd, cv = C.c_int32(), C.c_int32()
        h._chk(N.admix_lib().admix_run_qn(h.handle, n_iter, rtol, 0, recs, C.byref(nd), C.byref(cv)))
        return h.download(oa.X), nd.value, bool(cv.value), hist[:em], recs[nd.value - 1].ll_new


@pytest.mark.parametrize("flags", [0, 2])
def test_batch_matches_solo_runs_bit_for_bit(oa, cohort, flags):
    g = cohort
    Ks, seeds = [3, 3, 4, 2, 6], [0, 1, 0, 0, 5]
    with oa.AdmixBatch(g, Ks, flags=flags, seeds=seeds) as b:
        hist = b.init_em(5)
        rec = b.run_qn(300, 1e-7)
        xs = [b.x(m) for m in range(len(Ks))]
    for m, (K, s) in enumerate(zip(Ks, seeds)):
        x, nd, cv, h, ll = _solo(oa, g, K, s, flags, 5, 300, 1e-7)
        assert np.array_equal(hist[m], h), m
        assert rec["iterations"][m] == nd and rec["converged"][m] == cv, (m, rec["iterations"][m], nd)
        assert rec["ll"][m] == ll, m
        assert np.array_equal(xs[m], x), m
    # members finished at different iterations and left the batch independently
    assert len(set(rec["iterations"].tolist())) > 1
    assert rec["ms_device"] > 0


def _solo_em(oa, g, K, seed, flags, em):
    from openadmixture_b200 import _native as N
    d = oa.AdmixData(g.I, g.J, K, 3)
    d.x[:] = oa.init_x(g.I, g.J, K, seed)
    with oa.CuAdmixData(d, g, flags=flags) as h:
        h.upload(oa.X, d.x)
        hist = np.zeros(max(em, 1))
        h._chk(N.admix_lib().admix_init_em(h.handle, em, N.dptr(hist)))
        return h.download(oa.X)


def test_autotuned_batch_reaches_the_same_optima(oa, cohort):
    """Another work split regroups the FP64 sums across chunks (EM iterates agree with the solo
    run's to 1e-10) and the mixed form's FP32 Hessian blocks (a ~1e-7 perturbation).  At the
    cohort's own K = 6 every member reaches the solo run's optimum; below it, several merges of
    the 6 populations are local optima and such a perturbation may settle a run in another, so
    those members are held to convergence only."""
    g = cohort
    Ks = [6, 6, 6, 2, 3, 4]
    seeds = [0, 1, 2, 0, 0, 0]
    with oa.AdmixBatch(g, Ks, flags=2, seeds=seeds) as b:
        d, ms = b.autotune()
        assert d >= 1 and (d & (d - 1)) == 0 and ms > 0
        b.init_em(5)
        x_em = [b.x(m) for m in range(len(Ks))]
        rec = b.run_qn(500, 1e-7)
        ll = [b.members[m].loglik(oa.X) for m in range(len(Ks))]
    assert rec["converged"].all()
    for m, (K, s) in enumerate(zip(Ks, seeds)):
        assert np.abs(x_em[m] - _solo_em(oa, g, K, s, 2, 5)).max() < 1e-10, m
        if K != 6:
            continue
        x, nd, cv, _, _ = _solo(oa, g, K, s, 2, 5, 500, 1e-7)
        assert cv, m
        d_ = oa.AdmixData(g.I, g.J, K, 3)
        with oa.CuAdmixData(d_, g) as h:
            h.upload(oa.X, x)
            ll_solo = h.loglik(oa.X)
        assert abs(ll[m] - ll_solo) <= 1e-6 * abs(ll_solo), (m, ll[m], ll_solo)


def test_member_handles_and_errors(oa, cohort):
    from openadmixture_b200 import _native as N
    g = cohort
    with oa.AdmixBatch(g, [2, 3]) as b:
        h = C.c_void_p()
        assert N.admix_lib().admix_batch_member(b.handle, 2, C.byref(h)) == N.ADMIX_ERR_ARG
        assert b"outside" in N.admix_lib().admix_batch_last_error(b.handle)
        assert N.admix_lib().admix_batch_set_split(b.handle, 0) == N.ADMIX_ERR_ARG
        # a member is an ordinary handle: its loglik equals a solo handle's on the same x
        x = b.x(1)
        ll_m = b.members[1].loglik(oa.X)
        d = oa.AdmixData(g.I, g.J, 3, 3)
        with oa.CuAdmixData(d, g) as s:
            s.upload(oa.X, x)
            assert s.loglik(oa.X) == ll_m
        n = C.c_int32()
        assert N.admix_lib().admix_batch_size(b.handle, C.byref(n)) == 0 and n.value == 2


def test_run_restarts_and_k_sweep_helpers(oa, cohort):
    g = cohort
    x, ll, rec = oa.run_restarts(g, 3, 4, flags=2)
    assert x.shape == (g.I + g.J, 3) and np.isfinite(ll) and rec["converged"].all()
    res, rec = oa.k_sweep(g, [2, 3, 4], flags=2)
    lls = [res[K][1] for K in (2, 3, 4)]
    assert lls[0] < lls[1] < lls[2]          # more clusters fit better on the same data
