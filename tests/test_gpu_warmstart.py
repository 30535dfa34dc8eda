"""GPU tests of the learned warm start (csrc/mlp.cu) against the numpy checker: the sketch, the
MLP forward / backward (gradients), Adam, the closed-form P step; and the gain itself -- a
learned start (sketch + encoder + P step included) reaches the FP64 optimum in less time than
the random start + 5 EM -- and the fallback outside the populations the model was trained on."""
import sys
import time
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT / "oracle"))
import mlp_oracle as mo  # noqa: E402

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ws(oa):
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from openadmixture_b200 import warmstart
    return warmstart


def _cohort(oa, I, J, K, seed, **kw):
    spec = oa.COHORTS["c1"].scaled(I=I, J=J, K=K, seed=seed, **kw)
    return oa.make_cohort(spec)


def test_sketch_matches_oracle(oa, ws):
    g, _, _ = _cohort(oa, 1001, 700, 3, 11)
    snps = np.sort(np.random.default_rng(0).choice(700, 257, replace=False)).astype(np.int32)
    sk = ws.sketch(g, snps, R=32, seed=7)
    freq, dos, proj = mo.sketch(g.data, g.I, snps, 32, 7)
    assert np.array_equal(sk.dos.cpu().numpy(), dos)
    assert np.allclose(sk.freq.cpu().numpy(), freq, rtol=1e-6, atol=1e-7)
    # FP32 sums of 257 standardised terms
    assert np.allclose(sk.proj.cpu().numpy(), proj, rtol=1e-4, atol=1e-4)


def test_sketch_of_device_genotypes_is_identical(oa, ws):
    spec = oa.COHORTS["c1"].scaled(I=3001, J=500, K=3, seed=2)
    q, p = oa.truth(spec)
    gh, gd = oa.genotypes(spec, q, p), oa.genotypes_device(spec, q, p)
    snps = ws.sketch_snps(500, S=128, seed=1)
    a, b = ws.sketch(gh, snps), ws.sketch(gd, snps)
    assert np.array_equal(a.dos.cpu().numpy(), b.dos.cpu().numpy())
    assert np.array_equal(a.proj.cpu().numpy(), b.proj.cpu().numpy())


def _random_model(ws, S, R, K, H, seed):
    m = ws.WarmStartMLP(S, R, K, H=H, seed=seed)
    rng = np.random.default_rng(seed + 1)
    import torch
    for k in ("b1", "b2", "b3"):         # non-zero biases so every term of the gradient is exercised
        m.p[k].copy_(torch.tensor(rng.normal(0, 0.1, m.p[k].shape).astype(np.float32)))
    return m


@pytest.mark.parametrize("n,S,K", [(300, 100, 8), (65, 1000, 3), (1, 64, 2)])
def test_mlp_forward_backward_match_oracle(oa, ws, n, S, K):
    import ctypes as C
    import torch
    from openadmixture_b200 import _native as N
    R, H = 32, 256
    rng = np.random.default_rng(n)
    dos = rng.integers(0, 4, (n, S)).astype(np.int8)
    center = rng.uniform(0.1, 1.9, S).astype(np.float32)
    proj = rng.normal(0, 1, (n, R)).astype(np.float32)
    tgt = rng.dirichlet(np.full(K, 0.5), n).astype(np.float32)
    m = _random_model(ws, S, R, K, H, seed=n)
    params = m.numpy_params()
    loss_ref, g_ref = mo.loss_and_grads(params, dos, center.astype(np.float64), proj, tgt.astype(np.float64))
    *_, p_ref = mo.forward(params, dos, center.astype(np.float64), proj)

    dev = torch.device("cuda")
    t = lambda a: torch.tensor(a, device=dev)  # noqa: E731
    d_dos, d_c, d_pr, d_t = t(dos), t(center), t(proj), t(tgt)
    h1 = torch.empty((n, H), device=dev); h2 = torch.empty_like(h1); dh1 = torch.empty_like(h1); dh2 = torch.empty_like(h1)
    lg = torch.empty((n, K), device=dev); pr = torch.empty_like(lg); dl = torch.empty_like(lg)
    loss = torch.zeros(1, device=dev)
    grads = {k: torch.full_like(v, float("nan")) for k, v in m.p.items()}
    G = N.MLPGrads(*[grads[k].data_ptr() for k in ws.WarmStartMLP.NAMES])
    net = m.net()
    P = lambda x: C.c_void_p(x.data_ptr())  # noqa: E731
    lib = N.admix_lib()
    assert lib.admix_mlp_forward(C.byref(net), n, P(d_dos), P(d_c), P(d_pr), P(h1), P(h2), P(lg), P(pr), None) == 0
    assert lib.admix_mlp_backward(C.byref(net), C.byref(G), n, P(d_dos), P(d_c), P(d_pr), P(h1), P(h2), P(lg), P(d_t),
                                  P(pr), P(dl), P(dh2), P(dh1), P(loss), None) == 0
    torch.cuda.synchronize()
    # FP32 arithmetic against the FP64 checker: relative to each tensor's scale
    assert np.allclose(pr.cpu().numpy(), p_ref, atol=2e-5)
    assert abs(loss.item() / n - loss_ref) <= 1e-5 * max(1.0, abs(loss_ref))
    for k, ref in g_ref.items():
        got = grads[k].cpu().numpy().astype(np.float64)
        scale = np.abs(ref).max() + 1e-12
        assert np.abs(got - ref).max() <= 2e-4 * scale, (k, np.abs(got - ref).max() / scale)


def test_adam_matches_formula(oa, ws):
    import ctypes as C
    import torch
    from openadmixture_b200 import _native as N
    rng = np.random.default_rng(3)
    n = 70_001
    w0, g1, g2 = (rng.normal(0, 1, n).astype(np.float32) for _ in range(3))
    w, m, v = (torch.tensor(a, device="cuda") for a in (w0, np.zeros(n, np.float32), np.zeros(n, np.float32)))
    P = lambda x: C.c_void_p(x.data_ptr())  # noqa: E731
    ww, mm, vv = w0.astype(np.float64), np.zeros(n), np.zeros(n)
    for step, g in ((1, g1), (2, g2)):
        dg = torch.tensor(g, device="cuda")
        assert N.admix_lib().admix_mlp_adam(P(w), P(dg), P(m), P(v), n, 1e-2, 0.9, 0.999, 1e-8, step, None) == 0
        mm = 0.9 * mm + 0.1 * g
        vv = 0.999 * vv + 0.001 * g.astype(np.float64) ** 2
        ww = ww - 1e-2 * (mm / (1 - 0.9 ** step)) / (np.sqrt(vv / (1 - 0.999 ** step)) + 1e-8)
    torch.cuda.synchronize()
    assert np.allclose(w.cpu().numpy(), ww, rtol=0, atol=1e-5)


@pytest.mark.parametrize("K", [1, 5, 8, 16])
def test_warm_p_matches_oracle(oa, ws, K):
    g, _, _ = _cohort(oa, 1001, 333, max(K, 2), 5)
    q = np.random.default_rng(K).dirichlet(np.ones(K), g.I)
    got = ws.warm_p(g, q)
    ref = mo.warm_p(g.data, g.I, K, q)
    # FP32 accumulation over ~1000 individuals; the ratio keeps the relative error
    assert np.allclose(got, ref, rtol=2e-5, atol=1e-7)


def test_model_file_roundtrip_is_fp16(oa, ws, tmp_path):
    m = _random_model(ws, 128, 32, 4, 64, seed=1)
    m.save(tmp_path / "m.npz")
    z = np.load(tmp_path / "m.npz")
    assert z["w1"].dtype == np.float16 and z["w1"].shape == (160, 64)
    m2 = ws.WarmStartMLP.load(tmp_path / "m.npz")
    for k in ws.WarmStartMLP.NAMES:
        assert np.array_equal(m2.p[k].cpu().numpy(), m.p[k].cpu().numpy().astype(np.float16).astype(np.float32))


def _world(oa, name, I, J, K, seed, world):
    return oa.CohortSpec(name, I, J, K, alpha=0.2, miss=0.01, seed=seed, p_seed=world)


def test_learned_start_beats_random_start(oa, ws):
    """Train on 8 small cohorts of one world, then solve a held-out cohort of that world: the
    learned start reaches within 1e-6 (relative) of the FP64 optimum with fewer genotype passes
    than 5 EM iterations + QN from the random start."""
    import torch
    I, J, K, world = 3000, 4000, 3, 31
    snps = ws.sketch_snps(J, S=1024, seed=5)
    data = []
    for c in range(8):
        spec = _world(oa, f"t{c}", I, J, K, 100 + c, world)
        q, p = oa.truth(spec)
        g = oa.genotypes_device(spec, q, p)
        r = ws.run_to_target(g, K, rng=c)
        tgt = ws.align_to_populations(r["x"][:I], r["x"][I:], p)
        data.append((ws.sketch(g, snps), torch.tensor(tgt.astype(np.float32), device="cuda")))
    model = ws.WarmStartMLP(len(snps), 32, K, seed=0)
    hist = ws.train(model, data, epochs=12, batch=1024, lr=1e-3)
    assert hist[-1] < hist[0]

    spec = _world(oa, "held-out", I, J, K, 999, world)
    q, p = oa.truth(spec)
    g = oa.genotypes_device(spec, q, p)
    plain = ws.run_to_target(g, K, rng=1)
    target = plain["ll"] - 1e-6 * abs(plain["ll"])
    rand = ws.run_to_target(g, K, rng=1, target=target)
    start = ws.predict_start(model, g, snps)
    assert np.allclose(start[0].sum(1), 1.0) and start[1].shape == (J, K)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    start = ws.predict_start(model, g, snps)
    t_pred = time.perf_counter() - t0
    learned = ws.run_to_target(g, K, rng=1, start=start, target=target)
    assert rand["iterations_to_target"] is not None and learned["iterations_to_target"] is not None
    # Work to the target in passes over the genotypes (at this size a QN iteration takes well under
    # a millisecond, so wall time is launch noise; test_committed_model_gain compares seconds):
    # a QN iteration is 6 passes (4 sweeps, 2 log-likelihoods), an EM iteration 3 (2 sweeps and
    # its log-likelihood), the learned start 1 (the closed-form P step; sketch and encoder read
    # 4096 SNPs) plus its LEARNED_EM EM iterations.  The learned arm must need strictly fewer.
    work_learned = 6 * learned["iterations_to_target"] + 1 + 3 * ws.LEARNED_EM
    work_rand = 3 * 5 + 6 * rand["iterations_to_target"]
    assert work_learned < work_rand, (learned["iterations_to_target"], rand["iterations_to_target"], t_pred)
    # the learned start ends at the same optimum
    assert abs(learned["ll"] - plain["ll"]) <= 1e-6 * abs(plain["ll"])


def test_committed_model_gain(oa, ws):
    """The shipped K=8 model on a held-out cohort of its training world (I=20k, J=100k)."""
    import torch
    path = ws.default_model_path(8)
    if not path.exists():
        pytest.skip(f"{path.name} not trained")
    model = ws.WarmStartMLP.load(path)
    spec = _world(oa, "held-out", 20_000, 100_000, 8, 4242, ws.WORLD_SEED)
    q, p = oa.truth(spec)
    g = oa.genotypes_device(spec, q, p)
    assert np.array_equal(model.snps, ws.sketch_snps(100_000, S=model.S))
    plain = ws.run_to_target(g, 8, rng=1)
    target = plain["ll"] - 1e-6 * abs(plain["ll"])
    rand = ws.run_to_target(g, 8, flags=oa.ADMIX_FLAG_MIXED, rng=1, target=target)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    info = {}
    start = ws.learned_start(g, 8, model, info=info)
    t_pred = time.perf_counter() - t0
    assert start is not None and info["freq_corr"] > 0.99, info      # the training world passes the check
    learned = ws.run_to_target(g, 8, flags=oa.ADMIX_FLAG_MIXED, rng=1, start=start, target=target)
    assert learned["iterations_to_target"] is not None
    assert learned["seconds_to_target"] + t_pred < rand["seconds_to_target"], (learned, rand, t_pred)


def test_committed_model_falls_back_outside_its_world(oa, ws):
    """A cohort drawn from other ancestral populations (another p_seed) than the shipped model's
    training cohorts: its sketch-SNP allele frequencies do not match the model's record, so
    learned_start refuses and run_admixture takes the random start + EM -- the plain method stays
    the fallback, and the refused start is never used."""
    path = ws.default_model_path(8)
    if not path.exists():
        pytest.skip(f"{path.name} not trained")
    model = ws.WarmStartMLP.load(path)
    assert model.freq is not None
    spec = _world(oa, "other-world", 20_000, 100_000, 8, 4242, ws.WORLD_SEED + 1)
    q, p = oa.truth(spec)
    g = oa.genotypes_device(spec, q, p)
    info = {}
    assert ws.learned_start(g, 8, model, info=info) is None
    assert info["freq_corr"] < ws.MIN_FREQ_CORR and "other ancestral populations" in info["fallback"]
    d0, _, _ = oa.run_admixture(g, 8, rng=3, quiet=True, admix_n_iter=3)
    d1, _, _ = oa.run_admixture(g, 8, rng=3, quiet=True, admix_n_iter=3, warm_start="learned")
    assert np.array_equal(d0.x, d1.x) and d0.ll_new == d1.ll_new


def test_run_admixture_warm_start_plumbing(oa, ws, tmp_path):
    """run_admixture(warm_start=...) starts from the encoder's Q and the closed-form P with no EM;
    with no model for K it falls back to the random start + EM and matches the plain run."""
    g, _, _ = _cohort(oa, 1500, 2000, 3, 21)
    m = _random_model(ws, 256, 32, 3, 64, seed=3)
    m.snps = ws.sketch_snps(2000, S=256, seed=2)
    m.save(tmp_path / "m3.npz")
    d, _, _ = oa.run_admixture(g, 3, rng=4, warm_start=tmp_path / "m3.npz", quiet=True, admix_n_iter=200)
    assert np.allclose(d.q.sum(0), 1.0) and np.all(d.p >= 1e-5 - 1e-15)
    assert np.isfinite(d.ll_new)
    # fallback (no shipped K=3 model): identical to the plain call
    d0, _, _ = oa.run_admixture(g, 3, rng=4, quiet=True, admix_n_iter=200)
    d1, _, _ = oa.run_admixture(g, 3, rng=4, warm_start="learned", quiet=True, admix_n_iter=200)
    assert np.array_equal(d0.x, d1.x) and d0.ll_new == d1.ll_new
