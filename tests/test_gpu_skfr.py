"""GPU tests of the SKFR AIM pre-selection (admix_skfr, csrc/skfr.cu) against its CPU oracle
(oracle/skfr_oracle.py): the same seeded k-means++ start, then identical clusters, AIMs and
iteration counts, and the objective to FP64 rounding -- for both modes, several tries, sizes
that leave partial 16-individual words and more than one seeding slice (4096 SNPs); then
run_admixture(sparsity=...) end to end, with the filtered PLINK files it writes."""
import sys
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

sys.path.insert(0, str(Path(__file__).resolve().parents[1] / "oracle"))
import skfr_oracle as S  # noqa: E402


def _cohort(oa, I, J, K, seed, alpha=0.05):
    spec = oa.COHORTS["c1"].scaled(I=I, J=J, K=K, seed=seed, alpha=alpha)
    g, q, p = oa.make_cohort(spec)
    return g, q


@pytest.mark.parametrize("I,J,K,s,mode,tries", [
    (301, 2003, 3, 150, "global", 1),
    (301, 2003, 3, 150, "local", 1),
    (437, 5000, 4, 300, "global", 3),      # two seeding slices, partial words
    (250, 1200, 6, 100, "local", 2),
    (300, 6000, 3, 2500, "global", 1),     # three reassignment slices of 1024 kept SNPs
    (260, 5000, 4, 1501, "local", 1),      # two slices per cluster list, an odd last pair
    (200, 2500, 16, 1101, "global", 1),    # the largest K, an odd last pair
    (150, 800, 2, 5000, "local", 1),       # sparsity above J: every SNP kept
    (90, 700, 1, 100, "global", 1),        # one cluster
])
def test_skfr_matches_oracle(oa, I, J, K, s, mode, tries):
    g, _ = _cohort(oa, I, J, max(K, 2), seed=40 + K, alpha=0.1)
    c, aims, obj, it = oa.skfr(g, K, s, mode=mode, tries=tries, rng=17)
    c_o, aims_o, obj_o, it_o = S.skfr(g.data, g.I, K, s, mode=mode, tries=tries, seed=17)
    assert np.array_equal(c, c_o)
    assert np.array_equal(aims, aims_o)
    assert it == it_o
    assert abs(obj - obj_o) <= 1e-12 * abs(obj_o)


def test_skfr_on_device_genotypes_matches_host_genotypes(oa):
    import torch
    torch.cuda.set_device(0)
    spec = oa.COHORTS["c1"].scaled(I=500, J=3000, K=3, seed=3, alpha=0.05)
    q, p = oa.truth(spec)
    gd = oa.genotypes_device(spec, q, p)
    gh = gd.to_host()
    a = oa.skfr(gd, 3, 200, tries=2, rng=5)
    b = oa.skfr(gh, 3, 200, tries=2, rng=5)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1]) and a[2] == b[2]
    true = np.argmax(q, axis=1)
    purity = sum(np.bincount(true[a[0] == k], minlength=3).max() for k in range(3)) / 500
    assert purity >= 0.95


def test_run_admixture_with_sparsity(oa, tmp_path):
    K = 3
    g, q = _cohort(oa, 400, 3000, K, seed=61)
    bed = tmp_path / "cohort.bed"
    oa.write_bed(bed, g)
    d, clusters, aims = oa.run_admixture(str(bed), K, sparsity=500, skfr_tries=2, rng=3, quiet=True)
    assert clusters.shape == (g.I,) and len(aims) == 500
    assert d.J == 500 and d.I == g.I
    out = tmp_path / f"cohort_{K}_500aims.bed"
    assert out.exists() and out.with_suffix(".bim").exists() and out.with_suffix(".fam").exists()
    sub = oa.read_bed(out)
    assert sub.J == 500 and np.array_equal(np.asarray(sub.data), np.asarray(g.data)[aims])
    assert len(out.with_suffix(".bim").read_text().splitlines()) == 500
    # the engine ran to convergence on the AIMs: its log-likelihood equals a plain run on the
    # filtered genotypes from the same start
    d2, c2, a2 = oa.run_admixture(sub, K, rng=3, quiet=True)
    assert c2 is None and a2 is None
    assert abs(d.ll_new - d2.ll_new) <= 1e-9 * abs(d2.ll_new)
