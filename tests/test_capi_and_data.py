"""CPU tests: the C-ABI library loads and exports every symbol include/admix.h declares;
argument checks fail cleanly without a GPU; BED I/O and the cohort generator."""
import ctypes as C
import re
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent


def _declared_symbols(header: Path) -> set[str]:
    txt = header.read_text()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return set(re.findall(r"\b(admix_[a-z_0-9]+)\s*\(", txt))


def test_header_symbols_exported(oa):
    declared = _declared_symbols(ROOT / "include" / "admix.h")
    assert len(declared) >= 20
    lib = C.CDLL(str(ROOT / "openadmixture.jl_b200" / "lib" / "libadmix.so"))
    missing = [s for s in sorted(declared) if not hasattr(lib, s)]
    assert not missing, missing
    from openadmixture_b200 import _native
    assert declared == set(_native.ADMIX_SIGNATURES), declared ^ set(_native.ADMIX_SIGNATURES)


def test_synth_library_exports(oa):
    lib = C.CDLL(str(ROOT / "openadmixture.jl_b200" / "lib" / "libadmix_synth.so"))
    for s in ("syn_truth", "syn_bed_host", "syn_bed_device", "syn_init_x"):
        assert hasattr(lib, s)


def test_create_rejects_bad_arguments_without_touching_a_gpu(oa):
    from openadmixture_b200 import _native as N
    lib = N.admix_lib()
    h = C.c_void_p()
    bed = np.zeros((4, 1), np.uint8)
    assert lib.admix_create(4, 4, 17, 3, N.u8ptr(bed), 0, C.byref(h)) == N.ADMIX_ERR_UNSUPPORTED
    assert b"K=17" in lib.admix_last_error(None)
    assert lib.admix_create(4, 4, 3, 9, N.u8ptr(bed), 0, C.byref(h)) == N.ADMIX_ERR_UNSUPPORTED
    assert lib.admix_create(0, 4, 3, 3, N.u8ptr(bed), 0, C.byref(h)) == N.ADMIX_ERR_ARG
    assert lib.admix_create(4, 4, 3, 3, None, 0, C.byref(h)) == N.ADMIX_ERR_ARG
    assert lib.admix_create(4, 4, 3, 3, N.u8ptr(bed), 0x100, C.byref(h)) == N.ADMIX_ERR_ARG
    assert lib.admix_loglik_dev(None, 4, 4, 3, None, None, None, None, 0, None) == N.ADMIX_ERR_ARG
    # device variant: a source pitch below ceil(I/4) is rejected before any device call
    assert lib.admix_create_device(40, 4, 3, 3, None, 9, 0, C.byref(h)) == N.ADMIX_ERR_ARG
    assert b"src_pitch" in lib.admix_last_error(None)
    # the failure-reporting self-test and SKFR need a handle
    assert lib.admix_selftest_wait_timeout(None) == N.ADMIX_ERR_ARG
    assert lib.admix_skfr(None, 3, 10, 0, 50, 1, 0, None, None, 0, None, None, None) == N.ADMIX_ERR_ARG
    assert b"handle is NULL" in lib.admix_last_error(None)


def test_engine_requires_gpu_path(oa):
    d = oa.AdmixData(8, 8, 2, 3, rng=1)
    with pytest.raises(NotImplementedError):
        oa.update_q(d, None, d_cu=None)
    with pytest.raises(NotImplementedError):
        oa.run_admixture(oa.Genotypes(np.zeros((8, 2), np.uint8), 8, 8), 2, use_gpu=False)
    with pytest.raises(NotImplementedError, match="an integer"):     # a vector of sparsities
        oa.run_admixture(oa.Genotypes(np.zeros((8, 2), np.uint8), 8, 8), 2, sparsity=[100, 50])
    with pytest.raises(ValueError, match="global or :local"):        # driver.jl:63
        oa.run_admixture(oa.Genotypes(np.zeros((8, 2), np.uint8), 8, 8), 2, sparsity=4, skfr_mode=":nearest")
    with pytest.raises(NotImplementedError, match="Float64 and Float32"):
        oa.run_admixture(oa.Genotypes(np.zeros((8, 2), np.uint8), 8, 8), 2, T=np.float16)


def test_admixdata_init_matches_reference_contract(oa):
    d = oa.AdmixData(13, 29, 4, 3, rng=3)
    assert d.q.shape == (4, 13) and d.p.shape == (4, 29)
    assert np.allclose(d.q.sum(0), 1.0, rtol=0, atol=1e-15)
    assert np.all((d.p >= 0) & (d.p < 1))
    assert np.isnan(d.ll_new)


def test_generator_is_deterministic_and_ragged(oa):
    spec = oa.COHORTS["c1"].scaled(I=1001, J=77, seed=4)
    g1, q1, p1 = oa.make_cohort(spec)
    g2, q2, p2 = oa.make_cohort(spec)
    assert np.array_equal(g1.data, g2.data) and np.array_equal(q1, q2)
    assert g1.data.shape == (77, 251)
    # padding bits of the last byte are zero
    assert np.all(g1.data[:, -1] >> 2 == 0)
    gg, nm = g1.decode()
    assert abs(1 - nm.mean() - spec.miss) < 0.005
    assert np.allclose(q1.sum(1), 1.0)
    # allele frequency of the draw follows q p'
    f = q1 @ p1.T
    assert abs((gg * nm).sum() / (2 * nm.sum()) - (f * nm).sum() / nm.sum()) < 0.01


def test_generator_beta_frequencies(oa):
    spec = oa.COHORTS["c3"].scaled(I=64, J=4000, seed=1)
    q, p = oa.truth(spec)
    assert p.min() >= 1e-3 and p.max() <= 1 - 1e-3
    assert np.mean(p < 0.1) > 0.15          # U-shaped Beta(0.5, 0.5)


def test_bed_roundtrip_and_format_errors(oa, tmp_path):
    spec = oa.COHORTS["c1"].scaled(I=37, J=19, seed=2)
    g, _, _ = oa.make_cohort(spec)
    path = oa.write_bed(tmp_path / "toy.bed", g)
    h = oa.read_bed(path)
    assert (h.I, h.J) == (37, 19) and np.array_equal(h.data, g.data)
    bad = tmp_path / "bad.bed"
    bad.write_bytes(b"\x6c\x1b\x00" + g.data.tobytes())
    with pytest.raises(oa.BedFormatError, match="magic"):
        oa.read_bed(bad, I=37, J=19)
    short = tmp_path / "short.bed"
    short.write_bytes(b"\x6c\x1b\x01" + g.data.tobytes()[:-5])
    with pytest.raises(oa.BedFormatError, match="size"):
        oa.read_bed(short, I=37, J=19)
    with pytest.raises(oa.BedFormatError):
        oa.read_bed(tmp_path / "toy.txt", I=1, J=1)


def test_decode_matches_golden(oa):
    from conftest import load_golden
    z = load_golden("small_k3")
    g = oa.Genotypes(z["bed"], int(z["I"]), int(z["J"]))
    gg, nm = g.decode()
    assert np.array_equal((nm == 0).sum(1), z["miss_ind"])
    assert np.array_equal((nm == 0).sum(0), z["miss_snp"])


def test_batch_create_rejects_bad_arguments_without_touching_a_gpu(oa):
    from openadmixture_b200 import _native as N
    lib = N.admix_lib()
    b = C.c_void_p()
    bed = np.zeros((4, 1), np.uint8)
    ks = (C.c_int32 * 3)(3, 17, 4)
    assert lib.admix_batch_create(4, 4, N.u8ptr(bed), 0, ks, 3, 0, C.byref(b)) == N.ADMIX_ERR_ARG
    assert b"n >= 1" in lib.admix_batch_last_error(None)
    assert lib.admix_batch_create(4, 4, N.u8ptr(bed), 3, ks, 3, 0, C.byref(b)) == N.ADMIX_ERR_UNSUPPORTED
    assert b"member 1: K=17" in lib.admix_batch_last_error(None)
    ok = (C.c_int32 * 2)(3, 4)
    assert lib.admix_batch_create(4, 4, N.u8ptr(bed), 2, ok, 9, 0, C.byref(b)) == N.ADMIX_ERR_UNSUPPORTED
    assert lib.admix_batch_create(4, 4, N.u8ptr(bed), 2, ok, 3, 0x100, C.byref(b)) == N.ADMIX_ERR_ARG
    assert lib.admix_batch_create(4, 4, None, 2, ok, 3, 0, C.byref(b)) == N.ADMIX_ERR_ARG
    assert lib.admix_batch_create_device(40, 4, None, 9, 2, ok, 3, 0, C.byref(b)) == N.ADMIX_ERR_ARG
    assert lib.admix_batch_run_qn(None, 5, 1e-7, None, None, None, None) == N.ADMIX_ERR_ARG
    assert lib.admix_batch_destroy(None) == N.ADMIX_OK


def test_streamed_create_rejects_bad_block_size(oa):
    from openadmixture_b200 import _native as N
    lib = N.admix_lib()
    h = C.c_void_p()
    bed = np.zeros((64, 1), np.uint8)
    assert lib.admix_create_streamed(4, 64, 3, 3, N.u8ptr(bed), 48, 0, C.byref(h)) == N.ADMIX_ERR_ARG
    assert b"multiple of 32" in lib.admix_last_error(None)
    assert lib.admix_create_streamed(4, 64, 3, 3, N.u8ptr(bed), 0, 0, C.byref(h)) == N.ADMIX_ERR_ARG
