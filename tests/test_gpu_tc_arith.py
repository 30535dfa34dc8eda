"""The tensor-core arithmetic the mixed form is designed around, checked on the device through
admix_tc_probe (one tcgen05 BF16 MMA chain, FP32 accumulator in TMEM):

- BF16 x BF16 products and sums of small integers are exact, with A read from shared memory or
  from tensor memory (the two operand paths agree bit for bit);
- FP32 sums are truncated toward zero, inside one MMA and when an MMA adds to the accumulator:
  1 + 0.75 ulp gives 1, 1 + 1.5 ulp gives 1 + 1 ulp, the same in magnitude for negative sums;
- sixteen positive products of spread magnitude therefore never come out above the exact sum,
  and come out below it on average -- why every long FP32 sum in TMEM is restarted (the
  per-chunk diagonal, the 256-chunk Hessian blocks, the loglik's exact limb accumulators)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ULP1 = 2.0 ** -23


def _bf16_bits(x):
    x = np.ascontiguousarray(x, np.float32)
    u = x.view(np.uint32)
    assert np.all((u & 0xFFFF) == 0), "value not exact in BF16"
    return np.ascontiguousarray((u >> 16).astype(np.uint16))


def _run(oa, A, B, nsteps, a_in_tmem=0):
    lib = oa._native.admix_lib()
    a, b = _bf16_bits(A), _bf16_bits(B)
    d = np.zeros((128, 16), np.float32)
    rc = lib.admix_tc_probe(a.ctypes.data, b.ctypes.data, d.ctypes.data, nsteps, a_in_tmem)
    assert rc == 0, rc
    return d.astype(np.float64)


def test_products_and_small_sums_are_exact_from_either_operand_source(oa):
    rng = np.random.default_rng(3)
    A = rng.integers(-8, 9, size=(128, 64)).astype(np.float32)
    B = rng.integers(-8, 9, size=(16, 64)).astype(np.float32)
    for nsteps in (1, 2, 3, 4):
        ref = A[:, :16 * nsteps].astype(np.float64) @ B[:, :16 * nsteps].astype(np.float64).T
        d_smem = _run(oa, A, B, nsteps, 0)
        d_tmem = _run(oa, A, B, nsteps, 1)
        assert np.array_equal(d_smem, ref), nsteps
        assert np.array_equal(d_tmem, ref), nsteps


def test_fp32_accumulation_truncates_toward_zero(oa):
    """Row r: base + f ulp with the small part in the same MMA (column 0) or in the next MMA
    (column 1); columns 2 and 3 the negated sums."""
    cases = [(1.0, 0.75, 0), (1.0, 1.5, 1), (1.0, 2.5, 2), (1.5, 0.75 * 1.5, 1), (1.5, 2.5 * 1.5, 3),
             (1.0, 0.5, 0), (1.5, 1.5 * 1.5, 2)]
    A = np.zeros((128, 64), np.float32)
    B = np.zeros((16, 64), np.float32)
    for r, (base, f, _) in enumerate(cases):
        A[r, 0] = base
        A[r, 1] = f * ULP1          # same MMA
        A[r, 16] = f * ULP1         # next MMA
    B[0, 0:2] = 1.0
    B[1, 0] = 1.0; B[1, 16] = 1.0
    B[2, 0:2] = -1.0
    B[3, 0] = -1.0; B[3, 16] = -1.0
    d = _run(oa, A, B, 2)
    for r, (base, f, kept) in enumerate(cases):
        for col, sign in ((0, 1), (1, 1), (2, -1), (3, -1)):
            got_ulps = (sign * d[r, col] - base) / ULP1
            assert got_ulps == kept, (base, f, col, got_ulps)


def test_spread_products_never_round_up(oa):
    rng = np.random.default_rng(5)
    errs = []
    for spread in (2.0, 4.0, 8.0):
        A = np.zeros((128, 64), np.float32)
        B = np.zeros((16, 64), np.float32)
        a = (10.0 ** (-spread * rng.random((128, 16)))).astype(np.float32)
        A[:, :16] = (a.view(np.uint32) & 0xFFFF0000).view(np.float32)
        b = (rng.random((16, 16)) * 0.9 + 0.1).astype(np.float32)
        B[:, :16] = (b.view(np.uint32) & 0xFFFF0000).view(np.float32)
        d = _run(oa, A, B, 1)
        exact = A[:, :16].astype(np.float64) @ B[:, :16].astype(np.float64).T
        errs.append((d - exact) / exact)
    errs = np.concatenate(errs)
    assert errs.max() <= 0.0
    assert errs.mean() < 0.0
    assert np.abs(errs).max() < 4 * 2.0 ** -23
