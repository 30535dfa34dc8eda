"""admix_loglik_dev_noalloc: the log-likelihood entry point for callers that cannot allocate
device memory (their device memory comes only from a pool they do not control, or they must
not pay cudaMalloc's implicit synchronisation).  It keeps its partial sums in a fixed array
inside libadmix instead of a caller-provided workspace.

Checked through the C ABI against admix_loglik_dev (which takes a workspace) on the same
device arrays, on two calls in a row, at the FP64 tolerance the other parity tests use.  This
file is collected last so a run that stops at the first failure has already run the rest."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-10


def _dev_arrays(oa, I, J, K, seed):
    import torch
    spec = oa.COHORTS["c1"].scaled(I=I, J=J, K=K, seed=seed)
    g, _, _ = oa.make_cohort(spec)
    x = oa.init_x(I, J, K, seed + 1)
    dev = torch.device("cuda:0")
    bed = torch.from_numpy(g.data).to(dev)
    q = torch.from_numpy(np.ascontiguousarray(x[:I])).to(dev)
    p = torch.from_numpy(np.ascontiguousarray(x[I:])).to(dev)
    return bed, q, p


def _ptr(t):
    return C.c_void_p(t.data_ptr())


def test_noalloc_loglik_matches_workspace_entry(oa):
    import torch
    from openadmixture_b200 import _native as N
    lib = N.admix_lib()
    torch.cuda.set_device(0)
    stream = torch.cuda.current_stream().cuda_stream
    for (I, J, K, seed) in ((1203, 20011, 5, 3), (517, 3001, 12, 4)):
        bed, q, p = _dev_arrays(oa, I, J, K, seed)
        nbytes = lib.admix_loglik_dev_workspace(I, J, K)
        work = torch.empty(nbytes, dtype=torch.uint8, device="cuda:0")
        ref = torch.zeros(1, dtype=torch.float64, device="cuda:0")
        assert lib.admix_loglik_dev(_ptr(bed), I, J, K, _ptr(q), _ptr(p), _ptr(ref), _ptr(work), nbytes,
                                    C.c_void_p(stream)) == 0
        torch.cuda.synchronize()
        want = ref.item()
        for call in range(2):
            out = torch.full((1,), float("nan"), dtype=torch.float64, device="cuda:0")
            rc = lib.admix_loglik_dev_noalloc(_ptr(bed), I, J, K, _ptr(q), _ptr(p), _ptr(out), C.c_void_p(stream))
            assert rc == 0, lib.admix_noalloc_last_error()
            torch.cuda.synchronize()
            got = out.item()
            assert abs(got - want) <= FP64_TOL * abs(want), (call, got, want)


def test_noalloc_rejects_cohorts_beyond_the_static_scratch(oa):
    from openadmixture_b200 import _native as N
    lib = N.admix_lib()
    one = C.c_void_p(16)     # never dereferenced: the size check comes first
    I = 1 << 35              # needs far more partial sums than the static array holds
    rc = lib.admix_loglik_dev_noalloc(one, I, 1000, 4, one, one, one, None)
    assert rc == N.ADMIX_ERR_UNSUPPORTED
    assert b"static scratch" in lib.admix_noalloc_last_error()
