"""The allocation-free direct-sum entry point, hfmm_direct_noalloc.

It serves callers that cannot allocate device memory mid-run (code running
inside a JAX/XLA process, whose allocator owns the GPU memory): its scratch is a
fixed device array inside the library. Through the C ABI it must give the same
result as the allocating hfmm_direct, on two calls in a row (the array is reused
and keeps the previous call's contents), and refuse sizes beyond its limit.
This file is collected last so that a failure here leaves every other test run.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
TOL = 1e-13     # the tolerance of the direct-sum tests (test_gpu_reference_checks.py)


def _rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def _inputs(n, n_t, seed):
    import torch
    rng = np.random.default_rng(seed)
    pos = torch.as_tensor(rng.uniform(size=(n, 3))).cuda()
    q_re = torch.as_tensor(rng.normal(size=n)).cuda()
    q_im = torch.as_tensor(rng.normal(size=n)).cuda()
    tg = torch.as_tensor(rng.choice(n, n_t, replace=False).astype(np.int32)).cuda()
    return pos, q_re, q_im, tg


def _call(fn, pos, q_re, q_im, tg, k):
    import torch
    from hfmm_b200 import _lib
    n, n_t = pos.shape[0], tg.shape[0]
    phi = torch.empty(n_t, dtype=torch.complex128, device="cuda")
    E = torch.empty((n_t, 3), dtype=torch.complex128, device="cuda")
    s = torch.cuda.current_stream().cuda_stream
    rc = fn(pos.data_ptr(), q_re.data_ptr(), q_im.data_ptr(), n, tg.data_ptr(), n_t, k,
            phi.data_ptr(), E.data_ptr(), s)
    assert rc == 0, _lib.lib.hfmm_last_error()
    torch.cuda.synchronize()
    return phi.cpu().numpy(), E.cpu().numpy()


def test_noalloc_matches_allocating_entry_point_twice():
    from hfmm_b200 import _lib
    lib = _lib.load()
    k = 9.0
    pos, q_re, q_im, tg = _inputs(20000, 1024, 11)
    ref_phi, ref_E = _call(lib.hfmm_direct, pos, q_re, q_im, tg, k)
    for _ in range(2):
        phi, E = _call(lib.hfmm_direct_noalloc, pos, q_re, q_im, tg, k)
        assert _rel(phi, ref_phi) < TOL and _rel(E, ref_E) < TOL
    # a different, smaller problem right after: stale scratch must not leak in
    pos2, r2, i2, tg2 = _inputs(3000, 77, 12)
    a = _call(lib.hfmm_direct, pos2, r2, i2, tg2, 2.5)
    b = _call(lib.hfmm_direct_noalloc, pos2, r2, i2, tg2, 2.5)
    assert _rel(b[0], a[0]) < TOL and _rel(b[1], a[1]) < TOL


def test_noalloc_rejects_sizes_beyond_its_scratch():
    import torch
    from hfmm_b200 import _lib
    lib = _lib.load()
    n, n_t = 1000, 131073
    pos = torch.zeros((n, 3), dtype=torch.float64, device="cuda")
    q = torch.zeros(n, dtype=torch.float64, device="cuda")
    tg = torch.zeros(n_t, dtype=torch.int32, device="cuda")
    phi = torch.empty(n_t, dtype=torch.complex128, device="cuda")
    rc = lib.hfmm_direct_noalloc(pos.data_ptr(), q.data_ptr(), None, n, tg.data_ptr(), n_t, 1.0,
                                 phi.data_ptr(), None, torch.cuda.current_stream().cuda_stream)
    assert rc == -4
    assert b"131072" in lib.hfmm_last_error()


def test_noalloc_out_of_range_target_then_good_call():
    """A target index equal to n is skipped by the kernel's bounds check and the
    call returns HFMM_ERR_ARG; the shared error word is cleared per call, so the
    next good call returns 0 with the allocating entry point's result."""
    import torch
    from hfmm_b200 import _lib
    lib = _lib.load()
    n = 2000
    pos, q_re, q_im, tg = _inputs(n, 64, 13)
    bad = tg.clone()
    bad[5] = n
    phi = torch.empty(64, dtype=torch.complex128, device="cuda")
    s = torch.cuda.current_stream().cuda_stream
    rc = lib.hfmm_direct_noalloc(pos.data_ptr(), q_re.data_ptr(), q_im.data_ptr(), n,
                                 bad.data_ptr(), 64, 3.0, phi.data_ptr(), None, s)
    assert rc == -1
    assert b"out of range" in lib.hfmm_last_error()
    ref = _call(lib.hfmm_direct, pos, q_re, q_im, tg, 3.0)
    got = _call(lib.hfmm_direct_noalloc, pos, q_re, q_im, tg, 3.0)
    assert _rel(got[0], ref[0]) < TOL and _rel(got[1], ref[1]) < TOL
