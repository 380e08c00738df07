"""The reference's test.py assertions (test.py:24-77), run on the CUDA path, plus
the GPU direct-sum referee against the NumPy one and the device error flag."""
import numpy as np
import pytest

import oracle as O
from cases import uniform, clustered, complex_uniform

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n", [256, 640])
@pytest.mark.parametrize("clust", [False, True])
def test_reference_grid_on_gpu(n, clust):
    import hfmm_b200
    pos, q = (clustered if clust else uniform)(n)
    for k in (0.0, 1.0, 3.0):
        ref = O.direct(pos, q, k)
        baseline = None
        for p in (3, 5):
            st = hfmm_b200.setup(pos, k, p=p, N_max=16)
            act = hfmm_b200.evaluate(st, q)
            assert act.dtype == np.complex128 and np.isfinite(act).all()
            errs = np.array([O.relative_error(a, b) for a, b in
                             ((act, ref), (act.real, ref.real), (act.imag, ref.imag))])
            assert max(errs) < (5e-2 if p <= 3 else 5e-3), errs
            np.testing.assert_allclose(hfmm_b200.evaluate(st, -0.5 * q), -0.5 * act,
                                       rtol=1e-10, atol=1e-10)
            if k == 0:
                assert np.count_nonzero(act.imag) == 0
            if baseline is not None:
                assert np.all(errs < np.maximum(0.8 * baseline, 2e-6)), errs
            baseline = errs if baseline is None else baseline


def test_gpu_direct_matches_numpy():
    import hfmm_b200
    pos, q = complex_uniform(3000)
    k = 7.0
    st = hfmm_b200.setup(pos, k, p=3, N_max=64)
    tg = np.random.default_rng(1).choice(3000, 300, replace=False)
    phi, E = hfmm_b200.direct(st, q, tg, field=True)
    assert O.relative_error(phi, O.direct(pos, q, k, tg)) < 1e-13
    assert O.relative_error(E, O.direct_field(pos, q, k, tg)) < 1e-13


def test_torch_in_torch_out_and_repeatability():
    import torch
    import hfmm_b200
    pos, q = complex_uniform(2000)
    st = hfmm_b200.setup(torch.as_tensor(pos), 3.0, p=4, N_max=32)
    qt = torch.as_tensor(q, device="cuda")
    a, Ea = hfmm_b200.evaluate_field(st, qt)
    b, Eb = hfmm_b200.evaluate_field(st, qt)
    assert isinstance(a, torch.Tensor) and a.is_cuda and a.dtype == torch.complex128
    assert torch.equal(a, b) and torch.equal(Ea, Eb)       # deterministic: no atomics


@pytest.mark.parametrize("k", [50.0, 3000.0, 4.0e4, 2.0e5])
def test_referee_phase_range(k):
    """The referee's sin/cos: Cody-Waite reduction against pi/2 and the Taylor series
    up to |k r| = 1e5, sincos beyond (direct.cu). Against NumPy's sin/cos of the same
    FP64 phase, through the C ABI (hfmm_direct). Both sides round k r to FP64 the
    same way up to an ulp of the phase, so the bar grows with the largest phase:
    2e-15 relative x max(k r), plus 1e-13. k = 2e5 reaches k r = 3.4e5."""
    import torch
    from hfmm_b200 import _lib
    lib = _lib.load()
    n, m = 1500, 120
    rng = np.random.default_rng(11)
    pos = rng.random((n, 3))
    q = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    tg = np.sort(rng.choice(n, m, replace=False)).astype(np.int32)
    dev = "cuda"
    p_d = torch.as_tensor(pos.reshape(-1), device=dev)
    qr = torch.as_tensor(q.real.copy(), device=dev)
    qi = torch.as_tensor(q.imag.copy(), device=dev)
    t_d = torch.as_tensor(tg, device=dev)
    phi = torch.empty(m, dtype=torch.complex128, device=dev)
    E = torch.empty((m, 3), dtype=torch.complex128, device=dev)
    _lib.check(lib.hfmm_direct(p_d.data_ptr(), qr.data_ptr(), qi.data_ptr(), n, t_d.data_ptr(), m,
                               k, phi.data_ptr(), E.data_ptr(), None))
    torch.cuda.synchronize()
    d = pos[tg][:, None, :] - pos[None, :, :]
    r = np.sqrt((d ** 2).sum(-1))
    ok = r > 0
    rs = np.where(ok, r, 1.0)
    kr = k * rs
    G = np.where(ok, (np.cos(kr) + 1j * np.sin(kr)) / rs, 0.0)
    W = np.where(ok, (np.cos(kr) + 1j * np.sin(kr)) * (1 - 1j * kr) / rs ** 3, 0.0)
    bar = 2e-15 * k * np.sqrt(3.0) + 1e-13
    assert O.relative_error(phi.cpu().numpy(), G @ q) < bar
    assert O.relative_error(E.cpu().numpy(), np.einsum("ts,tsc,s->tc", W, d, q)) < bar
