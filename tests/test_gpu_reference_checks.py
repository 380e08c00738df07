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
