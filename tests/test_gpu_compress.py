"""The compressed M2L of the mixed path (K_d ~ U C_d U^T per level, U from the
level's M2L Gram matrix, with the decodes folded into the neighbouring operators):
close to the dense mixed M2L, within tolerance of the FP64 direct sum, and without
effect on the FP64 evaluate."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _problem(n, seed, clustered=False):
    rng = np.random.default_rng(seed)
    if clustered:
        c = rng.uniform(0.2, 0.8, (4, 3))
        x = np.clip(c[rng.integers(0, 4, n)] + 0.04 * rng.standard_normal((n, 3)), 0, 1)
    else:
        x = rng.random((n, 3))
    q = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    return x, q


def _rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.mark.parametrize("clustered", [False, True])
def test_compressed_mixed_m2l_matches_dense(clustered):
    import hfmm_b200 as hf
    x, q = _problem(60000, 3, clustered)
    k = 8.0
    dense = hf.setup(x, k, p=8, N_max=64)
    comp = hf.setup(x, k, p=8, N_max=64, m2l_compress=1e-8)
    ranks = comp.m2l_ranks
    assert all(1 <= r <= comp.info["n_s"] for r in ranks.values())
    md = comp.max_depth
    assert all(ranks[(1, l)] < ranks[(0, l)] for l in range(2, md + 1))   # sin is smoother
    if clustered:   # the folded tables' W (M2P) and X (P2L) branches run
        assert comp.info["n_w"] > 0 and comp.info["n_x"] > 0
    pd, ed = hf.evaluate_field(dense, q, hf.PREC_MIXED)
    pc, ec = hf.evaluate_field(comp, q, hf.PREC_MIXED)
    assert _rel(pc, pd) < 3e-7 and _rel(ec, ed) < 3e-7
    tg = np.random.default_rng(1).choice(len(x), 300, replace=False)
    dphi, dE = hf.direct(comp, q, tg, field=True)
    assert _rel(pc[tg], dphi) < 2e-6 and _rel(ec[tg], dE) < 2e-6
    # real charges take the R = 1 layout of the compressed buffers
    qr = q.real.copy()
    assert _rel(hf.evaluate(comp, qr, hf.PREC_MIXED), hf.evaluate(dense, qr, hf.PREC_MIXED)) < 3e-7
    # the FP64 evaluate does not use the compressed tables
    assert np.array_equal(hf.evaluate_field(comp, q)[0], hf.evaluate_field(dense, q)[0])
    dense.close()
    comp.close()


def test_compression_argument_checks():
    import hfmm_b200 as hf
    from hfmm_b200 import _lib
    x, q = _problem(3000, 4)
    st = hf.setup(x, 3.0, p=6, N_max=32)
    U = torch.zeros((st.info["n_s"], 4), dtype=torch.float64, device="cuda")
    C = torch.zeros((316, 4, 4), dtype=torch.float64, device="cuda")
    with pytest.raises(ValueError):   # rank beyond n_s
        _lib.check(_lib.lib.hfmm_plan_set_m2l_compressed(st.handle, 0, 2, st.info["n_s"] + 1,
                                                          U.data_ptr(), C.data_ptr()))
    with pytest.raises(ValueError):   # level out of range
        _lib.check(_lib.lib.hfmm_plan_set_m2l_compressed(st.handle, 0, 1, 4, U.data_ptr(),
                                                          C.data_ptr()))
    host = np.zeros(16)
    with pytest.raises(ValueError):   # host pointer
        _lib.check(_lib.lib.hfmm_plan_set_m2l_compressed(st.handle, 0, 2, 4, host.ctypes.data,
                                                          C.data_ptr()))
    st.close()
