"""The mixed-precision path (M2L + L2L as split 3xTF32 on tcgen05, FP32
accumulation) against the plain FP64 path on the same plan and against the
FP64 direct sum. Tolerances: mixed vs FP64 relative L2 below 2e-6 (TF32x3
products carry ~2^-22 relative error); mixed vs direct sum no worse than the
FP64 error plus 2e-6."""
import numpy as np
import pytest

import oracle as O
from cases import uniform, complex_uniform, sphere_clusters

pytestmark = pytest.mark.gpu
TOL_VS_FP64 = 2e-6


def _both(st, q, field):
    import hfmm_b200
    if field:
        a = hfmm_b200.evaluate_field(st, q, precision=hfmm_b200.PREC_FP64)
        b = hfmm_b200.evaluate_field(st, q, precision=hfmm_b200.PREC_MIXED)
    else:
        a = (hfmm_b200.evaluate(st, q, precision=hfmm_b200.PREC_FP64),)
        b = (hfmm_b200.evaluate(st, q, precision=hfmm_b200.PREC_MIXED),)
    return a, b


CASES = [
    ("small_real", uniform, 3000, 3.0, 6, 32, None, False),
    ("small_cplx_field", complex_uniform, 5000, 5.0, 6, 32, None, True),
    ("c1_shape", complex_uniform, 20000, 2 * np.pi, 8, 64, None, True),
    ("adaptive", sphere_clusters, 12000, 10.0, 6, 24, None, True),
    # near-field phases k r up to about 10: the P2P's series sin/cos hands over to sincosf
    ("large_phase", complex_uniform, 20000, 60.0, 6, 64, None, True),
]


@pytest.mark.parametrize("name,fn,n,k,p,nmax,md,field", CASES, ids=[c[0] for c in CASES])
def test_mixed_against_fp64_and_direct(name, fn, n, k, p, nmax, md, field):
    import hfmm_b200
    pos, q = fn(n)
    st = hfmm_b200.setup(pos, k, p=p, N_max=nmax, max_depth=md)
    a, b = _both(st, q, field)
    for x, y in zip(a, b):
        assert np.isfinite(y).all()
        assert O.relative_error(y, x) < TOL_VS_FP64
    tg = np.random.default_rng(5).choice(n, min(n, 400), replace=False)
    ref = O.direct(pos, q, k, tg)
    e64 = O.relative_error(a[0][tg], ref)
    emx = O.relative_error(b[0][tg], ref)
    assert emx < e64 + TOL_VS_FP64, (e64, emx)


def test_mixed_is_deterministic():
    import torch
    import hfmm_b200
    pos, q = complex_uniform(8000)
    st = hfmm_b200.setup(pos, 4.0, p=6, N_max=32)
    qt = torch.as_tensor(q, device="cuda")
    r1 = hfmm_b200.evaluate_field(st, qt, precision=hfmm_b200.PREC_MIXED)
    r2 = hfmm_b200.evaluate_field(st, qt, precision=hfmm_b200.PREC_MIXED)
    assert torch.equal(r1[0], r2[0]) and torch.equal(r1[1], r2[1])


def test_grid_sources_match_the_gather():
    """Complete tree levels with complex charges read their compressed densities from
    a dense box grid by strided TMA copies (the 1e6-point workload's path); the gather
    of the same sources per target must give the same result to the FP32 accumulation
    order (the two can split the active displacements into accumulation units
    differently only on tiles at the domain boundary), both within the mixed path's bar
    of the FP64 evaluate."""
    import torch
    import hfmm_b200
    from hfmm_b200 import _lib
    lib = _lib.load()
    pos, q = complex_uniform(60000)
    st = hfmm_b200.setup(pos, 8.0, p=8, N_max=32, m2l_compress=1e-7)
    assert st.max_depth >= 4
    qt = torch.as_tensor(q, device="cuda")
    ref = [x.cpu().numpy() for x in hfmm_b200.evaluate_field(st, qt, precision=hfmm_b200.PREC_FP64)]
    try:
        lib.hfmm_debug_m2l_grid(1)
        grid = [x.cpu().numpy() for x in hfmm_b200.evaluate_field(st, qt, precision=hfmm_b200.PREC_MIXED)]
        lib.hfmm_debug_m2l_grid(0)
        gath = [x.cpu().numpy() for x in hfmm_b200.evaluate_field(st, qt, precision=hfmm_b200.PREC_MIXED)]
    finally:
        lib.hfmm_debug_m2l_grid(1)
    for g, h, r in zip(grid, gath, ref):
        assert np.isfinite(g).all()
        assert O.relative_error(g, h) < 1e-6
        assert O.relative_error(g, r) < TOL_VS_FP64
        assert O.relative_error(h, r) < TOL_VS_FP64
    st.close()


@pytest.mark.parametrize("cplx", [True, False])
def test_plan_queue_matches_per_level_launches(cplx):
    """The plan's own queued M2L (one persistent launch over every level and family,
    hfmm_plan_set_m2l_queue, the default) computes each tile as the per-level launches
    on side streams do: the same results bit for bit, complex and real charges, on a
    depth-4 tree whose complete levels run in grid mode."""
    import torch
    import hfmm_b200
    from hfmm_b200 import _lib
    lib = _lib.load()
    pos, q = complex_uniform(40000)
    if not cplx:
        q = q.real.copy()
    st = hfmm_b200.setup(pos, 6.0, p=6, N_max=32, m2l_compress=1e-7)
    assert st.max_depth >= 4
    qt = torch.as_tensor(q, device="cuda")
    a = hfmm_b200.evaluate_field(st, qt, precision=hfmm_b200.PREC_MIXED)
    _lib.check(lib.hfmm_plan_set_m2l_queue(st.handle, 0))
    b = hfmm_b200.evaluate_field(st, qt, precision=hfmm_b200.PREC_MIXED)
    _lib.check(lib.hfmm_plan_set_m2l_queue(st.handle, 1))
    c = hfmm_b200.evaluate_field(st, qt, precision=hfmm_b200.PREC_MIXED)
    for x, y, z in zip(a, b, c):
        assert torch.equal(x, y) and torch.equal(x, z)
    st.close()
