"""Moving geometry (hfmm_b200.moving, hfmm_plan_rebuild): a plan built in a fixed
domain cube at a fixed depth rebuilds its tree, lists and schedules in place for
moved points and keeps its operator tables. The rebuilt plan must give, bit for bit,
what a plan built from scratch for the moved points in the same domain gives (same
tree, same lists, same tables); a point outside the domain is refused before
anything changes; the certified evaluator refits the domain then. Accuracy of the
moved evaluate against the FP64 direct sum at the FMM's own level."""
import numpy as np
import pytest

import oracle as O
from cases import complex_uniform, sphere_clusters

pytestmark = pytest.mark.gpu


def _drift(pos, t, seed=3):
    rng = np.random.default_rng(seed)
    v = rng.normal(size=pos.shape)
    return pos + 0.01 * t * v / np.linalg.norm(v, axis=1, keepdims=True)


def test_rebuild_equals_a_fresh_plan_in_the_same_domain():
    import hfmm_b200
    from hfmm_b200 import moving
    pos0, q = complex_uniform(6000)
    mp = moving.MovingPlan(pos0, 5.0, p=5, N_max=24, headroom=0.2)
    assert mp.builds == 1
    for t in (1, 2, 3):
        x = _drift(pos0, t)
        assert mp.inside(x)
        phi, E = mp.evaluate_field(x, q)
        cert = mp.certificate
        assert cert["inside_domain"] and not cert["plan_rebuilt"]
        fresh = hfmm_b200.setup(x, 5.0, p=5, N_max=24, max_depth=mp.depth, domain=mp.domain)
        f_phi, f_E = hfmm_b200.evaluate_field(fresh, q)
        assert np.array_equal(phi, f_phi) and np.array_equal(E, f_E)
        ta, tb = mp.state.tree(), fresh.tree()
        for key in ta:
            assert np.array_equal(ta[key], tb[key]), key
        for key in ("V", "U", "near", "W", "X"):
            assert np.array_equal(mp.state.pairs(key), fresh.pairs(key)), key
        fresh.close()
        tg = np.random.default_rng(t).choice(len(x), 300, replace=False)
        ref = O.direct(x, q, 5.0, tg)
        assert O.relative_error(phi[tg], ref) < 5e-4
    assert mp.builds == 1 and mp.moves == 3
    mp.close()


def test_points_leaving_the_domain_are_refused_then_refitted():
    import hfmm_b200
    from hfmm_b200 import moving
    pos0, q = sphere_clusters(5000)
    mp = moving.MovingPlan(pos0, 8.0, p=5, N_max=24, headroom=0.1)
    before = hfmm_b200.evaluate_field(mp.state, q)
    far = pos0.copy()
    far[0] += 5.0   # one point far outside the cube
    with pytest.raises(hfmm_b200.HFMMError) as ei:
        hfmm_b200.rebuild(mp.state, far)
    assert ei.value.code == -4
    again = hfmm_b200.evaluate_field(mp.state, q)   # the plan is unchanged
    assert np.array_equal(before[0], again[0]) and np.array_equal(before[1], again[1])
    phi, E = mp.evaluate_field(far, q)               # the evaluator refits the domain
    assert mp.certificate["plan_rebuilt"] and mp.builds == 2
    fresh = hfmm_b200.setup(far, 8.0, p=5, N_max=24, max_depth=mp.depth, domain=mp.domain)
    f_phi, f_E = hfmm_b200.evaluate_field(fresh, q)
    assert np.array_equal(phi, f_phi) and np.array_equal(E, f_E)
    fresh.close()
    mp.close()


def test_rebuild_needs_a_fixed_domain_plan():
    import hfmm_b200
    pos, q = complex_uniform(2000)
    st = hfmm_b200.setup(pos, 3.0, p=4, N_max=16)
    with pytest.raises(hfmm_b200.HFMMError) as ei:
        hfmm_b200.rebuild(st, pos)
    assert ei.value.code == -3
    st.close()


def test_moving_mixed_low_rank_plan():
    """The mixed evaluate's low-rank tables and folded operators survive the rebuild:
    the moved mixed result equals a fresh plan's and stays at the mixed bar of the
    FP64 evaluate on the same plan."""
    import torch
    import hfmm_b200
    from hfmm_b200 import moving
    pos0, q = complex_uniform(20000)
    mp = moving.MovingPlan(pos0, 6.0, p=6, N_max=32, headroom=0.2,
                           precision=hfmm_b200.PREC_MIXED, m2l_compress=1e-7)
    x = _drift(pos0, 2)
    phi, E = mp.evaluate_field(x, q)
    fresh = hfmm_b200.setup(x, 6.0, p=6, N_max=32, max_depth=mp.depth, domain=mp.domain,
                            m2l_compress=1e-7)
    f_phi, f_E = hfmm_b200.evaluate_field(fresh, q, hfmm_b200.PREC_MIXED)
    assert np.array_equal(phi, f_phi) and np.array_equal(E, f_E)
    d_phi, d_E = hfmm_b200.evaluate_field(fresh, q, hfmm_b200.PREC_FP64)
    assert O.relative_error(phi, d_phi) < 2e-6 and O.relative_error(E, d_E) < 2e-6
    fresh.close()
    mp.close()
