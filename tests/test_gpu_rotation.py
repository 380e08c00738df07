"""Rotation-based M2L of the FP64 evaluate (hfmm_b200/rotation.py, m2l_rotation.cu)
on a B200: the same plan's evaluate with the rotation M2L against its evaluate with
the dense M2L tables (the difference is the multipole truncation at order P, largest
at the nearest face displacements), both against the direct sum, bit-identical
repeats, the dense path restored bit for bit when the rotation is switched off, and
the mixed-precision evaluate untouched by it."""
import numpy as np
import pytest

import oracle as O
from cases import complex_uniform, clustered

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name,fn,n,k,P,bar", [
    ("uniform_k5_P20", complex_uniform, 4000, 5.0, 20, 2e-5),
    ("uniform_k5_P28", complex_uniform, 4000, 5.0, 28, 2e-6),
    ("clustered_k8_P24", clustered, 3000, 8.0, 24, 2e-5),
])
def test_rotation_m2l_matches_the_dense_tables(name, fn, n, k, P, bar):
    import torch
    import hfmm_b200
    from hfmm_b200 import rotation
    pos, q = fn(n)
    if not np.iscomplexobj(q):
        q = q + 1j * np.cos(np.arange(n))
    st = hfmm_b200.setup(pos, k, p=6, N_max=32)
    qt = torch.as_tensor(q, device="cuda")
    dense = [x.cpu().numpy() for x in hfmm_b200.evaluate_field(st, qt)]
    mixed = [x.cpu().numpy() for x in hfmm_b200.evaluate_field(st, qt, precision=hfmm_b200.PREC_MIXED)]
    rotation.enable(st, P)
    rot = [x.cpu().numpy() for x in hfmm_b200.evaluate_field(st, qt)]
    again = [x.cpu().numpy() for x in hfmm_b200.evaluate_field(st, qt)]
    assert all(np.array_equal(a, b) for a, b in zip(rot, again))
    for a, b in zip(rot, dense):
        assert np.isfinite(a).all()
        assert O.relative_error(a, b) < bar, (name, O.relative_error(a, b))
    # both against the direct sum on sampled targets: the rotation adds no more than
    # its truncation to the dense path's error
    tg = np.random.default_rng(3).choice(n, 200, replace=False)
    d_phi, d_E = hfmm_b200.direct(st, q, tg, field=True)
    for a, b, d in ((rot[0], dense[0], d_phi), (rot[1], dense[1], d_E)):
        e_rot, e_dense = O.relative_error(a[tg], d), O.relative_error(b[tg], d)
        assert e_rot <= e_dense + bar
    m2 = [x.cpu().numpy() for x in hfmm_b200.evaluate_field(st, qt, precision=hfmm_b200.PREC_MIXED)]
    assert all(np.array_equal(a, b) for a, b in zip(m2, mixed))
    rotation.disable(st)
    back = [x.cpu().numpy() for x in hfmm_b200.evaluate_field(st, qt)]
    assert all(np.array_equal(a, b) for a, b in zip(back, dense))
    st.close()


def test_rotation_refuses_other_kernels_and_bad_orders():
    import hfmm_b200
    from hfmm_b200 import _lib, kernels, rotation
    pos, q = complex_uniform(1500)
    st = hfmm_b200.kernel_setup(pos, kernels.yukawa(2.0), p=4, N_max=32)
    with pytest.raises(ValueError):
        rotation.enable(st, 10)
    st.close()
    st = hfmm_b200.setup(pos, 3.0, p=4, N_max=32)
    with pytest.raises(ValueError):
        _lib.check(_lib.lib.hfmm_plan_set_m2l_rotation(st.handle, 41, None, 0, None, None, None, 0))
    with pytest.raises(hfmm_b200.HFMMError):   # level operators before the order
        _lib.check(_lib.lib.hfmm_plan_set_rotation_level(st.handle, 0, 2, None, None, None, 1.0))
    st.close()
