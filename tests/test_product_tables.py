"""The library's host table builder (hfmm_b200.operators) produces exactly the
oracle's tables (restating kifmm/operators.py:72-99, 276-425, 572-641 and
kifmm/surfaces.py:40-85): same surfaces, and bit-identical decode factors, M2M,
L2L and M2L matrices for every level the library consumes."""
import numpy as np
import pytest

import oracle as O
from hfmm_b200 import operators as H


@pytest.mark.parametrize("p", [2, 3, 4, 6])
def test_surfaces(p):
    for r in (H.R_EQUIV, H.R_CHECK, 1.0):
        a, b = H.surface_pts(p, r), O.surface_pts(p, r)
        assert a.shape == (H.n_surf(p), 3) and np.array_equal(a, b)


@pytest.mark.parametrize("p,md,k,imag,eps", [(3, 3, 2.0, False, 1e-7), (4, 4, 6.0, True, 1e-12),
                                              (5, 3, 0.0, False, 1e-7)])
def test_level_tables_bitwise(p, md, k, imag, eps):
    extent = 0.987654321
    ref = O.build_operators_leveled(p, md, extent, O.helmholtz_G_np(k, imag), eps)
    for level in range(2, md + 1):
        t = H.level_tables(p, level, md, extent, k, imag, eps)
        for i in range(3):
            assert np.array_equal(t["F_up"][i], ref["F_up_lv"][i][level])
            assert np.array_equal(t["F_dn"][i], ref["F_dn_lv"][i][level])
        assert np.array_equal(t["M2L_K"], ref["M2L_K_lv"][level])
        if level < md:
            assert np.array_equal(t["M2M_K"], ref["M2M_K_lv"][level])
        else:
            assert t["M2M_K"] is None
        if level >= 3:
            assert np.array_equal(t["L2L_K"], ref["L2L_K_lv"][level - 1])
        else:
            assert t["L2L_K"] is None
