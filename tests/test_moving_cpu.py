"""Host logic of the moving-geometry evaluator (hfmm_b200.moving): the domain fit
and the automatic depth, the latter against the oracle's tree builder (the
reference's build_fmm_tree_auto, trees/cubic.py:577-585, before refinement)."""
import numpy as np

import oracle as O
from cases import uniform


def test_fit_domain_contains_the_points_with_headroom():
    from hfmm_b200.moving import fit_domain
    rng = np.random.default_rng(0)
    x = rng.normal(size=(500, 3)) * [1.0, 3.0, 0.5]
    lo, ext = fit_domain(x, 0.15)
    assert ((x >= lo) & (x <= lo + ext)).all()
    assert np.isclose(ext, (x.max(0) - x.min(0)).max() * 1.15)
    c = (x.max(0) + x.min(0)) / 2
    assert np.allclose(lo + ext / 2, c)
    lo1, ext1 = fit_domain(np.zeros((4, 3)), 0.1)   # all points equal: a unit cube
    assert np.isclose(ext1, 1.1)


def test_auto_depth_matches_the_tree_builder():
    from hfmm_b200.moving import auto_depth
    for n, nmax in ((1000, 16), (6000, 24), (20000, 64), (5000, 8)):
        pos, _ = uniform(n)
        _, _, md, maxleaf = O.build_fmm_tree_auto(pos, N_max=nmax)
        if maxleaf <= 2 * nmax:      # no refinement step taken
            assert auto_depth(n, nmax) == md, (n, nmax)
