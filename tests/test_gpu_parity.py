"""Parity of the CUDA path with the reference and the oracle.

Integer work (tree arrays, particle slots, interaction lists) must match bit
for bit; potentials and fields must match to a relative L2 of 1e-12 (float64
everywhere; the bar of the plain path). Cases: the committed golden fixtures,
which are the reference's own outputs (tests/golden/make_golden.py runs its
code on a NumPy stand-in for JAX), and live oracle runs on further clouds
(plane / depth refinement, tiny N, duplicates, explicit max_depth, the C3
shape), whose inputs tests/golden/edge/ pins the oracle on against the
reference in the same way."""
import glob
import os

import numpy as np
import pytest

import oracle as O
from cases import (uniform, clustered, plane, with_duplicates, complex_uniform, sphere_clusters,
                   sphere_and_clusters)

pytestmark = pytest.mark.gpu
TOL = 1e-12
GOLD = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "*.npz")))


def load(path):
    with np.load(path) as z:
        return {k: z[k] for k in z.files}


def _setup(pos, k, p, nmax, md):
    import hfmm_b200
    return hfmm_b200.setup(pos, k, p=p, N_max=nmax, max_depth=md)


def _compare_tree(st, s_or_g, oracle_state=True):
    t = st.tree()
    nb = st.info["n_boxes"]
    for key in ("m_id", "p_id", "lvls", "counts", "is_leaf"):
        ref = s_or_g[key][:nb] if oracle_state else s_or_g[key]
        assert len(ref) == nb and np.array_equal(t[key], ref), key
    if oracle_state:
        assert not (s_or_g["lvls"][nb:] > 0).any()
    assert np.array_equal(t["sort_idx"], s_or_g["sort_idx"])
    ref_pil = s_or_g["pil"][:nb]
    assert np.array_equal(st.pil(), ref_pil)


def _compare_lists(st, ref):
    for key, rk in (("V", "V"), ("U", "U"), ("near", "near"), ("W", "W"), ("X", "X")):
        r = ref[rk]
        r = np.empty((0, 2), np.int32) if r is None else r
        got = st.pairs(key)
        assert got.shape == r.shape and np.array_equal(got, r), key


@pytest.mark.parametrize("path", GOLD, ids=[os.path.basename(p)[:-4] for p in GOLD])
def test_golden(path):
    import hfmm_b200
    g = load(path)
    md = int(g["max_depth"])
    st = _setup(g["positions"], float(g["k"]), int(g["p"]), int(g["N_max"]), None if md < 0 else md)
    assert st.info["max_depth"] == int(g["realised_depth"])
    assert st.info["maxleaf"] == int(g["maxleaf"])
    assert st.info["max_boxes"] == int(g["max_boxes"])
    assert st.info["domain_extent"] == float(g["domain_extent"])
    _compare_tree(st, g, oracle_state=False)
    _compare_lists(st, g)
    q = g["charges"]
    if "E" in g:
        phi, E = hfmm_b200.evaluate_field(st, q)
        assert O.relative_error(E, g["E"]) < TOL
    else:
        phi = hfmm_b200.evaluate(st, q)
    assert phi.dtype == np.complex128
    assert O.relative_error(phi, g["phi"]) < TOL


LIVE = [
    ("plane", plane, 3000, 3.0, 4, 16, None),
    ("dups", with_duplicates, 1200, 2.0, 4, 16, None),
    ("tiny1", uniform, 1, 1.0, 3, 16, None),
    ("tiny2", uniform, 2, 1.0, 3, 16, None),
    ("tiny17", uniform, 17, 1.0, 3, 16, None),
    ("depth5", uniform, 3000, 4.0, 4, 8, 5),
    ("clustered_d3", clustered, 2500, 6.0, 5, 32, 3),
    ("sphere", sphere_clusters, 4000, 10.0, 4, 24, None),
    # the C3 shape: deep, adaptive, and the tree buffer doubles once (6096 -> 12192)
    ("c3_shape", sphere_and_clusters, 8000, 20.0, 4, 16, None),
]
# Tolerance per case: 1e-12, except where the FP64 method's own rounding floor is
# higher. On the C3 shape (depth 6, k = 20) the oracle's two summation orders (one
# decode per site or one fused decode per box) already differ by 2.3e-12 on the real
# charges: the damped sin-component decodes (eps_rel 1e-12) amplify summation-order
# differences. The bar there is 1e-11, about four times that floor (which the test
# re-measures); the CUDA path measured 3.7e-12.
CASE_TOL = {"c3_shape": 1e-11}


@pytest.mark.parametrize("name,fn,n,k,p,nmax,md", LIVE, ids=[c[0] for c in LIVE])
def test_live_oracle(name, fn, n, k, p, nmax, md):
    import hfmm_b200
    tol = CASE_TOL.get(name, TOL)
    pos, q = fn(n)
    ref = O.setup(pos, k, p=p, N_max=nmax, max_depth=md)
    st = _setup(pos, k, p, nmax, md)
    s = ref[0]
    assert st.info["max_depth"] == s["max_depth"] and st.info["maxleaf"] == s["maxleaf"]
    assert st.info["max_boxes"] == s["max_boxes"]
    _compare_tree(st, s)
    _compare_lists(st, dict(V=s["V"], U=s["U"], near=s["dir_cnct"], W=s["W"], X=s["X"]))
    qc = q if np.iscomplexobj(q) else q + 0.5j * np.cos(np.arange(n))
    if s["domain_extent"] == 0.0:
        # all points coincide: every pair is a self pair, the potential is exactly 0.
        # (The reference's level tables are assembled at scale 0 there and are NaN.)
        phi, E = hfmm_b200.evaluate_field(st, qc)
        assert np.all(phi == 0) and np.all(E == 0)
        return
    phi_r = hfmm_b200.evaluate(st, qc.real)
    ref_r = O.evaluate(ref, qc.real)
    if tol > TOL:   # the floor that justifies the wider bar is still there, and below it
        fused = O.evaluate_complex(ref, qc.real, fused_decode=True)
        floor = O.relative_error(fused, ref_r)
        assert 1e-13 < floor < tol / 2, floor
    assert O.relative_error(phi_r, ref_r) < tol
    phi, E = hfmm_b200.evaluate_field(st, qc)
    rphi, rE = O.evaluate_complex(ref, qc, field=True)
    assert O.relative_error(phi, rphi) < tol
    assert O.relative_error(E, rE) < tol


def test_c1_shape_against_oracle():
    """The CPU-runnable workload's shape at reduced N: complex charges, potential +
    field, k = 2 pi, p = 8, leaf size 64 (depth 3)."""
    import hfmm_b200
    pos, q = complex_uniform(6000)
    k = 2 * np.pi
    ref = O.setup(pos, k, p=8, N_max=64, max_depth=3)
    st = _setup(pos, k, 8, 64, 3)
    phi, E = hfmm_b200.evaluate_field(st, q)
    rphi, rE = O.evaluate_complex(ref, q, field=True)
    assert O.relative_error(phi, rphi) < TOL
    assert O.relative_error(E, rE) < TOL
