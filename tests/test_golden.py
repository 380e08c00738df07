"""The oracle reproduces the reference's own outputs, stored as golden fixtures
(tests/golden/*.npz, made by tests/golden/make_golden.py, which runs the
reference's Python code on a NumPy stand-in for JAX): tree arrays, particle
slots, the V/U/near/W/X lists and the sizes (box buffer, depth, widest leaf,
domain extent) bit for bit; potentials and fields to a relative L2
of 1e-12.

The float bar is the parity bar of the plain path, not tighter: the reference
and the oracle sum the same terms in different orders (per pair in `lax.map`
batches against grouped by displacement), and the sin component's damped
decodes (eps_rel 1e-12) amplify that to a few 1e-13 (measured at most 3.6e-13,
on cplx2000_k8_p6_d4). Two summation orders inside the oracle differ by as much
(`test_oracle_rounding_floor`).

Edge fixture tiny1 (one point): the domain extent is 0 and the reference
assembles its level tables at scale 0, so its potential is NaN. The oracle
follows it there; the CUDA path deliberately returns the exact answer, 0 (the
sum over j != i is empty), which tests/test_gpu_parity.py checks."""
import glob
import os

import numpy as np
import pytest

import oracle as O

TOL = 1e-12
# The C3 shape (depth 6, k = 20): the oracle's two summation orders differ by
# 2.3e-12 there, and the reference's order by 2.5e-12; the bar is 1e-11, with
# the floor re-measured below (as in tests/test_gpu_parity.py).
CASE_TOL = {"c3shape8000_k20_p4": 1e-11}
GOLD = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "*.npz")))
EDGE = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "edge", "*.npz")))
# expansion order 12 (n_s = 728): the reference's own outputs; the p12/oracle_* files
# are the oracle's, at sizes the reference cannot reach on the stand-in
P12 = sorted(p for p in glob.glob(os.path.join(os.path.dirname(__file__), "golden", "p12", "*.npz"))
             if not os.path.basename(p).startswith("oracle_"))


def load(path):
    with np.load(path) as z:
        return {k: z[k] for k in z.files}


@pytest.mark.parametrize("path", GOLD + EDGE + P12,
                         ids=[os.path.basename(p)[:-4] for p in GOLD + EDGE + P12])
@pytest.mark.filterwarnings("ignore:invalid value encountered in divide:RuntimeWarning")  # tiny1
def test_oracle_reproduces_golden(path):
    g = load(path)
    md = int(g["max_depth"])
    st = O.setup(g["positions"], float(g["k"]), p=int(g["p"]), N_max=int(g["N_max"]),
                 max_depth=None if md < 0 else md)
    s = st[0]
    nb = len(g["m_id"])
    assert s["max_boxes"] == int(g["max_boxes"]) and s["max_depth"] == int(g["realised_depth"])
    assert s["maxleaf"] == int(g["maxleaf"]) and s["domain_extent"] == float(g["domain_extent"])
    assert not (s["lvls"][nb:] > 0).any()
    for key in ("m_id", "p_id", "lvls", "counts", "is_leaf", "pil"):
        assert np.array_equal(s[key][:nb], g[key]), key
    assert np.array_equal(s["sort_idx"], g["sort_idx"])
    for key, sk in (("V", "V"), ("U", "U"), ("near", "dir_cnct"), ("W", "W"), ("X", "X")):
        mine = np.empty((0, 2), np.int32) if s[sk] is None else s[sk]
        assert mine.shape == g[key].shape and np.array_equal(mine, g[key]), key
    q = g["charges"]
    if float(g["domain_extent"]) == 0.0:
        assert np.isnan(g["phi"]).all() and np.isnan(O.evaluate(st, q)).all()
        return
    tol = CASE_TOL.get(os.path.basename(path)[:-4], TOL)
    if "E" in g:
        phi, E = O.evaluate_complex(st, q, field=True)
        assert O.relative_error(E, g["E"]) < tol
    else:
        phi = O.evaluate(st, q)
    if tol > TOL:
        floor = O.relative_error(O.evaluate_complex(st, q, fused_decode=True), phi)
        assert 1e-13 < floor < tol / 2, floor
    assert O.relative_error(phi, g["phi"]) < tol


def test_fixtures_present():
    assert len(GOLD) >= 6 and len(EDGE) >= 8 and len(P12) >= 2



PHASES = os.path.join(os.path.dirname(__file__), "golden", "phases", "clustered600_k2_p4.npz")


def _surface_potential(x, comp, up, st, k, nb):
    """The potential each box's density makes on its own check surface at its
    level's scale: G(check, equiv) x for upward equivalent densities,
    G(equiv, check) y for downward ones (the matrices the level's pseudoinverse
    factors invert, operators.py:72-99)."""
    s0 = st[0]
    ext, lv = s0["domain_extent"], s0["lvls"][:nb]
    eq, ck = s0["ops"]["equiv_pts"], s0["ops"]["check_pts"]
    G = O.helmholtz_G_np(k, comp == "sin")
    out = np.empty_like(x)
    for level in np.unique(lv):
        sc = ext * 0.5 ** (level + 1)
        K = G(ck * sc, eq * sc) if up else G(eq * sc, ck * sc)
        out[lv == level] = x[lv == level] @ K.T
    return out


def test_oracle_phases_match_the_reference():
    """Each phase's output, as core.evaluate hands it on (core.py:297-335), against
    the reference's own on an adaptive cloud where V, U, W and X are all non-empty,
    for both kernel components: equivalent densities after P2M and M2M, local
    densities after M2L, P2L and L2L, and the L2P, P2P and M2P potentials.

    Densities are compared through the potential they make on their check surface
    (measured 4e-16 to 5e-14). The densities themselves are not a stable quantity
    for the sin component. Its decodes are damped at eps_rel 1e-12, so rounding
    moves the density along near-null directions of the kernel matrix by up to
    1e-5 relative, while the potential does not move. The cos component's
    densities also match directly (measured 1.4e-12)."""
    g = load(PHASES)
    k = float(g["k"])
    st = O.setup(g["positions"], k, p=int(g["p"]), N_max=int(g["N_max"]))
    nb = int(g["n_boxes"])
    assert int((st[0]["lvls"] > 0).sum()) == nb
    assert st[0]["W"] is not None and st[0]["X"] is not None
    for comp, s in (("cos", st[0]), ("sin", st[1])):
        tr = {}
        pot = O.evaluate_setup(s, g["charges"][:, None], trace=tr)[:, 0]
        for key in ("s2m", "m2m", "m2l", "p2l", "l2l"):
            mine, ref = tr[key][:, 0, :], g[f"{comp}_{key}"]
            assert not np.any(mine[nb:]), (comp, key)
            up = key in ("s2m", "m2m")
            err = O.relative_error(_surface_potential(mine[:nb], comp, up, st, k, nb),
                                   _surface_potential(ref, comp, up, st, k, nb))
            assert err < 1e-12, (comp, key, err)
            if comp == "cos":
                assert O.relative_error(mine[:nb], ref) < 1e-11, (comp, key)
        for key in ("l2p", "p2p", "m2p"):
            err = O.relative_error(tr[key][:, 0], g[f"{comp}_{key}"])
            assert err < 1e-12, (comp, key, err)
        assert O.relative_error(pot, g[f"{comp}_potential"]) < 1e-12


C1 = os.path.join(os.path.dirname(__file__), "golden", "c1", "c1_n20000_k2pi_p8.npz")


def test_oracle_matches_the_reference_at_the_cpu_runnable_configuration():
    """20 000 uniform points, complex N(0, 1) charges, k = 2 pi, p = 8, leaf size 64
    (depth 3), potential and field: the oracle's tree and lists equal the
    reference's, and its outputs on the 1024 sampled targets match the reference's
    own to 1e-12 (tests/golden/make_golden.py --c1 made the fixture)."""
    g = load(C1)
    n = 20_000
    rng = np.random.default_rng(42 + n)
    pos = rng.uniform(0.0, 1.0, (n, 3))
    q = rng.normal(size=n) + 1j * rng.normal(size=n)
    assert pos.sum() == g["positions_sum"] and q.sum() == g["charges_sum"]
    st = O.setup(pos, float(g["k"]), p=int(g["p"]), N_max=int(g["N_max"]))
    s = st[0]
    nb = len(g["m_id"])
    assert s["max_boxes"] == int(g["max_boxes"]) and s["max_depth"] == int(g["realised_depth"])
    assert s["maxleaf"] == int(g["maxleaf"]) and s["domain_extent"] == float(g["domain_extent"])
    for key in ("m_id", "p_id", "lvls", "counts", "is_leaf"):
        assert np.array_equal(s[key][:nb], g[key]), key
    assert np.array_equal(s["sort_idx"], g["sort_idx"])
    for key, sk in (("V", "V"), ("U", "U"), ("near", "dir_cnct")):
        assert np.array_equal(s[sk], g[key]), key
    phi, E = O.evaluate_complex(st, q, field=True)
    sample = g["sample"]
    assert O.relative_error(phi[sample], g["phi"]) < TOL
    assert O.relative_error(E[sample], g["E"]) < TOL


TABLES = os.path.join(os.path.dirname(__file__), "golden", "tables", "reference_table_digests.json")


def test_oracle_tables_match_the_reference():
    """The per-level operator tables (kifmm/operators.py:572-641) of the oracle against
    the reference's own build_operators_leveled, two configurations, both kernel
    components. Where the fixture was made all of them were bit-identical (recorded
    in it). Here, where LAPACK and libm may be other builds, the check is: surfaces
    bit for bit (pure arithmetic); kernel matrices on seeded samples to 1e-14 of the
    largest; the damped singular values to 1e-12 of the largest; the singular
    vectors by shape and norm (they are arbitrary within degenerate subspaces)."""
    import json
    with open(TABLES) as f:
        ref = json.load(f)
    mg = _golden_module()
    assert len(ref) == 2 * len(mg.TABLE_CASES)
    for (p, md, ext, k) in mg.TABLE_CASES:
        for imaginary, eps in ((False, 1e-7), (True, 1e-12)):
            r = ref[f"p{p}_md{md}_ext{ext}_k{k}_{'sin' if imaginary else 'cos'}"]
            assert r["oracle_bit_identical_when_made"]
            mine = mg.table_arrays(O.build_operators_leveled(p, md, ext, O.helmholtz_G_np(k, imaginary),
                                                             eps_rel=eps))
            for name, a in mine.items():
                want = r[name]
                dtype, shape = want["digest"].split(" ", 1)[0], want["digest"].split(" ", 1)[1].rsplit(" ", 1)[0]
                assert a.dtype.str == dtype and str(a.shape) == shape, name
                got = np.ascontiguousarray(a).ravel()[want["idx"]]
                vals = np.asarray(want["values"])
                if name in ("equiv_pts", "check_pts"):
                    assert mg.table_digest(a) == want["digest"], name
                elif name.endswith(".U") or name.endswith(".Vt"):
                    assert abs(np.linalg.norm(a) - want["norm"]) <= 1e-12 * want["norm"], name
                elif name.endswith(".d"):
                    assert np.abs(got - vals).max() <= 1e-12 * np.abs(vals).max(), name
                else:
                    assert np.abs(got - vals).max() <= 1e-14 * np.abs(vals).max(), name
                    assert abs(np.linalg.norm(a) - want["norm"]) <= 1e-13 * want["norm"], name


def _golden_module():
    import importlib.util
    path = os.path.join(os.path.dirname(__file__), "golden", "make_golden.py")
    spec = importlib.util.spec_from_file_location("make_golden", path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod
