"""Generate the golden fixtures under tests/golden/ by running the reference itself.

JAX is not installed here and there is no network, so the reference's own
Python code (`HFMM.py` and the `jaxfmm` package) runs on `jax_on_numpy`, a NumPy
stand-in for the part of JAX it calls (eager, host only; see that module for the
JAX semantics it reproduces). Every array in a fixture comes from the
reference's functions, not from this repository's oracle:

* tree: `build_fmm_tree_auto` (trees/cubic.py:530-600) as `core.setup_geometry`
  calls it (m_id, p_id, lvls, counts, is_leaf, sort_idx, max_boxes, depth);
* U list: `build_ulist_eager` (trees/lists.py:857-889), recorded on its way
  into `setup_geometry`;
* particles-in-leaf table, V / W / X lists, near list (`dir_cnct`), maxleaf,
  domain extent: the state that `HFMM.setup` (HFMM.py:55-80) returns;
* potentials: `HFMM.evaluate` (HFMM.py:83-91); complex charges by linearity,
  `evaluate(re) + 1j * evaluate(im)`, since the reference takes real charges only;
* fields (-grad phi): `kifmm.evaluate_setup(state, q, field=True)`
  (kifmm/setup.py:229-261) of each component and each charge column, combined
  as F(re) + 1j * F(im) with F(q) = F_cos(q) + 1j * F_sin(q).

Needs the reference source tree, given as `--reference DIR` or in the
environment variable HFMM0_REFERENCE; run from the repo root:

    python tests/golden/make_golden.py --reference DIR [--edge] [case ...]
    python tests/golden/make_golden.py --reference DIR --p12
    python tests/golden/make_golden.py --reference DIR --kernels
    python tests/golden/make_golden.py --reference DIR --grid
    python tests/golden/make_golden.py --reference DIR --phases
    python tests/golden/make_golden.py --reference DIR --c1
    python tests/golden/make_golden.py --reference DIR --errors
    python tests/golden/make_golden.py --reference DIR --tables

The inputs are the seeded clouds of tests/cases.py.
"""
import argparse
import hashlib
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
sys.path.insert(0, os.path.dirname(HERE))

from cases import (uniform, clustered, sphere_clusters, with_duplicates, complex_uniform,  # noqa: E402
                   plane, sphere_and_clusters)

CASES = {
    # name: (cloud, n, k, p, N_max, max_depth, complex charges + field)
    "uniform640_k3_p5": (uniform, 640, 3.0, 5, 16, None, False),
    "clustered900_k2_p4": (clustered, 900, 2.0, 4, 16, None, True),
    "sphere1500_k5_p4": (sphere_clusters, 1500, 5.0, 4, 20, None, True),
    "uniform256_k0_p3": (uniform, 256, 0.0, 3, 16, None, False),
    "dup500_k1_p3": (with_duplicates, 500, 1.0, 3, 16, None, False),
    "cplx2000_k8_p6_d4": (complex_uniform, 2000, 8.0, 6, 32, 4, True),
}

# Expansion order 12 (tests/golden/p12/), the plain path's order at the 1e6-point
# workload (n_s = 728 surface points, not a multiple of the GEMM tiles): a uniform
# depth-2 cloud and an adaptive depth-4 cloud with W and X lists, k = 10.
P12 = {
    "cplx3000_k10_p12": (complex_uniform, 3000, 10.0, 12, 64, None, True),
    "sphere2000_k10_p12_d4": (sphere_clusters, 2000, 10.0, 12, 32, 4, True),
}

# Other kernels through the reference's Kernel seam (tests/golden/kernels/):
# kifmm.setup(positions, p, N_max, kernel=...) with the exact FP64 near field
# (p2p_mixed=False), potential and field of real charges (kifmm/setup.py:19-261).
# name: (cloud, n, kernel ("yukawa", kappa) or ("laplace", None), p, N_max)
KERNEL_CASES = {
    "yukawa1500_kappa3_p5": (uniform, 1500, ("yukawa", 3.0), 5, 24),
    "yukawa2000_kappa8_p4_clustered": (clustered, 2000, ("yukawa", 8.0), 4, 16),
    "laplace1500_p5": (uniform, 1500, ("laplace", None), 5, 24),
    "laplace2500_p4_sphere": (sphere_clusters, 2500, ("laplace", None), 4, 16),
}


def run_kernels(folder, keep=False):
    """The reference's kifmm.setup / evaluate_setup with its yukawa and LAPLACE kernels."""
    from jaxfmm import kifmm
    from jaxfmm.kernels import LAPLACE, yukawa
    os.makedirs(folder, exist_ok=True)
    for name, (fn, n, (kind, kappa), p, nmax) in KERNEL_CASES.items():
        if keep and os.path.exists(os.path.join(folder, name + ".npz")):
            continue
        t = time.time()
        pos, q = fn(n)
        q = np.real(q)
        kern = LAPLACE if kind == "laplace" else yukawa(kappa)
        s = kifmm.setup(pos, p=p, N_max=nmax, kernel=kern, p2p_mixed=False)
        pot = np.asarray(kifmm.evaluate_setup(s, q))
        fld = np.asarray(kifmm.evaluate_setup(s, q, field=True))
        np.savez_compressed(os.path.join(folder, name + ".npz"), positions=pos, charges=q,
                            kind=kind, kappa=np.float64(kappa or 0.0), p=p, N_max=nmax,
                            realised_depth=int(s["max_depth"]), pot=pot, field=fld)
        print(name, "depth", int(s["max_depth"]), f"{time.time() - t:.0f} s", flush=True)


# Edge cases (tests/golden/edge/): a single point, two points, one box over its
# leaf size, a plane (depth refinement), many duplicates, explicit depths, and the
# C3 shape, where the box buffer overflows once and the build retries doubled.
EDGE = {
    "tiny1": (uniform, 1, 1.0, 3, 16, None, False),
    "tiny2": (uniform, 2, 1.0, 3, 16, None, False),
    "tiny17": (uniform, 17, 1.0, 3, 16, None, False),
    "plane3000_k3_p4": (plane, 3000, 3.0, 4, 16, None, False),
    "dups1200_k2_p4": (with_duplicates, 1200, 2.0, 4, 16, None, False),
    "depth5_3000_k4_p4": (uniform, 3000, 4.0, 4, 8, 5, False),
    "clustered2500_k6_p5_d3": (clustered, 2500, 6.0, 5, 32, 3, False),
    "c3shape8000_k20_p4": (sphere_and_clusters, 8000, 20.0, 4, 16, None, True),
}


def load_reference(path):
    """Import `HFMM` from the reference tree on the NumPy stand-in, with recorders
    on the two builder functions whose outputs `HFMM.setup` does not keep."""
    import jax_on_numpy
    jax_on_numpy.install()
    sys.path.insert(0, path)
    import HFMM
    import jaxfmm.trees as trees

    seen = {}
    tree_auto, ulist = trees.build_fmm_tree_auto, trees.build_ulist_eager

    def record_tree(*a, **k):
        out = tree_auto(*a, **k)
        seen["tree"] = out
        return out

    def record_u(*a, **k):
        u = ulist(*a, **k)
        seen["U"] = np.asarray(u)
        return u

    trees.build_fmm_tree_auto, trees.build_ulist_eager = record_tree, record_u
    return HFMM, seen


def _pairs(x):
    return np.empty((0, 2), np.int32) if x is None else np.asarray(x).astype(np.int32)


def make(HFMM, seen, name, table=CASES, folder=HERE):
    from jaxfmm import kifmm
    fn, n, k, p, nmax, md, cplx = table[name]
    pos, q = fn(n)
    if cplx and not np.iscomplexobj(q):
        q = q + 1j * np.random.default_rng(n).normal(size=n)
    seen.clear()
    state = HFMM.setup(pos, k, p=p, N_max=nmax, max_depth=md)
    s = state[0]
    (tree, mb, depth, maxleaf) = seen["tree"]
    m_id, p_id, lvls, counts, is_leaf, sort_idx = (np.asarray(a) for a in tree[:6])
    nb = int((lvls > 0).sum())
    assert not (lvls[nb:] > 0).any()
    out = dict(positions=pos, charges=q, k=k, p=p, N_max=nmax,
               max_depth=-1 if md is None else md, realised_depth=int(s["max_depth"]),
               maxleaf=int(s["maxleaf"]), max_boxes=int(mb),
               domain_extent=float(s["domain_extent"]),
               m_id=m_id[:nb], p_id=p_id[:nb], lvls=lvls[:nb], counts=counts[:nb],
               is_leaf=is_leaf[:nb], sort_idx=sort_idx.astype(np.int32),
               pil=np.asarray(s["pil"])[:nb], V=_pairs(s["V"]), U=_pairs(seen["U"]),
               near=_pairs(s["dir_cnct"]), W=_pairs(s["W"]), X=_pairs(s["X"]))
    assert int(depth) == out["realised_depth"] and int(maxleaf) == out["maxleaf"]
    for key in ("m_id", "p_id", "lvls", "is_leaf"):
        assert np.array_equal(np.asarray(s[key])[:nb], out[key]), key

    def potential(qr):
        return np.asarray(HFMM.evaluate(state, qr))

    def field(qr):
        fc = np.asarray(kifmm.evaluate_setup(state[0], qr, field=True))
        fs = (np.asarray(kifmm.evaluate_setup(state[1], qr, field=True)) if state[1] is not None
              else np.zeros_like(fc))
        return fc + 1j * fs

    if np.iscomplexobj(q):
        out["phi"] = potential(q.real) + 1j * potential(q.imag)
    else:
        out["phi"] = potential(q)
    if cplx:
        out["E"] = field(q.real) + 1j * field(q.imag)
    os.makedirs(folder, exist_ok=True)
    np.savez_compressed(os.path.join(folder, name + ".npz"), **out)
    return out


def run_test_py_grid(HFMM, folder):
    """The reference's own check script (test.py:24-77) on its default grid,
    uniform and clustered: n in (256, 640), k in (0, 1, 3), p in (3, 5), leaf
    size 16, seed 42 + n. Records the reference's potentials for each case, and
    asserts test.py's checks on them (the error bounds against the direct sum,
    linearity at 1e-10, an exactly-zero imaginary part at k = 0, improvement
    with p)."""
    out = {}
    for clustered_cloud in (False, True):
        for n in (256, 640):
            rng = np.random.default_rng(42 + n)
            positions = rng.uniform(0., 1., (n, 3))
            if clustered_cloud:
                positions[:n // 2] = rng.uniform(.1, .25, (n // 2, 3))
            charges = rng.normal(size=n)
            tag = f"{'clustered' if clustered_cloud else 'uniform'}{n}"
            out[f"{tag}_positions"] = positions
            out[f"{tag}_charges"] = charges
            for k in (0.0, 1.0, 3.0):
                d = positions[:, None, :] - positions[None, :, :]
                r = np.linalg.norm(d, axis=-1)
                direct = np.where(r > 0, np.exp(1j * k * r) / np.where(r > 0, r, 1.), 0.) @ charges
                base = None
                for p in (3, 5):
                    t = time.time()
                    state = HFMM.setup(positions, k, p=p, N_max=16)
                    phi = np.asarray(HFMM.evaluate(state, charges))
                    half = np.asarray(HFMM.evaluate(state, -.5 * charges))
                    errs = np.array([np.linalg.norm(a - b) / (np.linalg.norm(b) or 1.0) for a, b in
                                     ((phi, direct), (phi.real, direct.real), (phi.imag, direct.imag))])
                    assert errs.max() < (5e-2 if p <= 3 else 5e-3), errs
                    np.testing.assert_allclose(half, -.5 * phi, rtol=1e-10, atol=1e-10)
                    if k == 0:
                        assert np.count_nonzero(phi.imag) == 0
                    if base is not None:
                        assert np.all(errs < np.maximum(.8 * base, 2e-6)), errs
                    base = errs if base is None else base
                    key = f"{tag}_k{k:g}_p{p}"
                    out[key + "_phi"] = phi
                    out[key + "_errors"] = errs
                    print(key, "errors", errs, f"{time.time() - t:.0f} s", flush=True)
    os.makedirs(folder, exist_ok=True)
    np.savez_compressed(os.path.join(folder, "test_py_grid.npz"), **out)


# Per-phase outputs (tests/golden/phases/): an adaptive cloud with V, U, W and X
# lists all non-empty, real charges, both kernel components.
PHASE_CASE = (clustered, 600, 2.0, 4, 16)
PHASE_FNS = {"p2m_padded_leveled": "s2m", "m2m_factored_leveled": "m2m", "m2l_leveled": "m2l",
             "p2l_leveled": "p2l", "l2l_factored_leveled": "l2l", "l2p_padded": "l2p",
             "m2p": "m2p"}


def run_phases(HFMM, folder):
    """Record what each phase hands to the next inside the reference's evaluate
    (core.py:297-335): the closures of kifmm/assemble.py:15-89 look their phase
    functions up in that module at call time, and core.evaluate calls
    `eval_direct` from its own namespace, so recorders placed there see every
    phase. Box arrays keep the active boxes' rows (the rest are asserted zero)."""
    import jaxfmm.core as core
    import jaxfmm.kifmm.assemble as assemble
    from jaxfmm import kifmm
    rec = {}

    def recorder(fn, key):
        def wrapped(*a, **k):
            out = fn(*a, **k)
            rec[key] = np.asarray(out)
            return out
        return wrapped

    for name, key in PHASE_FNS.items():
        setattr(assemble, name, recorder(getattr(assemble, name), key))
    core.eval_direct = recorder(core.eval_direct, "p2p")

    fn, n, k, p, nmax = PHASE_CASE
    pos, q = fn(n)
    state = HFMM.setup(pos, k, p=p, N_max=nmax)
    s = state[0]
    assert s["W"] is not None and s["X"] is not None and len(s["V"])
    nb = int((np.asarray(s["lvls"]) > 0).sum())
    out = dict(positions=pos, charges=q, k=k, p=p, N_max=nmax, n_boxes=nb)
    for comp, st in (("cos", state[0]), ("sin", state[1])):
        rec.clear()
        pot = np.asarray(kifmm.evaluate_setup(st, q))
        assert set(rec) == set(PHASE_FNS.values()) | {"p2p"}, sorted(rec)
        for key, val in rec.items():
            if val.shape[0] == np.asarray(s["lvls"]).shape[0]:
                assert not np.any(val[nb:]), key
                val = val[:nb]
            out[f"{comp}_{key}"] = val
        out[f"{comp}_potential"] = pot
        print(comp, {key: v.shape for key, v in rec.items()}, flush=True)
    os.makedirs(folder, exist_ok=True)
    np.savez_compressed(os.path.join(folder, "clustered600_k2_p4.npz"), **out)


def c1_problem():
    """The reference's CPU-runnable configuration: 20 000 points uniform in the unit
    cube, complex N(0, 1) charges, seeded default_rng(42 + N) (test.py:40
    convention: positions, then real and imaginary charge parts), k = 2 pi, p = 8,
    leaf size 64 (auto depth 3), potential and field, checked on 1024 targets
    drawn by default_rng(42 + N + 1)."""
    n = 20_000
    rng = np.random.default_rng(42 + n)
    pos = rng.uniform(0.0, 1.0, (n, 3))
    q = rng.normal(size=n) + 1j * rng.normal(size=n)
    sample = np.sort(np.random.default_rng(42 + n + 1).choice(n, 1024, replace=False))
    return pos, q, 2 * np.pi, 8, 64, sample


def run_c1(HFMM, seen, folder):
    from jaxfmm import kifmm
    pos, q, k, p, nmax, sample = c1_problem()
    t = time.time()
    seen.clear()
    state = HFMM.setup(pos, k, p=p, N_max=nmax)
    s = state[0]
    (tree, mb, depth, maxleaf) = seen["tree"]
    m_id, p_id, lvls, counts, is_leaf, sort_idx = (np.asarray(a) for a in tree[:6])
    nb = int((lvls > 0).sum())
    print("setup", f"{time.time() - t:.0f} s", flush=True)

    def both(qr, field):
        a = np.asarray(kifmm.evaluate_setup(state[0], qr, field=field))
        b = np.asarray(kifmm.evaluate_setup(state[1], qr, field=field))
        return a + 1j * b

    phi = both(q.real, False) + 1j * both(q.imag, False)
    E = both(q.real, True) + 1j * both(q.imag, True)
    print("evaluate", f"{time.time() - t:.0f} s", flush=True)
    out = dict(positions_sum=np.float64(pos.sum()), charges_sum=q.sum(), k=k, p=p, N_max=nmax,
               sample=sample, realised_depth=int(s["max_depth"]), maxleaf=int(s["maxleaf"]),
               max_boxes=int(mb), domain_extent=float(s["domain_extent"]),
               m_id=m_id[:nb], p_id=p_id[:nb], lvls=lvls[:nb], counts=counts[:nb],
               is_leaf=is_leaf[:nb], sort_idx=sort_idx.astype(np.int32),
               V=_pairs(s["V"]), U=_pairs(seen["U"]), near=_pairs(s["dir_cnct"]),
               phi=phi[sample], E=E[sample])
    os.makedirs(folder, exist_ok=True)
    np.savez_compressed(os.path.join(folder, "c1_n20000_k2pi_p8.npz"), **out)


# Invalid inputs of HFMM.setup / HFMM.evaluate (HFMM.py:14-16, 57-64, 86-87).
def _error_cases():
    good = np.random.default_rng(0).uniform(size=(64, 3))
    bad_pos = {"empty": np.zeros((0, 3)), "two_columns": np.zeros((4, 2)),
               "nan": np.array([[0.0, 0.0, np.nan]]), "inf": np.array([[0.0, np.inf, 0.0]]),
               "one_dim": np.zeros(3)}
    cases = {f"positions_{n}": dict(positions=x) for n, x in bad_pos.items()}
    for name, kw in (("p_1", dict(p=1)), ("p_2.5", dict(p=2.5)), ("p_0", dict(p=0)),
                     ("N_max_0", dict(N_max=0)), ("N_max_2.5", dict(N_max=2.5)),
                     ("max_depth_0", dict(max_depth=0)), ("max_depth_1.5", dict(max_depth=1.5)),
                     ("max_depth_-1", dict(max_depth=-1)),
                     ("k_nan", dict(k=np.nan)), ("k_inf", dict(k=np.inf)),
                     ("k_-inf", dict(k=-np.inf))):
        cases[name] = kw
    return good, cases


def run_errors(HFMM, folder):
    """Which exception the reference raises for each invalid input (none of them
    reaches the tree build), and for invalid charges on a small valid state."""
    import json
    good, cases = _error_cases()
    out = {}
    for name, kw in cases.items():
        args = dict(positions=good, k=1.0, p=3, N_max=16, max_depth=None)
        args.update(kw)
        try:
            HFMM.setup(args.pop("positions"), args.pop("k"), **args)
            out[name] = None
        except Exception as e:          # the type is the record
            out[name] = type(e).__name__
    state = HFMM.setup(good, 1.0, p=2, N_max=16)
    for name, q in (("charges_complex", np.ones(64) + 1j), ("charges_short", np.ones(63)),
                    ("charges_two_columns", np.ones((64, 2)))):
        try:
            HFMM.evaluate(state, q)
            out[name] = None
        except Exception as e:
            out[name] = type(e).__name__
    os.makedirs(folder, exist_ok=True)
    with open(os.path.join(folder, "reference_errors.json"), "w") as f:
        json.dump(out, f, indent=1, sort_keys=True)
    print(out)


# Operator tables (kifmm/operators.py:572-641): (p, max_depth, domain extent, k).
TABLE_CASES = ((3, 3, 0.97, 2.0), (5, 2, 1.3, 7.5))
TABLE_KEYS = ("equiv_pts", "check_pts", "M2M_K_lv", "L2L_K_lv", "M2L_K_lv")


def table_digest(a):
    a = np.ascontiguousarray(np.asarray(a))
    return f"{a.dtype.str} {a.shape} " + hashlib.sha256(a.tobytes()).hexdigest()


def table_arrays(t):
    """name -> array of one leveled table set (the reference's dict or the oracle's)."""
    arrs = {key: np.asarray(t[key]) for key in TABLE_KEYS}
    for key in ("F_up_lv", "F_dn_lv"):
        for i, part in enumerate(("U", "d", "Vt")):
            arrs[f"{key}.{part}"] = np.asarray(t[key][i])
    return arrs


def table_summary(a, n_samples=64):
    """Digest, Frobenius norm and seeded sample entries of one table."""
    flat = np.ascontiguousarray(a).ravel()
    idx = np.random.default_rng(flat.size).choice(flat.size, min(n_samples, flat.size),
                                                  replace=False)
    return dict(digest=table_digest(a), norm=float(np.linalg.norm(flat)),
                idx=idx.tolist(), values=flat[idx].tolist())


def run_tables(HFMM, folder):
    """Every per-level table the reference's build_operators_leveled makes
    (surfaces, damped-SVD factors U, d, Vt up and down, M2M, L2L and M2L kernel
    matrices) for both kernel components (eps_rel 1e-7 and 1e-12, HFMM.py:65-77):
    digest, norm and sample entries, and whether the oracle's tables were
    bit-identical on the machine that ran this (the SVD and libm bits may differ
    on another CPU, so the tests compare samples and norms)."""
    import json
    from jaxfmm.kifmm.operators import build_operators_leveled
    sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
    import oracle as O
    out = {}
    for (p, md, ext, k) in TABLE_CASES:
        for imaginary, eps in ((False, 1e-7), (True, 1e-12)):
            t = table_arrays(build_operators_leveled(
                p, md, ext, HFMM.helmholtz_component(k, imaginary), eps_rel=eps))
            mine = table_arrays(O.build_operators_leveled(
                p, md, ext, O.helmholtz_G_np(k, imaginary), eps_rel=eps))
            d = {name: table_summary(a) for name, a in t.items()}
            d["oracle_bit_identical_when_made"] = all(
                mine[name].shape == a.shape and np.array_equal(mine[name], a)
                for name, a in t.items())
            out[f"p{p}_md{md}_ext{ext}_k{k}_{'sin' if imaginary else 'cos'}"] = d
    os.makedirs(folder, exist_ok=True)
    with open(os.path.join(folder, "reference_table_digests.json"), "w") as f:
        json.dump(out, f, indent=1, sort_keys=True)
    print(len(out), "table sets")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=os.environ.get("HFMM0_REFERENCE"),
                    help="the reference source tree (or set HFMM0_REFERENCE)")
    ap.add_argument("--p12", action="store_true", help="the expansion-order-12 cases, into p12/")
    ap.add_argument("--kernels", action="store_true",
                    help="the Yukawa and Laplace kernels of kifmm.setup, into kernels/")
    ap.add_argument("--keep", action="store_true", help="--kernels: skip fixtures already made")
    ap.add_argument("--edge", action="store_true", help="the edge cases, into edge/")
    ap.add_argument("--grid", action="store_true",
                    help="the reference's test.py grid, into grid/test_py_grid.npz")
    ap.add_argument("--phases", action="store_true",
                    help="per-phase outputs of one adaptive case, into phases/")
    ap.add_argument("--c1", action="store_true",
                    help="the 2e4-point CPU-runnable configuration, into c1/")
    ap.add_argument("--errors", action="store_true",
                    help="the exceptions of invalid inputs, into errors/")
    ap.add_argument("--tables", action="store_true",
                    help="digests of the operator tables, into tables/")
    ap.add_argument("cases", nargs="*")
    a = ap.parse_args()
    if not a.reference:
        ap.error("give the reference source tree: --reference DIR or HFMM0_REFERENCE")
    HFMM, seen = load_reference(a.reference)
    if a.tables:
        return run_tables(HFMM, os.path.join(HERE, "tables"))
    if a.kernels:
        return run_kernels(os.path.join(HERE, "kernels"), keep=a.keep)
    if a.errors:
        return run_errors(HFMM, os.path.join(HERE, "errors"))
    if a.c1:
        return run_c1(HFMM, seen, os.path.join(HERE, "c1"))
    if a.phases:
        return run_phases(HFMM, os.path.join(HERE, "phases"))
    if a.grid:
        return run_test_py_grid(HFMM, os.path.join(HERE, "grid"))
    table, folder = (EDGE, os.path.join(HERE, "edge")) if a.edge else (CASES, HERE)
    if a.p12:
        table, folder = P12, os.path.join(HERE, "p12")
    for name in (a.cases or table):
        t = time.time()
        o = make(HFMM, seen, name, table, folder)
        print(name, "boxes", len(o["m_id"]), "V", len(o["V"]), "U", len(o["U"]),
              "near", len(o["near"]), "W", len(o["W"]), "X", len(o["X"]),
              f"{time.time() - t:.0f} s", flush=True)


if __name__ == "__main__":
    main()
