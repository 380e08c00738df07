"""Generate the golden fixtures under tests/golden/ from the oracle.

The reference (JAX) cannot run in this environment, so the fixtures record the
oracle's outputs -- pinned against the reference's own known-answer checks in
tests/test_oracle_known_answers.py -- for small seeded cases: the tree arrays
(build_fmm_tree outputs for the active boxes), the particles-in-leaf table,
the V/U/W/X/near lists and the evaluate outputs. Run from the repo root:

    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
sys.path.insert(0, os.path.dirname(HERE))

import oracle as O  # noqa: E402
from cases import uniform, clustered, sphere_clusters, with_duplicates, complex_uniform  # noqa: E402

CASES = {
    # name: (cloud, n, k, p, N_max, max_depth, complex charges + field)
    "uniform640_k3_p5": (uniform, 640, 3.0, 5, 16, None, False),
    "clustered900_k2_p4": (clustered, 900, 2.0, 4, 16, None, True),
    "sphere1500_k5_p4": (sphere_clusters, 1500, 5.0, 4, 20, None, True),
    "uniform256_k0_p3": (uniform, 256, 0.0, 3, 16, None, False),
    "dup500_k1_p3": (with_duplicates, 500, 1.0, 3, 16, None, False),
    "cplx2000_k8_p6_d4": (complex_uniform, 2000, 8.0, 6, 32, 4, True),
}


def make(name):
    fn, n, k, p, nmax, md, cplx = CASES[name]
    pos, q = fn(n)
    if cplx and not np.iscomplexobj(q):
        q = q + 1j * np.random.default_rng(n).normal(size=n)
    st = O.setup(pos, k, p=p, N_max=nmax, max_depth=md)
    s = st[0]
    nb = int((s["lvls"] > 0).sum())
    out = dict(positions=pos, charges=q, k=k, p=p, N_max=nmax,
               max_depth=-1 if md is None else md, realised_depth=s["max_depth"],
               maxleaf=s["maxleaf"], max_boxes=s["max_boxes"], domain_extent=s["domain_extent"],
               m_id=s["m_id"][:nb], p_id=s["p_id"][:nb], lvls=s["lvls"][:nb],
               counts=s["counts"][:nb], is_leaf=s["is_leaf"][:nb], sort_idx=s["sort_idx"],
               pil=s["pil"][:nb], V=s["V"], U=s["U"], near=s["dir_cnct"],
               W=s["W"] if s["W"] is not None else np.empty((0, 2), np.int32),
               X=s["X"] if s["X"] is not None else np.empty((0, 2), np.int32))
    if cplx:
        phi, E = O.evaluate_complex(st, q, field=True)
        out.update(phi=phi, E=E)
    else:
        out.update(phi=O.evaluate(st, q))
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
    return out


if __name__ == "__main__":
    for name in (sys.argv[1:] or CASES):
        o = make(name)
        print(name, "boxes", len(o["m_id"]), "V", len(o["V"]), "near", len(o["near"]),
              "W", len(o["W"]), "X", len(o["X"]))
