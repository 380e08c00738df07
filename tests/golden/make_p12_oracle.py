"""Generate the oracle's expansion-order-12 fixtures under tests/golden/p12/.

The order-12 plain path (n_s = 728 surface points per box) is the FP64 path of
the 1e6-point workload. Its outputs at sizes where the reference itself is too
slow on the NumPy stand-in for JAX (tests/golden/make_golden.py, hours here) come
from the oracle, which tests/golden/p12/ also pins to the reference at order 12
on two smaller clouds (`make_golden.py --p12`; tests/test_golden.py checks them).

Cases (the seeded clouds of tests/cases.py, complex charges, potential + field):

* oracle_uniform20000_k10_p12: 20 000 uniform points, k = 10, leaf size 64
  (auto depth 3);
* oracle_sphere6000_k10_p12_d4: 6 000 points half on a sphere and half in eight
  Gaussian clusters, k = 10, leaf size 32, max_depth = 4 (adaptive: W and X
  lists are non-empty).

Run from the repo root (about 4 minutes on 8 cores):

    python tests/golden/make_p12_oracle.py
"""
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from cases import complex_uniform, sphere_clusters  # noqa: E402
import oracle as O  # noqa: E402

CASES = {
    # name: (cloud, n, k, p, N_max, max_depth)
    "oracle_uniform20000_k10_p12": (complex_uniform, 20000, 10.0, 12, 64, None),
    "oracle_sphere6000_k10_p12_d4": (sphere_clusters, 6000, 10.0, 12, 32, 4),
}


def make(name):
    fn, n, k, p, nmax, md = CASES[name]
    pos, q = fn(n)
    t = time.time()
    st = O.setup(pos, k, p=p, N_max=nmax, max_depth=md)
    s = st[0]
    phi, E = O.evaluate_complex(st, q, field=True)
    out = dict(positions_sum=np.float64(pos.sum()), charges_sum=q.sum(), n=n, k=k, p=p,
               N_max=nmax, max_depth=-1 if md is None else md,
               realised_depth=int(s["max_depth"]), n_v=len(s["V"]),
               n_w=0 if s["W"] is None else len(s["W"]), n_x=0 if s["X"] is None else len(s["X"]),
               phi=phi, E=E)
    os.makedirs(os.path.join(HERE, "p12"), exist_ok=True)
    np.savez_compressed(os.path.join(HERE, "p12", name + ".npz"), **out)
    print(name, "depth", out["realised_depth"], "V", out["n_v"], "W", out["n_w"],
          f"{time.time() - t:.0f} s", flush=True)


if __name__ == "__main__":
    for name in (sys.argv[1:] or CASES):
        make(name)
