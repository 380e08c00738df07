"""The oracle still reproduces the committed golden fixtures (tests/golden/*.npz,
made by tests/golden/make_golden.py): integer arrays bit for bit, evaluate
outputs to 1e-13 relative L2."""
import glob
import os

import numpy as np
import pytest

import oracle as O

GOLD = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "*.npz")))


def load(path):
    with np.load(path) as z:
        return {k: z[k] for k in z.files}


@pytest.mark.parametrize("path", GOLD, ids=[os.path.basename(p)[:-4] for p in GOLD])
def test_oracle_reproduces_golden(path):
    g = load(path)
    md = int(g["max_depth"])
    st = O.setup(g["positions"], float(g["k"]), p=int(g["p"]), N_max=int(g["N_max"]),
                 max_depth=None if md < 0 else md)
    s = st[0]
    nb = len(g["m_id"])
    for key in ("m_id", "p_id", "lvls", "counts", "is_leaf", "pil"):
        assert np.array_equal(s[key][:nb], g[key]), key
    assert np.array_equal(s["sort_idx"], g["sort_idx"])
    for key, sk in (("V", "V"), ("U", "U"), ("near", "dir_cnct")):
        assert np.array_equal(s[sk], g[key]), key
    q = g["charges"]
    if "E" in g:
        phi, E = O.evaluate_complex(st, q, field=True)
        assert O.relative_error(E, g["E"]) < 1e-13
    else:
        phi = O.evaluate(st, q)
    assert O.relative_error(phi, g["phi"]) < 1e-13


def test_fixtures_present():
    assert len(GOLD) >= 6
