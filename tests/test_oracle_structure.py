"""Structural invariants of the oracle's tree and lists.

The interaction lists must partition the leaf-leaf interaction space: for
every (target leaf, source leaf) pair, exactly one of the near field (U + self,
core.py:138-140), the V list (through every leaf under both boxes), the W list
(every leaf under the source box) and the X list (every leaf under the target
box) covers it. This holds only if the tree is 2:1 balanced and the lists follow
lists.py exactly, so it checks the tree builder and all four list builders at once.
"""
import numpy as np
import pytest

import oracle as O
from oracle.hfmm import HelmholtzComponent
from cases import uniform, clustered, sphere_clusters, with_duplicates, plane, sphere_and_clusters


def _leaves_under(s):
    nb = s["m_id"].shape[0]
    lv, pid, leaf = s["lvls"], s["p_id"], s["is_leaf"] & (s["lvls"] > 0)
    under = {b: [] for b in range(nb)}
    for b in np.nonzero(leaf)[0]:
        a = b
        while True:
            under[a].append(b)
            if lv[a] <= 1:
                break
            a = pid[a]
    return under


def coverage(s):
    leaf = np.nonzero(s["is_leaf"] & (s["lvls"] > 0))[0]
    pos = {b: i for i, b in enumerate(leaf)}
    cov = np.zeros((len(leaf), len(leaf)), dtype=np.int64)
    under = _leaves_under(s)
    for t, sb in s["dir_cnct"]:
        cov[pos[t], pos[sb]] += 1
    for t, sb in s["V"]:
        for a in under[t]:
            for b in under[sb]:
                cov[pos[a], pos[b]] += 1
    for t, sb in (s["W"] if s["W"] is not None else []):
        for b in under[sb]:
            cov[pos[t], pos[b]] += 1
    for t, sb in (s["X"] if s["X"] is not None else []):
        for a in under[t]:
            cov[pos[a], pos[sb]] += 1
    return cov


CLOUDS = [(uniform, 700, 16), (clustered, 900, 16), (sphere_clusters, 1500, 20),
          (with_duplicates, 500, 16), (plane, 800, 16)]


def _state(fn, n, nmax):
    pos, _ = fn(n)
    return O.kifmm_setup(pos, 3, nmax, None, HelmholtzComponent(1.0, False))


@pytest.mark.parametrize("fn,n,nmax", CLOUDS)
def test_lists_partition_interactions(fn, n, nmax):
    s = _state(fn, n, nmax)
    cov = coverage(s)
    assert cov.min() == 1 and cov.max() == 1


@pytest.mark.parametrize("fn,n,nmax", CLOUDS)
def test_tree_invariants(fn, n, nmax):
    s = _state(fn, n, nmax)
    lv, pid, cnt, leaf, m = s["lvls"], s["p_id"], s["counts"], s["is_leaf"], s["m_id"]
    act = lv > 0
    nb = int(act.sum())
    assert act[:nb].all() and not act[nb:].any()          # packed, inactive at the end
    assert np.all(np.diff(lv[:nb]) <= 0)                   # fine-to-coarse
    # each particle in exactly one leaf, pil rows = leaf counts
    pil = s["pil"]
    got = pil[pil >= 0]
    assert np.array_equal(np.sort(got), np.arange(len(s["positions"])))
    assert np.array_equal((pil >= 0).sum(1)[:nb][leaf[:nb]], cnt[:nb][leaf[:nb]])
    # parent relations
    for b in range(nb):
        if lv[b] > 1:
            p = pid[b]
            assert lv[p] == lv[b] - 1 and m[p] == m[b] >> np.uint64(3) and not leaf[p]
        else:
            assert pid[b] == b
    # counts add up
    for b in range(nb):
        if not leaf[b]:
            assert cnt[b] == cnt[(pid == b) & (lv == lv[b] + 1)].sum()
    # 2:1 balance between adjacent leaves
    L = np.nonzero(leaf & act)[0]
    gx, gy, gz = (c.astype(np.int64) for c in O.morton_decode(m[L]))
    lo = np.stack([gx, gy, gz], 1) * (2 ** (s["max_depth"] - lv[L]))[:, None]
    size = (2 ** (s["max_depth"] - lv[L]))[:, None]
    hi = lo + size
    for i in range(len(L)):
        touch = np.all((lo <= hi[i]) & (hi >= lo[i]), axis=1)
        touch[i] = False
        assert np.all(np.abs(lv[L][touch] - lv[L[i]]) <= 1)


def test_adaptive_cloud_has_w_and_x():
    s = _state(sphere_clusters, 1500, 20)
    assert s["adaptive"] and s["W"] is not None and s["X"] is not None


def test_oracle_rounding_floor():
    """Two summation orders of the oracle (per-site decodes vs one fused decode per
    box) agree far below the 1e-12 parity bar."""
    from cases import complex_uniform
    pos, q = complex_uniform(1500)
    st = O.setup(pos, 6.0, p=6, N_max=32)
    a = O.evaluate_complex(st, q, field=False, fused_decode=False)
    b = O.evaluate_complex(st, q, field=False, fused_decode=True)
    assert O.relative_error(b, a) < 1e-13


def test_tree_build_retries_when_the_buffer_overflows():
    """A deep adaptive cloud whose box ids outgrow the first buffer: the reference
    discards that pass and doubles the buffer (cubic.py:586-595); the restatement
    must do the same instead of indexing past its arrays."""
    from oracle.tree import build_fmm_tree_auto, initial_max_boxes
    pos, _ = sphere_and_clusters(8000)
    t, mb, md, maxleaf = build_fmm_tree_auto(pos, N_max=16)
    assert mb == 2 * initial_max_boxes(len(pos), 16) and md == 6
    leaf = t["is_leaf"] & (t["lvls"] > 0)
    assert int(t["counts"][leaf].sum()) == len(pos)
    assert not t["max_boxes_exceeded"]

