"""Oracle: cubic-octree interaction lists (test infrastructure only).

Restates the eager block builders of jaxfmm/trees/lists.py (open boundaries),
including their output order, so the pair arrays are reproduced row for row:

* ``_not_adjacent`` (lists.py:14-24), ``_adj_coarse_ax``/``_adj_fine_ax`` (573-580);
* ``_sorted_boxids``/``_blk_lookup`` (583-599): box ids ``(lvl << 3*max_depth) | m``;
* ``_v_block`` (619-661): children of the parent's 26 neighbours, same level,
  non-adjacent, not self; order (target, neighbour, child);
* ``_ua_block`` (664-738): per block of 262144 targets, same-level neighbours,
  then coarser parent-colleagues, then finer colleague children, each in
  (target, neighbour[, child]) order;
* ``_wx_block`` (741-802): W (finer, non-adjacent) and X (coarser, non-adjacent).
* ``core.setup_geometry`` (core.py:115-140): near pairs = U + leaf self pairs.
"""
import numpy as np

from .tree import get_26_neighbors, morton_decode, MAXU

BLOCK = 262144   # lists.py:563


def _sorted_boxids(m_id, lvls, max_depth):
    shift = np.uint64(3 * max_depth)
    box_ids = (lvls.astype(np.uint64) << shift) | m_id
    active = np.where(lvls > 0, box_ids, MAXU)
    order = np.argsort(active, kind="stable")
    return active, order, active[order]


def _lookup(cand, tabs, mb):
    active, order, sorted_ids = tabs
    flat = cand.reshape(-1)
    ins = np.clip(np.searchsorted(sorted_ids, flat, side="left"), 0, mb - 1)
    orig = order[ins]
    found = active[orig] == flat
    return orig.reshape(cand.shape).astype(np.int32), found.reshape(cand.shape)


def _ids(lvl, m, shift):
    # (lvl << shift) | m with the reference's uint64 wrap for lvl = -1
    return (lvl.astype(np.int64).astype(np.uint64) << shift) | m


def _blocks(mb):
    for lo in range(0, mb, BLOCK):
        yield lo, min(lo + BLOCK, mb)


def build_v(m_id, lvls, is_leaf, max_depth):
    """Compact V list (n, 2) int32 of (target, source) (lists.py:619-661, 818-854)."""
    mb = m_id.shape[0]
    tabs = _sorted_boxids(m_id, lvls, max_depth)
    shift = np.uint64(3 * max_depth)
    out = []
    for lo, hi in _blocks(mb):
        m_b, l_b = m_id[lo:hi], lvls[lo:hi]
        B = hi - lo
        par_m = m_b // np.uint64(8)
        par_l = np.maximum(l_b - 1, 0)
        pn, pv = get_26_neighbors(par_m, par_l)
        cand = pn[:, :, None] * np.uint64(8) + np.arange(8, dtype=np.uint64)[None, None, :]
        orig, found = _lookup(_ids(l_b[:, None, None], cand, shift), tabs, mb)
        found = pv[:, :, None] & found
        tx, ty, tz = (c.astype(np.int64) for c in morton_decode(m_b))
        cx, cy, cz = (c.astype(np.int64).reshape(B, 26, 8) for c in morton_decode(cand.reshape(-1)))
        na = ((cx - tx[:, None, None] > 1) | (tx[:, None, None] - cx > 1)
              | (cy - ty[:, None, None] > 1) | (ty[:, None, None] - cy > 1)
              | (cz - tz[:, None, None] > 1) | (tz[:, None, None] - cz > 1))
        not_self = cand != m_b[:, None, None]
        valid = (l_b > 0)[:, None, None] & found & na & not_self
        t = np.broadcast_to(np.arange(lo, hi, dtype=np.int32)[:, None, None], valid.shape)
        out.append(np.stack([t[valid], orig[valid]], 1))
    return np.concatenate(out).astype(np.int32) if out else np.empty((0, 2), np.int32)


def _adj_coarse(b, c):
    return (b <= 2 * c + 2) & (2 * c <= b + 1)


def _adj_fine(b, f):
    return (2 * b <= f + 1) & (f <= 2 * b + 2)


def _coarse_fine(m_b, l_b, m_id, lvls, tabs, mb, shift):
    """Shared candidate sets of _ua_block/_wx_block for one block."""
    B = m_b.shape[0]
    bx, by, bz = (c.astype(np.int64) for c in morton_decode(m_b))
    nS, vS = get_26_neighbors(m_b, l_b)
    oS, fS = _lookup(_ids(l_b[:, None], nS, shift), tabs, mb)
    par_m = m_b // np.uint64(8)
    par_l = np.maximum(l_b - 1, 0)
    pn, pv = get_26_neighbors(par_m, par_l)
    oC, fC = _lookup(_ids((l_b - 1)[:, None], pn, shift), tabs, mb)
    cx, cy, cz = (c.astype(np.int64).reshape(B, 26) for c in morton_decode(pn.reshape(-1)))
    adjC = (_adj_coarse(bx[:, None], cx) & _adj_coarse(by[:, None], cy)
            & _adj_coarse(bz[:, None], cz))
    chm = nS[:, :, None] * np.uint64(8) + np.arange(8, dtype=np.uint64)[None, None, :]
    oF, fF = _lookup(_ids((l_b + 1)[:, None, None], chm, shift), tabs, mb)
    fx, fy, fz = (c.astype(np.int64).reshape(B, 26, 8) for c in morton_decode(chm.reshape(-1)))
    adjF = (_adj_fine(bx[:, None, None], fx) & _adj_fine(by[:, None, None], fy)
            & _adj_fine(bz[:, None, None], fz))
    return (nS, vS, oS, fS), (pv, oC, fC, adjC), (oF, fF, adjF)


def build_u(m_id, lvls, is_leaf, max_depth):
    """Compact adaptive U list (n, 2) int32, no self pairs (lists.py:664-738, 857-889)."""
    mb = m_id.shape[0]
    tabs = _sorted_boxids(m_id, lvls, max_depth)
    shift = np.uint64(3 * max_depth)
    leaf_g = is_leaf & (lvls > 0)
    out = []
    for lo, hi in _blocks(mb):
        m_b, l_b, leaf_b = m_id[lo:hi], lvls[lo:hi], leaf_g[lo:hi]
        (nS, vS, oS, fS), (pv, oC, fC, adjC), (oF, fF, adjF) = _coarse_fine(
            m_b, l_b, m_id, lvls, tabs, mb, shift)
        t = np.arange(lo, hi, dtype=np.int32)
        vSp = leaf_b[:, None] & vS & fS & leaf_g[oS]
        vCp = leaf_b[:, None] & (l_b > 1)[:, None] & pv & fC & leaf_g[oC] & adjC
        vFp = leaf_b[:, None, None] & vS[:, :, None] & fF & leaf_g[oF] & adjF
        for valid, src in ((vSp, oS), (vCp, oC), (vFp, oF)):
            tt = np.broadcast_to(t.reshape((-1,) + (1,) * (valid.ndim - 1)), valid.shape)
            out.append(np.stack([tt[valid], src[valid]], 1))
    return np.concatenate(out).astype(np.int32) if out else np.empty((0, 2), np.int32)


def build_wx(m_id, lvls, is_leaf, max_depth):
    """Compact W (target leaf, finer source box) and X (target box, coarser source
    leaf) lists (lists.py:741-802, 892-931)."""
    mb = m_id.shape[0]
    tabs = _sorted_boxids(m_id, lvls, max_depth)
    shift = np.uint64(3 * max_depth)
    leaf_g = is_leaf & (lvls > 0)
    Wp, Xp = [], []
    for lo, hi in _blocks(mb):
        m_b, l_b, leaf_b = m_id[lo:hi], lvls[lo:hi], leaf_g[lo:hi]
        (nS, vS, oS, fS), (pv, oC, fC, adjC), (oF, fF, adjF) = _coarse_fine(
            m_b, l_b, m_id, lvls, tabs, mb, shift)
        t = np.arange(lo, hi, dtype=np.int32)
        xv = (l_b > 0)[:, None] & (l_b > 1)[:, None] & pv & fC & leaf_g[oC] & ~adjC
        wv = leaf_b[:, None, None] & vS[:, :, None] & fF & ~adjF
        tt = np.broadcast_to(t[:, None], xv.shape)
        Xp.append(np.stack([tt[xv], oC[xv]], 1))
        tt = np.broadcast_to(t[:, None, None], wv.shape)
        Wp.append(np.stack([tt[wv], oF[wv]], 1))
    W = np.concatenate(Wp).astype(np.int32) if Wp else np.empty((0, 2), np.int32)
    X = np.concatenate(Xp).astype(np.int32) if Xp else np.empty((0, 2), np.int32)
    return W, X


def near_pairs(U, lvls, is_leaf):
    """U pairs followed by leaf self pairs in index order (core.py:138-140)."""
    leaf_idx = np.nonzero(is_leaf & (lvls > 0))[0].astype(np.int32)
    return np.concatenate([U, np.stack([leaf_idx, leaf_idx], 1)]).astype(np.int32)
