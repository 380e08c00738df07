"""Oracle: 2:1-balanced cubic octree (test infrastructure only).

Restates jaxfmm/trees/cubic.py with the reference's fixed-buffer array
semantics, so box numbering, parent pointers and particle slots are reproduced
index for index:

* Morton helpers ``_expand_bits``/``_compact_bits``/``_morton_3d`` (cubic.py:73-110);
* neighbour tables ``_build_neighbor_tables`` (cubic.py:29-66);
* ``get_26_neighbors`` (cubic.py:164-201);
* ``build_fmm_tree`` (cubic.py:316-527): Morton codes at ``max_depth``, stable
  argsort, run-length boxes, bottom-up coarsening with count and 2:1-balance
  tests, fine-to-coarse compaction;
* ``build_fmm_tree_auto`` (cubic.py:530-600): buffer doubling and depth refinement;
* ``assign_particles`` (cubic.py:605-695) and ``box_geometry`` (cubic.py:116-160).

Scatter conventions. Two reference scatters write repeated indices:
``child_ids.at[p_id, m_id % 8].set(...)`` (cubic.py:464-465, declared
``unique_indices`` but not unique for inactive boxes and for parents whose
pointer is not set yet) and negative indices wrap (JAX index normalisation).
The oracle uses last-write-wins in index order (the largest writer index) and
NumPy wrapping for negative indices. Only rows that are never read by the
balance test receive conflicting writes, except row 0 when a single box remains
at a level (trees of one box per level), which the tests do not rely on.
"""
import math

import numpy as np

U64 = np.uint64
MAXU = np.uint64(0xFFFFFFFFFFFFFFFF)


def _expand_bits(v):
    v = v.astype(np.uint64)
    v = (v | (v << U64(32))) & U64(0x1F00000000FFFF)
    v = (v | (v << U64(16))) & U64(0x1F0000FF0000FF)
    v = (v | (v << U64(8))) & U64(0x100F00F00F00F00F)
    v = (v | (v << U64(4))) & U64(0x10C30C30C30C30C3)
    v = (v | (v << U64(2))) & U64(0x1249249249249249)
    return v


def _compact_bits(v):
    v = v.astype(np.uint64) & U64(0x1249249249249249)
    v = (v | (v >> U64(2))) & U64(0x10C30C30C30C30C3)
    v = (v | (v >> U64(4))) & U64(0x100F00F00F00F00F)
    v = (v | (v >> U64(8))) & U64(0x1F0000FF0000FF)
    v = (v | (v >> U64(16))) & U64(0x1F00000000FFFF)
    v = (v | (v >> U64(32))) & U64(0x1FFFFF)
    return v


def morton_encode(x, y, z):
    """Interleave grid coordinates, x in bit 0 (cubic.py:101-103)."""
    return _expand_bits(x) | (_expand_bits(y) << U64(1)) | (_expand_bits(z) << U64(2))


def morton_decode(m):
    """Grid coordinates of Morton codes (cubic.py:105-107)."""
    m = np.asarray(m, dtype=np.uint64)
    return _compact_bits(m), _compact_bits(m >> U64(1)), _compact_bits(m >> U64(2))


def _neighbor_tables():
    """26 neighbour offsets (dx outer, dz inner, centre removed) and the mask of
    neighbour children touching the centre box (cubic.py:29-66)."""
    dx, dy, dz = np.meshgrid([-1, 0, 1], [-1, 0, 1], [-1, 0, 1], indexing="ij")
    off = np.stack([np.delete(a.flatten(), 13) for a in (dx, dy, dz)], 1).astype(np.int32)
    mask = np.zeros((26, 8), dtype=bool)
    for i in range(26):
        for c in range(8):
            cb = (c & 1, (c >> 1) & 1, (c >> 2) & 1)
            ok = True
            for ax in range(3):
                d = off[i, ax]
                ok &= (d == -1 and cb[ax] == 1) or (d == 1 and cb[ax] == 0) or d == 0
            mask[i, c] = ok
    return off, mask


NEIGH_OFFSETS, ADJ_CHILD_MASK = _neighbor_tables()


def get_26_neighbors(m, lvl):
    """Same-level neighbour codes and in-domain mask (cubic.py:164-201)."""
    m = np.asarray(m, dtype=np.uint64)
    grid = (2 ** np.asarray(lvl, dtype=np.int64))[:, None]
    x, y, z = morton_decode(m)
    n = [c.astype(np.int64)[:, None] + NEIGH_OFFSETS[None, :, a] for a, c in enumerate((x, y, z))]
    valid = np.ones(n[0].shape, dtype=bool)
    for c in n:
        valid &= (c >= 0) & (c < grid)
    safe = [np.clip(c, 0, grid - 1).astype(np.uint64) for c in n]
    return morton_encode(*safe), valid


def _segment_sum(vals, ids, num):
    keep = (ids >= 0) & (ids < num)
    return np.bincount(ids[keep], weights=None if vals is None else vals[keep],
                       minlength=num)[:num]


def _segment_max_u64(vals, ids, num):
    out = np.zeros(num, dtype=np.uint64)
    keep = (ids >= 0) & (ids < num)
    np.maximum.at(out, ids[keep], vals[keep])
    return out


def _compact(arr, scatter, mb):
    out = np.zeros_like(arr)
    ok = scatter < mb
    out[scatter[ok]] = arr[ok]
    return out


class _Overflow(Exception):
    pass


def build_fmm_tree(positions, max_boxes, max_depth, N_max):
    """One fixed-buffer build (cubic.py:316-527).

    Returns dict with m_id (u64), p_id (i32), lvls (i32), counts (i32),
    is_leaf (bool), sort_idx (i32), domain_extent, pmin, overflow flag and the
    largest box id touched (``max_box_count``).

    A pass whose box ids reach the buffer size is discarded by the caller
    (cubic.py:586-595 retries with a doubled buffer); the reference's JAX gathers
    clamp the out-of-range ids of such a pass, NumPy's would raise, so the pass
    stops there and only reports the overflow.
    """
    pos = np.asarray(positions, dtype=np.float64)
    mb = int(max_boxes)
    md = int(max_depth)
    pmax = pos.max(0)
    pmin = pos.min(0)
    grid = 2 ** md
    extent = np.max(pmax - pmin)
    with np.errstate(invalid="ignore", divide="ignore"):
        scaled = (pos - pmin) / extent * grid
    # extent == 0 (all points equal) gives NaN; XLA's float->int conversion saturates
    # and maps NaN to 0, which NumPy's cast does not guarantee, so apply it explicitly.
    scaled = np.where(np.isnan(scaled), 0.0, scaled)
    gc = np.clip(scaled.astype(np.uint64), U64(0), U64(grid - 1))
    part_m = morton_encode(gc[:, 0], gc[:, 1], gc[:, 2])
    sort_idx = np.argsort(part_m, kind="stable").astype(np.int32)
    sm = part_m[sort_idx]
    changes = np.concatenate([[False], sm[1:] != sm[:-1]])
    node_ids = np.cumsum(changes).astype(np.int64)

    if int(node_ids[-1]) >= mb:
        return dict(max_boxes_exceeded=True, max_box_count=int(node_ids[-1]))
    counts = _segment_sum(None, node_ids, mb).astype(np.int32)
    m_id = _segment_max_u64(sm, node_ids, mb)
    lvls = (counts > 0).astype(np.int32) * md
    p_id = np.zeros(mb, dtype=np.int32)
    is_leaf = counts > 0
    max_box_count = int(node_ids[-1])
    allids = np.arange(mb, dtype=np.int64)
    if max_box_count >= mb:
        return dict(max_boxes_exceeded=True, max_box_count=max_box_count)

    def step(i, check_balance):
        nonlocal m_id, p_id, lvls, counts, is_leaf, max_box_count
        L = md - i
        on = lvls == L
        ofs = int((lvls >= L).sum())
        prev_m = np.where(on, m_id, MAXU)
        prev_c = np.where(on, counts, 0)
        par_m = prev_m // U64(8)
        cc = np.concatenate([[False], par_m[1:] > par_m[:-1]])
        par_m = np.where(on, par_m, U64(0))
        tn = (np.cumsum(cc) + ofs).astype(np.int64)
        max_box_count = max(max_box_count, int(tn[-1]))
        if max_box_count >= mb:
            raise _Overflow()
        this_c = _segment_sum(prev_c.astype(np.int64), tn, mb).astype(np.int32)
        this_m = _segment_max_u64(par_m, tn, mb)
        m_id = m_id + this_m
        lvls = lvls + (this_c > 0).astype(np.int32) * np.int32(L - 1)
        counts = counts + this_c
        p_id = np.where(on, tn, p_id).astype(np.int32)
        count_ok = this_c <= N_max
        delete = count_ok[p_id] & on
        mark = count_ok & (this_c > 0)
        if check_balance:
            neighs, valid = get_26_neighbors(m_id, lvls)
            tms = np.where(counts > 0, this_m, MAXU)
            ins = np.searchsorted(tms, neighs, side="right").astype(np.int64) - 1
            valid = valid & (neighs == tms[ins])
            # last write wins in index order = the largest writer index (module docstring)
            rows = p_id.astype(np.int64) % mb
            flat = np.zeros(mb * 8, dtype=np.int64)
            np.maximum.at(flat, rows * 8 + (m_id % U64(8)).astype(np.int64), allids)
            child_ids = flat.reshape(mb, 8)
            cal = (~valid)[:, :, None] | is_leaf[child_ids[ins]]
            bal = np.all(cal | ~ADJ_CHILD_MASK[None], axis=(1, 2))
            delete = delete & bal[p_id]
            mark = mark & bal
        keep = ~delete
        tgt = (np.cumsum(keep) - 1).astype(np.int64)
        sc = np.where(keep, tgt, mb)
        m_id = _compact(m_id, sc, mb)
        lvls = _compact(lvls, sc, mb)
        counts = _compact(counts, sc, mb)
        p_id = tgt[p_id.astype(np.int64)].astype(np.int32)
        p_id = _compact(p_id, sc, mb)
        is_leaf = _compact(is_leaf | mark, sc, mb)

    try:
        step(0, False)
        for i in range(1, md - 1):
            step(i, True)
    except _Overflow:
        return dict(max_boxes_exceeded=True, max_box_count=max_box_count)
    lvl1 = lvls == 1
    p_id = np.where(lvl1, np.arange(mb, dtype=np.int32), p_id).astype(np.int32)
    return dict(m_id=m_id, p_id=p_id, lvls=lvls.astype(np.int32), counts=counts.astype(np.int32),
                is_leaf=is_leaf, sort_idx=sort_idx, domain_extent=float(extent), pmin=pmin,
                max_boxes_exceeded=max_box_count >= mb, max_box_count=max_box_count)


def initial_max_boxes(N, N_max):
    """Starting buffer size of build_fmm_tree_auto (cubic.py:585)."""
    return max(4 * N // N_max, 512) + 4096


def auto_depth(N, N_max):
    """Volume-filling starting depth (cubic.py:583-584)."""
    return max(2, math.ceil(math.log(max(N / max(N_max, 1), 1.0)) / math.log(8)))


def build_fmm_tree_auto(positions, N_max=64, max_depth=None, refine_factor=2, depth_cap=10):
    """Buffer-doubling, depth-refining driver (cubic.py:530-600).

    Returns (tree dict, max_boxes, max_depth, maxleaf).
    """
    N = positions.shape[0]
    md_given = max_depth is not None
    md = int(max_depth) if md_given else auto_depth(N, N_max)
    mb = initial_max_boxes(N, N_max)
    while True:
        for _ in range(10):
            t = build_fmm_tree(positions, mb, md, N_max)
            if not t["max_boxes_exceeded"]:
                break
            mb *= 2
        else:
            raise ValueError("build_fmm_tree_auto: box buffer kept overflowing; check max_depth/N_max")
        leafm = t["is_leaf"] & (t["lvls"] > 0)
        maxleaf = int(t["counts"][leafm].max())
        if md_given or maxleaf <= refine_factor * N_max or md >= depth_cap:
            return t, mb, md, maxleaf
        md += 1


def assign_particles(sort_idx, m_id, lvls, counts, is_leaf, max_depth, N_max):
    """Leaf of each particle and the (max_boxes, N_max) particles-in-leaf table
    (cubic.py:605-695)."""
    N = sort_idx.shape[0]
    mb = m_id.shape[0]
    leafm = is_leaf & (lvls > 0)
    diff = (np.int64(max_depth) - lvls.astype(np.int64)).astype(np.uint64)
    scaled = np.where(leafm, m_id << (U64(3) * diff), MAXU)
    leaf_order = np.argsort(scaled, kind="stable")
    leaf_counts = np.where(leafm, counts, 0).astype(np.int64)
    cum = np.cumsum(leaf_counts[leaf_order])
    k = np.arange(N, dtype=np.int64)
    rank = np.searchsorted(cum, k, side="right")
    leaf_of_sorted = leaf_order[rank].astype(np.int32)
    leaf_of_particle = np.zeros(N, dtype=np.int32)
    leaf_of_particle[sort_idx] = leaf_of_sorted
    start = np.concatenate([[0], cum[:-1]])
    pos_in_leaf = k - start[rank]
    pil = np.full((mb, N_max), -1, dtype=np.int32)
    ok = pos_in_leaf < N_max
    pil[leaf_of_sorted[ok], pos_in_leaf[ok]] = sort_idx[ok]
    return leaf_of_particle, pil


def box_geometry(m_id, lvls, domain_extent, pmin):
    """Box centres and half-sides (cubic.py:116-160)."""
    x, y, z = morton_decode(m_id)
    coords = np.stack([x, y, z], -1).astype(np.float64)
    lv = lvls.astype(np.int64)
    coords = coords * domain_extent / (2.0 ** lv)[:, None]
    coords = coords + domain_extent * 0.5 ** (lv[:, None] + 1) + pmin
    h = domain_extent * 0.5 ** (lvls.astype(np.float64) + 1.0)
    return coords, h
