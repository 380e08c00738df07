"""The folded decodes of the low-rank mixed path, restated on the oracle's phases.

The CUDA path keeps every box in scaled SVD coordinates, y = d .* (U^T x), and
multiplies the decodes' other factor into the operators beside it (M2M, L2L,
M2L here; compression and expansion in the product): only leaves leave the
coordinates (U after P2M, Vt before L2P). Because d is never multiplied into a
table, the two-step decode's rounding stays in the near-null directions that the
next operator damps, and the result equals the reference's decode order
(phases.py:21-76) to rounding. Folding the whole damped pseudo-inverse
U diag(d) Vt into M2M as one matrix does not: that is why the product keeps the
factors apart. CPU only, small problem."""
import numpy as np

from oracle import hfmm as H
from oracle.tree import box_geometry


def _folded(s, Q, whole_pinv_in_m2m=False):
    kern, ops, lvls, md = s["kernel"], s["ops"], s["lvls"], s["max_depth"]
    centres, h = box_geometry(s["m_id"], lvls, s["domain_extent"], s["pmin"])
    ppts, pchg, rev = H._build_padded(s["positions"], Q, s["pil"])
    Fu = [tuple(f[l] for f in ops["F_up_lv"]) for l in range(md + 1)]
    Fd = [tuple(f[l] for f in ops["F_dn_lv"]) for l in range(md + 1)]
    leaf = s["is_leaf"]
    chk = H.p2m(s, kern, ppts, pchg, centres, h)
    y = np.zeros_like(chk)
    for l in range(md + 1):
        r = np.nonzero((lvls == l) & leaf)[0]
        if r.size:
            y[r] = (chk[r] @ Fu[l][0]) * Fu[l][1]
    for cl in range(md, 1, -1):
        pl = cl - 1
        K = ops["M2M_K_lv"][pl]
        acc = np.zeros_like(chk)
        kids = np.nonzero(lvls == cl)[0]
        octs = (s["m_id"][kids] % np.uint64(8)).astype(np.int64)
        for o in range(8):
            b = kids[octs == o]
            if not b.size:
                continue
            if whole_pinv_in_m2m:   # x_child = y Vt, then the parent's U^T ... d as one matrix
                T = Fu[cl][2] @ K[o].T @ ((Fu[pl][0] * Fu[pl][1]) @ Fu[pl][2])
            else:
                T = Fu[cl][2] @ K[o].T @ Fu[pl][0]
            np.add.at(acc, s["p_id"][b], y[b] @ T)
        r = np.nonzero((lvls == pl) & ~leaf)[0]
        if whole_pinv_in_m2m:   # acc is already the parent's density: back to coordinates
            y[r] = (acc[r] @ Fu[pl][2].T)
        else:
            y[r] = acc[r] * Fu[pl][1]
    V = s["V"]
    tgt, src = V[:, 0].astype(np.int64), V[:, 1].astype(np.int64)
    key = lvls[tgt].astype(np.int64) * 343 + H._disp_ids(s, tgt, src)
    order = np.argsort(key, kind="stable")
    cuts = np.nonzero(np.diff(key[order]))[0] + 1
    acc = np.zeros_like(chk)
    for grp in np.split(order, cuts):
        kk = key[grp[0]]
        l = kk // 343
        acc[tgt[grp]] += y[src[grp]] @ (Fu[l][2] @ ops["M2L_K_lv"][l][kk % 343].T @ Fd[l][0])
    yd = np.zeros_like(chk)
    for cl in range(2, md + 1):
        r = np.nonzero(lvls == cl)[0]
        a = acc[r].copy()
        if cl >= 3:
            K = ops["L2L_K_lv"][cl - 1]
            octs = (s["m_id"][r] % np.uint64(8)).astype(np.int64)
            for o in range(8):
                sel = octs == o
                a[sel] += yd[s["p_id"][r[sel]]] @ (Fd[cl - 1][2] @ K[o].T @ Fd[cl][0])
        yd[r] = a * Fd[cl][1]
    loc = np.zeros_like(chk)
    for l in range(md + 1):
        r = np.nonzero((lvls == l) & leaf)[0]
        if r.size:
            loc[r] = yd[r] @ Fd[l][2]
    far = H.l2p(s, kern, loc, ppts, rev, centres, h, False)
    return far + H.eval_direct(s, kern, ppts, pchg, rev, False)


def _problem():
    rng = np.random.default_rng(3)
    x = rng.random((2500, 3))
    q = rng.standard_normal(2500) + 1j * rng.standard_normal(2500)
    return x, q


def test_factored_fold_equals_the_two_step_decode():
    x, q = _problem()
    st = H.setup(x, 6.0, p=6, N_max=16)
    assert st[0]["max_depth"] >= 3   # at least one folded M2M and one folded L2L level
    Q = np.stack([q.real, q.imag], 1)
    for s in st:                     # both components: eps_rel 1e-7 (cos) and 1e-12 (sin)
        ref = H.evaluate_setup(s, Q, fused_decode=True)
        got = _folded(s, Q)
        assert np.linalg.norm(got - ref) <= 1e-11 * np.linalg.norm(ref)


def test_folding_the_whole_pseudo_inverse_loses_accuracy():
    x, q = _problem()
    st = H.setup(x, 6.0, p=6, N_max=16)
    s = st[1]                        # the sin component: eps_rel 1e-12, the hard one
    Q = np.stack([q.real, q.imag], 1)
    ref = H.evaluate_setup(s, Q, fused_decode=True)
    bad = _folded(s, Q, whole_pinv_in_m2m=True)
    good = _folded(s, Q)
    e_bad = np.linalg.norm(bad - ref) / np.linalg.norm(ref)
    e_good = np.linalg.norm(good - ref) / np.linalg.norm(ref)
    assert e_bad > 1e3 * max(e_good, 1e-16), (e_bad, e_good)
