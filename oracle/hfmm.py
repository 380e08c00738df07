"""Oracle: HFMM setup / evaluate and the KIFMM phases (test infrastructure only).

Restatement of the reference's HFMM path in NumPy float64:

* ``setup`` / ``evaluate``: HFMM.py:55-91 (real charges, complex128 result);
* ``kifmm_setup``: jaxfmm/kifmm/setup.py:19-226 on the leveled branch with
  core.setup_geometry (core.py:39-160) and the host pil/perm block (setup.py:140-150);
* ``evaluate_setup``: kifmm/setup.py:229-261 -> assemble.evaluate (assemble.py:295-399)
  -> core.evaluate (core.py:214-335) with the leveled closures (assemble.py:15-89);
* phases: p2m_padded_leveled (phases.py:79-125), m2m_factored_leveled (128-173),
  m2l_leveled (176-237), l2l_factored_leveled (240-280), l2p_padded (1533-1582),
  p2l_leveled (1709-1770), m2p (1064-1140), _decode_leveled (21-76);
* near field: eval_direct flat path (near.py:48-312) with _build_padded (589-598),
  the "pair" coincidence floor (near.py:252-261) and the Helmholtz k2/k2g
  weights (HFMM.py:29-47);
* ``direct``: the O(N^2) referee of test.py:11-18.

Every function accepts R right-hand sides at once (charges of shape (N,) or
(N, R)); the phases are linear, so column r of the result is the evaluate of
charge column r. M2L is grouped by (level, displacement), which changes only
the summation order. ``fused_decode=True`` instead sums the M2L, P2L and L2L
check potentials of a box and decodes once (the CUDA path's order); comparing
the two measures the oracle's own rounding floor.
"""
import math

import numpy as np

from .surfaces import n_surf
from .operators import helmholtz_G_np, build_operators_leveled
from .tree import build_fmm_tree_auto, assign_particles, box_geometry, morton_decode
from .lists import build_v, build_u, build_wx, near_pairs

EPS = np.finfo(np.float64).eps


# ---------------------------------------------------------------- kernels (HFMM.py:12-52)
class HelmholtzComponent:
    """Device-side callables of ``helmholtz_component(k, imaginary)`` (HFMM.py:12-52)."""

    def __init__(self, k, imaginary):
        k = float(k)
        if not np.isfinite(k):
            raise ValueError("k must be a finite real number")
        self.k = k
        self.imaginary = bool(imaginary)
        self.trig = np.sin if imaginary else np.cos
        self.G_np = helmholtz_G_np(k, imaginary)

    def g_box(self, r):
        """g(r) with the ULP floor taken per leading index (HFMM.py:25-27 under vmap)."""
        mx = r.max(axis=tuple(range(1, r.ndim)), keepdims=True)
        ok = r > 16 * EPS * mx
        return np.where(ok, self.trig(self.k * r) / np.where(ok, r, 1.0), 0.0)

    def field_weight(self, d2):
        """(cos + kr sin)/r^3 or (sin - kr cos)/r^3, 0 at d2 = 0 (HFMM.py:29-35)."""
        safe = np.where(d2 > 0, d2, 1.0)
        r = np.sqrt(safe)
        kr = self.k * r
        if self.imaginary:
            num = np.sin(kr) - kr * np.cos(kr)
        else:
            num = np.cos(kr) + kr * np.sin(kr)
        return np.where(d2 > 0, num / (safe * r), 0.0)

    def g_grad_box(self, d):
        """-grad G for d = eval - src, floor per leading index (HFMM.py:37-40)."""
        d2 = np.sum(d * d, axis=-1)
        mx = d2.max(axis=tuple(range(1, d2.ndim)), keepdims=True)
        ok = d2 > (16 * EPS) ** 2 * mx
        return d * self.field_weight(np.where(ok, d2, 0.0))[..., None]

    def k2(self, d2):
        """4 pi-scaled near weight (HFMM.py:42-44)."""
        r = np.sqrt(np.where(d2 > 0, d2, 1.0))
        return 4 * np.pi * np.where(d2 > 0, self.trig(self.k * r) / r, 0.0)

    def k2g(self, d2):
        """4 pi-scaled near field factor (HFMM.py:46-47)."""
        return 4 * np.pi * self.field_weight(d2)


class YukawaKernel:
    """The reference's screened-Coulomb kernel G = exp(-kappa r) / (4 pi r)
    (jaxfmm/kernels/yukawa/kernel.py:10-75); kappa = 0 is its Laplace kernel
    1 / (4 pi r) (jaxfmm/kernels/laplace/kernel.py:40-104), whose value and field
    functions are the same expressions with exp(0) = 1."""

    def __init__(self, kappa):
        kappa = float(kappa)
        if not (np.isfinite(kappa) and kappa >= 0):
            raise ValueError("kappa must be finite and >= 0")
        self.kappa = kappa
        self.name = "laplace" if kappa == 0 else f"yukawa(kappa={kappa:g})"

        def G_np(x, y):
            d = x[:, None, :] - y[None, :, :]
            r = np.sqrt((d ** 2).sum(-1))
            with np.errstate(divide="ignore", invalid="ignore"):
                K = np.exp(-kappa * r) / (4.0 * np.pi * r)
            K[r <= 16 * EPS * r.max(initial=0.0)] = 0.0          # ULP-relative
            return K
        self.G_np = G_np

    def g_box(self, r):
        mx = r.max(axis=tuple(range(1, r.ndim)), keepdims=True)
        ok = r > 16 * EPS * mx
        return np.where(ok, 0.25 / np.pi * np.exp(-self.kappa * r) / np.where(ok, r, 1.0), 0.0)

    def field_weight(self, d2):
        """(1 + kappa r) exp(-kappa r) / r^3 (4 pi-free), 0 at d2 = 0."""
        safe = np.where(d2 > 0, d2, 1.0)
        r = np.sqrt(safe)
        return np.where(d2 > 0, (1 + self.kappa * r) * np.exp(-self.kappa * r) / (safe * r), 0.0)

    def g_grad_box(self, d):
        d2 = np.sum(d * d, axis=-1)
        mx = d2.max(axis=tuple(range(1, d2.ndim)), keepdims=True)
        ok = d2 > (16 * EPS) ** 2 * mx
        return d * (0.25 / np.pi * self.field_weight(np.where(ok, d2, 0.0)))[..., None]

    def k2(self, d2):
        r = np.sqrt(np.where(d2 > 0, d2, 1.0))
        return np.where(d2 > 0, np.exp(-self.kappa * r) / r, 0.0)

    def k2g(self, d2):
        return self.field_weight(d2)


def kernel_setup(positions, kernel, p=4, N_max=16, max_depth=None):
    """kifmm.setup(positions, p, N_max, max_depth, kernel=...) for a real kernel
    (kifmm/setup.py:19-226, leveled operators, FP64 near field): the oracle of the
    other kernels the CUDA path takes through its kernel seam."""
    return kifmm_setup(positions, int(p), int(N_max), max_depth, kernel)


# ---------------------------------------------------------------- setup
def kifmm_setup(positions, p, N_max, max_depth, kernel, eps_rel=1e-7):
    """Leveled KIFMM setup (kifmm/setup.py:19-226 with HFMM's arguments)."""
    x = np.asarray(positions, dtype=np.float64)
    if x.ndim != 2 or x.shape[1] != 3 or x.shape[0] == 0:
        raise ValueError("positions: expected a nonempty (N, 3) array")
    t, mb, md, maxleaf = build_fmm_tree_auto(x, N_max=N_max, max_depth=max_depth)
    m_id, p_id, lvls, counts, is_leaf = (t[k] for k in ("m_id", "p_id", "lvls", "counts", "is_leaf"))
    leaf = is_leaf & (lvls > 0)
    adaptive = np.unique(lvls[leaf]).size > 1
    V = build_v(m_id, lvls, is_leaf, md)
    U = build_u(m_id, lvls, is_leaf, md)
    W = X = None
    if adaptive:
        Wn, Xn = build_wx(m_id, lvls, is_leaf, md)
        W = Wn if Wn.shape[0] else None
        X = Xn if Xn.shape[0] else None
    dc = near_pairs(U, lvls, is_leaf)
    _, pil = assign_particles(t["sort_idx"], m_id, lvls, counts, is_leaf, md, maxleaf)
    ops = build_operators_leveled(p, md, float(t["domain_extent"]), kernel.G_np, eps_rel,
                                  m2l_from_level=2)   # V pairs start at level 2
    return dict(positions=x, pil=pil, dir_cnct=dc, V=V, U=U, W=W, X=X, m_id=m_id, p_id=p_id,
                lvls=lvls, counts=counts, is_leaf=is_leaf, sort_idx=t["sort_idx"],
                domain_extent=float(t["domain_extent"]), pmin=t["pmin"], ops=ops,
                max_depth=int(md), maxleaf=int(maxleaf), adaptive=bool(adaptive),
                max_boxes=int(mb), kernel=kernel, p=int(p))


def setup(positions, k, p=4, N_max=16, max_depth=None):
    """HFMM.setup (HFMM.py:55-80)."""
    x = np.asarray(positions, dtype=np.float64)
    if x.ndim != 2 or x.shape[1] != 3 or len(x) == 0 or not np.isfinite(x).all():
        raise ValueError("positions must be a nonempty finite (N,3) array")
    if p < 2 or int(p) != p or N_max < 1 or int(N_max) != N_max:
        raise ValueError("p must be an integer >=2; N_max must be a positive integer")
    if max_depth is not None and (max_depth < 1 or int(max_depth) != max_depth):
        raise ValueError("max_depth must be a positive integer or None")
    kr = HelmholtzComponent(k, False)
    real = kifmm_setup(x, int(p), int(N_max), max_depth, kr)
    if float(k) == 0:
        return real, None
    ki = HelmholtzComponent(k, True)
    imag_ops = build_operators_leveled(int(p), real["max_depth"], float(real["domain_extent"]),
                                       ki.G_np, eps_rel=1e-12, m2l_from_level=2)
    return real, dict(real, ops=imag_ops, kernel=ki)


# ---------------------------------------------------------------- phases
def _decode(X, F):
    """((X @ U) * d) @ Vt over the last axis (phases.py:21-34)."""
    U, d, Vt = F
    return ((X @ U) * d) @ Vt


def _decode_leveled(X, F_lv, lvls, md):
    """Per-box decode with the box level's factors (phases.py:69-76)."""
    out = np.zeros_like(X)
    for l in range(md + 1):
        rows = np.nonzero(lvls == l)[0]
        if rows.size:
            out[rows] = _decode(X[rows], tuple(f[l] for f in F_lv))
    return out


def _build_padded(positions, Q, pil):
    """Padded per-box points/charges and the gather-out map (near.py:589-598)."""
    mb, w = pil.shape
    N = positions.shape[0]
    valid = pil >= 0
    safe = np.where(valid, pil, 0)
    ppts = positions[safe]
    pchg = np.where(valid[..., None], Q[safe], 0.0)            # (mb, w, R)
    flat = np.arange(mb * w, dtype=np.int64).reshape(mb, w)
    rev = np.zeros(N, dtype=np.int64)
    rev[pil[valid]] = flat[valid]
    return ppts, pchg, rev


def p2m(s, kern, ppts, pchg, centres, h):
    """Leaf check potentials, then the level decode (phases.py:79-125)."""
    ops = s["ops"]
    mb, R = ppts.shape[0], pchg.shape[2]
    check = np.zeros((mb, R, ops["n_s"]))
    leaves = np.nonzero(s["is_leaf"])[0]
    for lo in range(0, leaves.size, 256):
        b = leaves[lo:lo + 256]
        cp = ops["check_pts"][None] * h[b][:, None, None] + centres[b][:, None, :]
        d = cp[:, :, None, :] - ppts[b][:, None, :, :]
        K = kern.g_box(np.sqrt(np.sum(d * d, axis=-1)))        # (B, n_s, w)
        check[b] = np.einsum("bjw,bwr->brj", K, pchg[b])
    return check


def m2m_check(s, equiv, cl):
    """Child level ``cl`` -> parent check potentials (phases.py:163-171)."""
    ops = s["ops"]
    pl = cl - 1
    K = ops["M2M_K_lv"][pl]
    check = np.zeros_like(equiv)
    kids = np.nonzero(s["lvls"] == cl)[0]
    octs = (s["m_id"][kids] % np.uint64(8)).astype(np.int64)
    for o in range(8):
        b = kids[octs == o]
        if b.size:
            np.add.at(check, s["p_id"][b], equiv[b] @ K[o].T)
    return check


def _disp_ids(s, tgt, src):
    gx, gy, gz = (c.astype(np.int64) for c in morton_decode(s["m_id"]))
    return (gx[tgt] - gx[src] + 3) * 49 + (gy[tgt] - gy[src] + 3) * 7 + (gz[tgt] - gz[src] + 3)


def m2l_check(s, equiv):
    """V-list check potentials grouped by (target level, displacement) (phases.py:211-236)."""
    ops = s["ops"]
    check = np.zeros_like(equiv)
    V = s["V"]
    if V.shape[0] == 0:
        return check
    tgt, src = V[:, 0].astype(np.int64), V[:, 1].astype(np.int64)
    key = s["lvls"][tgt].astype(np.int64) * 343 + _disp_ids(s, tgt, src)
    order = np.argsort(key, kind="stable")
    ks = key[order]
    cuts = np.nonzero(np.diff(ks))[0] + 1
    for grp in np.split(order, cuts):
        kk = key[grp[0]]
        A = ops["M2L_K_lv"][kk // 343][kk % 343]
        check[tgt[grp]] += equiv[src[grp]] @ A.T           # targets unique per group
    return check


def p2l_check(s, kern, positions, Q, centres, h):
    """X-list check potentials at the target's downward check surface (phases.py:1755-1769)."""
    ops = s["ops"]
    R = Q.shape[1]
    out = np.zeros((s["m_id"].shape[0], R, ops["n_s"]))
    per_pair = []
    X = s["X"]
    if X is None:
        return out, per_pair
    pil = s["pil"]
    for t, sb in X:
        idx = pil[sb]
        valid = idx >= 0
        idx_s = np.where(valid, idx, 0)
        q = np.where(valid[:, None], Q[idx_s], 0.0)
        cp = ops["equiv_pts"] * h[t] + centres[t]
        d = cp[:, None, :] - positions[idx_s][None, :, :]
        K = kern.g_box(np.sqrt(np.sum(d * d, axis=-1))[None])[0]
        per_pair.append((t, (K @ q).T))
    return out, per_pair


def l2l_check(s, loc, cl):
    """Parent locals -> child check potentials at child level ``cl`` (phases.py:273-278)."""
    ops = s["ops"]
    K = ops["L2L_K_lv"][cl - 1]
    check = np.zeros_like(loc)
    kids = np.nonzero(s["lvls"] == cl)[0]
    octs = (s["m_id"][kids] % np.uint64(8)).astype(np.int64)
    for o in range(8):
        b = kids[octs == o]
        if b.size:
            check[b] = loc[s["p_id"][b]] @ K[o].T
    return check


def l2p(s, kern, loc, ppts, rev, centres, h, field):
    """Leaf local -> particle potential or field, gathered by ``rev`` (phases.py:1571-1582)."""
    ops = s["ops"]
    mb, w = ppts.shape[:2]
    R = loc.shape[1]
    out = np.zeros((mb, w, R, 3) if field else (mb, w, R))
    leaves = np.nonzero(s["is_leaf"])[0]
    for lo in range(0, leaves.size, 64):
        b = leaves[lo:lo + 64]
        ep = ops["check_pts"][None] * h[b][:, None, None] + centres[b][:, None, :]
        d = ppts[b][:, :, None, :] - ep[:, None, :, :]          # (B, w, n_s, 3)
        if field:
            out[b] = np.einsum("bwjc,brj->bwrc", kern.g_grad_box(d), loc[b])
        else:
            K = kern.g_box(np.sqrt(np.sum(d * d, axis=-1)))
            out[b] = np.einsum("bwj,brj->bwr", K, loc[b])
    flat = out.reshape((mb * w,) + out.shape[2:])
    return flat[rev]


def m2p(s, kern, equiv, positions, centres, h, field):
    """W-list source equivalents evaluated at target-leaf particles (phases.py:1101-1140)."""
    ops = s["ops"]
    N = positions.shape[0]
    R = equiv.shape[1]
    pot = np.zeros((N, R, 3) if field else (N, R))
    if s["W"] is None:
        return pot
    pil = s["pil"]
    for t, sb in s["W"]:
        idx = pil[t]
        valid = idx >= 0
        idx_s = np.where(valid, idx, 0)
        ep = ops["equiv_pts"] * h[sb] + centres[sb]
        d = positions[idx_s][:, None, :] - ep[None, :, :]
        if field:
            c = np.einsum("pjc,rj->prc", kern.g_grad_box(d[None])[0], equiv[sb])
            c = np.where(valid[:, None, None], c, 0.0)
        else:
            K = kern.g_box(np.sqrt(np.sum(d * d, axis=-1))[None])[0]
            c = np.where(valid[:, None], K @ equiv[sb].T, 0.0)
        np.add.at(pot, idx_s, c)
    return pot


def eval_direct(s, kern, ppts, pchg, rev, field, batch=512):
    """Flat P2P over the near pairs with the pair coincidence floor (near.py:193-312)."""
    dc = s["dir_cnct"]
    mb, w = ppts.shape[:2]
    R = pchg.shape[2]
    buf = np.zeros((mb, w, R, 3) if field else (mb, w, R))
    feps = min(EPS, float(np.finfo(np.float32).eps))
    # A row's real points come first, its padding (point 0 again, charge 0) after them.
    # Padded sources add 0 and padded targets are dropped, so with the state's "pil"
    # each batch is cut to its widest real row (pairs run narrowest first so that a
    # batch's rows are alike); the floor's scale still takes the maximum over the whole
    # padded row, as near.py does. near_trim=False in the state (or no "pil") evaluates
    # every padded slot, as the reference does: the CPU cost the benchmark times.
    pil = s.get("pil") if s.get("near_trim", True) else None
    nv = (pil >= 0).sum(axis=1) if pil is not None else np.full(mb, w)
    width = np.maximum(nv[dc[:, 0]], nv[dc[:, 1]])
    order = np.argsort(width, kind="stable")
    n_pairs, lo = dc.shape[0], 0
    while lo < n_pairs:
        w_hi = int(width[order[min(lo + batch, n_pairs) - 1]])
        hi = min(n_pairs, lo + max(1, min(batch, (1 << 22) // max(1, w_hi * w_hi))))
        pr = dc[order[lo:hi]]
        lo = hi
        we, ws = max(1, int(nv[pr[:, 0]].max())), max(1, int(nv[pr[:, 1]].max()))
        kt_row, kp_row = ppts[pr[:, 0]], ppts[pr[:, 1]]       # (B, w, 3), padding included
        rs = np.sqrt(np.max(kp_row[..., 0] ** 2 + kp_row[..., 1] ** 2 + kp_row[..., 2] ** 2, axis=1))
        re = np.sqrt(np.max(np.sum(kt_row ** 2, axis=-1), axis=1))
        kt, kp = kt_row[:, :we], kp_row[:, :ws]               # (B, w_e, 3), (B, w_s, 3)
        dd = [kt[:, None, :, c] - kp[:, :, None, c] for c in range(3)]   # (B, w_s, w_e)
        d2 = dd[0] ** 2 + dd[1] ** 2 + dd[2] ** 2
        scale = ((re + rs) ** 2)[:, None, None]
        d2 = np.where(d2 > (16 * feps) ** 2 * scale, d2, 0.0)
        q = pchg[pr[:, 1], :ws]                               # (B, w_s, R)
        if field:
            kw = kern.k2g(d2)
            pot = np.stack([np.einsum("bse,bsr->ber", kw * dd[c], q) for c in range(3)], -1)
        else:
            kw = kern.k2(d2)
            pot = np.einsum("bse,bsr->ber", kw, q)
        np.add.at(buf[:, :we], pr[:, 0], pot)
    flat = buf.reshape((mb * w,) + buf.shape[2:])
    return flat[rev] / (4 * np.pi)


def evaluate_setup(s, charges, field=False, fused_decode=False, trace=None):
    """Potential (N, R) or field (N, R, 3) of the real KIFMM for charge columns
    (kifmm/setup.py:229-261 -> core.evaluate, core.py:274-335).

    ``trace``: a dict that receives each phase's output, keyed by the phase
    (``s2m``, ``m2m``, ``m2l``, ``p2l``, ``l2l``, ``l2p``, ``p2p``, ``m2p``), at the
    points where core.evaluate hands it to the next phase (core.py:297-335)."""
    rec = (lambda key, val: trace.__setitem__(key, val)) if trace is not None else (lambda *_: None)
    kern = s["kernel"]
    Q = np.asarray(charges, dtype=np.float64)
    squeeze = Q.ndim == 1
    if squeeze:
        Q = Q[:, None]
    positions = s["positions"]
    md = s["max_depth"]
    ops = s["ops"]
    lvls = s["lvls"]
    centres, h = box_geometry(s["m_id"], lvls, s["domain_extent"], s["pmin"])
    ppts, pchg, rev = _build_padded(positions, Q, s["pil"])

    # upward pass: P2M + decode, then M2M level by level (phases.py:118-125, 163-173)
    equiv = _decode_leveled(p2m(s, kern, ppts, pchg, centres, h), ops["F_up_lv"], lvls, md)
    rec("s2m", equiv)
    for cl in range(md, 1, -1):
        chk = m2m_check(s, equiv, cl)
        pl = cl - 1
        solved = _decode(chk, tuple(f[pl] for f in ops["F_up_lv"]))
        equiv = equiv + np.where((lvls == pl)[:, None, None], solved, 0.0)
    rec("m2m", equiv)

    # downward pass
    m2l_c = m2l_check(s, equiv)
    p2l_c, p2l_pairs = p2l_check(s, kern, positions, Q, centres, h)
    if fused_decode:
        for t, c in p2l_pairs:
            p2l_c[t] += c
        loc = np.zeros_like(equiv)
        for cl in range(2, md + 1):
            rows = np.nonzero(lvls == cl)[0]
            chk = m2l_c + p2l_c
            if cl >= 3:
                chk = chk + l2l_check(s, loc, cl)
            if rows.size:
                loc[rows] = _decode(chk[rows], tuple(f[cl] for f in ops["F_dn_lv"]))
    else:
        loc = _decode_leveled(m2l_c, ops["F_dn_lv"], lvls, md)        # phases.py:237
        rec("m2l", loc.copy())
        for t, c in p2l_pairs:                                         # phases.py:1766-1770
            loc[t] += _decode(c[None], tuple(f[lvls[t]] for f in ops["F_dn_lv"]))[0]
        if p2l_pairs:
            rec("p2l", loc.copy())
        for cl in range(2, md + 1):                                    # phases.py:273-280
            add = _decode(l2l_check(s, loc, cl), tuple(f[cl] for f in ops["F_dn_lv"]))
            loc = loc + np.where((lvls == cl)[:, None, None], add, 0.0)
    rec("l2l", loc)

    far = l2p(s, kern, loc, ppts, rev, centres, h, field)
    near = eval_direct(s, kern, ppts, pchg, rev, field)
    rec("l2p", far)
    rec("p2p", near)
    pot = far + near
    if s["W"] is not None:
        mp = m2p(s, kern, equiv, positions, centres, h, field)
        rec("m2p", mp)
        pot = pot + mp
    return pot[:, 0] if squeeze else pot


def evaluate(state, charges):
    """HFMM.evaluate (HFMM.py:83-91): real charges -> complex128 potential."""
    q = np.asarray(charges)
    if q.shape != (state[0]["positions"].shape[0],) or np.iscomplexobj(q):
        raise ValueError("charges must be a real array of shape (N,)")
    q = q.astype(np.float64)
    real = evaluate_setup(state[0], q)
    imag = evaluate_setup(state[1], q) if state[1] is not None else np.zeros_like(real)
    return real + 1j * imag


def evaluate_complex(state, charges, field=False, fused_decode=False):
    """Complex charges (and optionally the field -grad phi) by linearity:
    phi = E_cos(q_re) - E_sin(q_im) + i (E_sin(q_re) + E_cos(q_im))."""
    q = np.asarray(charges).astype(np.complex128)
    Q = np.stack([q.real, q.imag], 1)
    ec = evaluate_setup(state[0], Q, fused_decode=fused_decode)
    es = (evaluate_setup(state[1], Q, fused_decode=fused_decode) if state[1] is not None
          else np.zeros_like(ec))
    phi = (ec[:, 0] - es[:, 1]) + 1j * (es[:, 0] + ec[:, 1])
    if not field:
        return phi
    fc = evaluate_setup(state[0], Q, field=True, fused_decode=fused_decode)
    fs = (evaluate_setup(state[1], Q, field=True, fused_decode=fused_decode)
          if state[1] is not None else np.zeros_like(fc))
    E = (fc[:, 0] - fs[:, 1]) + 1j * (fs[:, 0] + fc[:, 1])
    return phi, E


# ---------------------------------------------------------------- referee
def direct(positions, charges, k, targets=None):
    """O(N*S) sum of q e^{ikr}/r over j != i (test.py:11-18), optionally at a subset."""
    pos = np.asarray(positions, dtype=np.float64)
    q = np.asarray(charges)
    tg = np.arange(len(pos)) if targets is None else np.asarray(targets)
    out = np.empty(len(tg), dtype=np.complex128)
    for lo in range(0, len(tg), 256):
        x = pos[tg[lo:lo + 256]]
        r = np.linalg.norm(x[:, None, :] - pos[None, :, :], axis=-1)
        wgt = np.where(r > 0, np.exp(1j * k * r) / np.where(r > 0, r, 1.0), 0.0)
        out[lo:lo + len(x)] = wgt @ q
    return out


def direct_field(positions, charges, k, targets=None):
    """-grad phi of the direct sum: sum q e^{ikr}(1 - ikr)/r^3 (x - y)."""
    pos = np.asarray(positions, dtype=np.float64)
    q = np.asarray(charges)
    tg = np.arange(len(pos)) if targets is None else np.asarray(targets)
    out = np.empty((len(tg), 3), dtype=np.complex128)
    for lo in range(0, len(tg), 128):
        x = pos[tg[lo:lo + 128]]
        d = x[:, None, :] - pos[None, :, :]
        r = np.linalg.norm(d, axis=-1)
        rs = np.where(r > 0, r, 1.0)
        wgt = np.where(r > 0, np.exp(1j * k * r) * (1 - 1j * k * r) / rs ** 3, 0.0)
        out[lo:lo + len(x)] = np.einsum("ts,tsc,s->tc", wgt, d, q)
    return out


def relative_error(actual, reference):
    """test.py:20-22."""
    norm = np.linalg.norm(reference)
    return float(np.linalg.norm(actual - reference) / (norm if norm else 1.0))
