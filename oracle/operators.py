"""Oracle: per-level KIFMM operator tables for the Helmholtz kernels.

Test infrastructure only. Restates the parts of jaxfmm/kifmm/operators.py that
the HFMM (leveled) path consumes:

* ``_pinv_factors`` (operators.py:72-99): damped SVD factors
  ``U, s/(s^2+(eps_rel*s_max)^2), Vt``;
* ``build_operators`` (operators.py:276-425) restricted to the members the
  leveled phases read (``F_up``, ``F_dn``, ``M2M_K``, ``L2L_K``, ``M2L_K_table``);
* ``build_operators_leveled`` (operators.py:572-641): one set per level with the
  scaled kernel ``G(s*x, s*y)``, ``s = extent * 0.5**(l+1)``.

The Helmholtz component kernel is HFMM.py:20-23 (``cos|sin(k r)/r`` with an
ULP-relative zero at r ~ 0, no 1/(4 pi)).
"""
import numpy as np

from .surfaces import surface_pts, R_EQUIV, R_CHECK

# Child-octant centres in parent coordinates (operators.py:64-69): bit0=x, bit1=y, bit2=z.
CHILD_OFFSETS = np.array([(-1, -1, -1), (1, -1, -1), (-1, 1, -1), (1, 1, -1),
                          (-1, -1, 1), (1, -1, 1), (-1, 1, 1), (1, 1, 1)], dtype=np.float64)


def helmholtz_G_np(k, imaginary):
    """Host kernel-matrix function of HFMM.py:12-23 for one trig component."""
    k = float(k)
    if not np.isfinite(k):
        raise ValueError("k must be a finite real number")
    trig = np.sin if imaginary else np.cos

    def G(x, y):
        # |x - y| as np.linalg.norm(axis=-1) forms it, (dx^2 + dy^2) + dz^2, one
        # component at a time instead of through an (n, m, 3) array
        r = None
        for c in range(3):
            dc = x[:, c, None] - y[None, :, c]
            r = dc * dc if r is None else r + dc * dc
        np.sqrt(r, out=r)
        ok = r > 16 * np.finfo(r.dtype).eps * r.max(initial=0.0)
        return np.where(ok, trig(k * r) / np.where(ok, r, 1.0), 0.0)
    return G


def pinv_factors(A, eps_rel=1e-7):
    """Damped pseudoinverse factors (operators.py:72-99)."""
    U, s, Vt = np.linalg.svd(A, full_matrices=False)
    eps = eps_rel * s[0]
    return U, s / (s * s + eps * eps), Vt


def build_operators(p, G, eps_rel=1e-7, m2l_out=None, with_m2l=True):
    """Unit-box operator set for kernel matrix function ``G`` (operators.py:330-403).

    Returns the members the leveled path uses. ``M2L_K_table`` has shape
    (343, n_s, n_s) in displacement order ``(dx+3)*49 + (dy+3)*7 + (dz+3)`` with
    zero matrices at the 27 adjacent displacements; ``m2l_out``, if given, is the
    zeroed array it is written into; ``with_m2l=False`` leaves it zero.
    """
    equiv = surface_pts(p, R_EQUIV)
    check = surface_pts(p, R_CHECK)
    n_s = equiv.shape[0]
    F_up = pinv_factors(G(check, equiv), eps_rel)
    F_dn = pinv_factors(G(equiv, check), eps_rel)
    parent_check = check * 2.0
    M2M_K = np.empty((8, n_s, n_s))
    for c in range(8):
        M2M_K[c] = G(parent_check, equiv + CHILD_OFFSETS[c])
    M2L = np.zeros((343, n_s, n_s)) if m2l_out is None else m2l_out
    for dxi in range(7 if with_m2l else 0):
        for dyi in range(7):
            for dzi in range(7):
                dx, dy, dz = dxi - 3, dyi - 3, dzi - 3
                if max(abs(dx), abs(dy), abs(dz)) <= 1:
                    continue
                d_vec = np.array([2.0 * dx, 2.0 * dy, 2.0 * dz])
                M2L[dxi * 49 + dyi * 7 + dzi] = G(equiv + d_vec, equiv)
    parent_equiv_dn = check * 2.0
    L2L_K = np.empty((8, n_s, n_s))
    for c in range(8):
        L2L_K[c] = G(equiv + CHILD_OFFSETS[c], parent_equiv_dn)
    return dict(F_up=F_up, F_dn=F_dn, M2M_K=M2M_K, L2L_K=L2L_K, M2L_K_table=M2L,
                equiv_pts=equiv, check_pts=check, n_s=n_s, p=p)


def build_operators_leveled(p, max_depth, domain_extent, G, eps_rel=1e-7, m2l_from_level=0):
    """Per-level tables (operators.py:572-641).

    ``M2M_K_lv[pl]`` (parent level pl) and ``L2L_K_lv[cl-1]`` (child level cl) are
    both taken from the CHILD level's assembly, as in the reference. M2L tables of the
    levels below ``m2l_from_level`` are left zero: ``setup`` passes 2, the first level
    with V pairs; the reference builds them and never reads them.
    """
    n_s = surface_pts(p, R_EQUIV).shape[0]
    m2l = np.zeros((max_depth + 1, 343, n_s, n_s))   # filled in place, level by level
    per = []
    for l in range(max_depth + 1):
        s = float(domain_extent) * 0.5 ** (l + 1)
        Gs = (lambda x, y, _s=s: G(x * _s, y * _s))
        per.append(build_operators(p, Gs, eps_rel, m2l_out=m2l[l], with_m2l=l >= m2l_from_level))

    def stack_f(key):
        return tuple(np.stack([np.asarray(o[key][i]) for o in per]) for i in range(3))
    return dict(
        max_depth=int(max_depth), p=p, n_s=per[0]["n_s"],
        equiv_pts=per[0]["equiv_pts"], check_pts=per[0]["check_pts"],
        F_up_lv=stack_f("F_up"), F_dn_lv=stack_f("F_dn"),
        M2M_K_lv=np.stack([per[pl + 1]["M2M_K"] for pl in range(max_depth)]),
        L2L_K_lv=np.stack([per[cl]["L2L_K"] for cl in range(1, max_depth + 1)]),
        M2L_K_lv=m2l,
    )
