"""Host precompute of the per-level KIFMM operator tables (float64, NumPy).

Setup-time work, the same split the reference makes (operator assembly in host
NumPy, jaxfmm/kifmm/operators.py:276-425 and 572-641; surfaces in
kifmm/surfaces.py:40-85). Each table entry is computed with exactly the
reference's NumPy expression, so the library consumes the tables the reference
would build:

* the Helmholtz component matrix ``cos|sin(k r)/r`` with an ULP-relative zero
  (HFMM.py:20-23), scaled per level as ``G(s x, s y)``, ``s = extent * 2^-(l+1)``
  (operators.py:616-621);
* damped-SVD decode factors ``U, s/(s^2 + (eps_rel s_max)^2), Vt``
  (operators.py:72-99); ``eps_rel`` is 1e-7 for the cos component and 1e-12 for
  the sin component (HFMM.py:75-77);
* M2M child kernels of the parent level taken from the child level's assembly,
  L2L kernels of the child level, and the 7x7x7 M2L raw-kernel table
  (operators.py:363-403, 633-640).

Only levels 2..max_depth are built: levels 0 and 1 have no V, W or X pairs, so
their tables would never be read.
"""
import numpy as np

R_EQUIV = 1.05
R_CHECK = 2.95
CHILD_OFFSETS = np.array([(-1, -1, -1), (1, -1, -1), (-1, 1, -1), (1, 1, -1),
                          (-1, -1, 1), (1, -1, 1), (-1, 1, 1), (1, 1, 1)], dtype=np.float64)


def n_surf(p):
    """6p^2 - 12p + 8 surface points (kifmm/surfaces.py:24-37)."""
    return 6 * p * p - 12 * p + 8


def surface_pts(p, r):
    """Cube-surface grid of p x p points per face, duplicates removed in first-occurrence
    order (kifmm/surfaces.py:40-85)."""
    if p < 2:
        raise ValueError(f"p must be >= 2, got {p}")
    t = np.linspace(-r, r, p)
    a, b = np.meshgrid(t, t, indexing="ij")
    a, b = a.reshape(-1), b.reshape(-1)
    f = np.full(p * p, r)
    pts = np.vstack([np.stack(c, 1) for c in ((f, a, b), (-f, a, b), (a, f, b), (a, -f, b),
                                               (a, b, f), (a, b, -f))])
    _, first = np.unique(np.round(pts / max(r, 1e-300), 14), axis=0, return_index=True)
    return pts[np.sort(first)]


def component_matrix(k, imaginary):
    """G(x, y) = trig(k |x - y|) / |x - y| with the ULP-relative zero of HFMM.py:20-23."""
    trig = np.sin if imaginary else np.cos
    k = float(k)

    def G(x, y):
        r = np.linalg.norm(x[:, None, :] - y[None, :, :], axis=-1)
        ok = r > 16 * np.finfo(r.dtype).eps * r.max(initial=0.0)
        return np.where(ok, trig(k * r) / np.where(ok, r, 1.0), 0.0)
    return G


def screened_matrix(kappa):
    """G(x, y) = exp(-kappa r) / (4 pi r) with the ULP-relative zero, the reference's
    yukawa G_np (jaxfmm/kernels/yukawa/kernel.py:36-42); kappa = 0 gives its Laplace
    G_np 1 / (4 pi r) (kernels/laplace/kernel.py:40-43) to the last bit."""
    kappa = float(kappa)

    def G(x, y):
        d = x[:, None, :] - y[None, :, :]
        r = np.sqrt((d ** 2).sum(-1))
        with np.errstate(divide="ignore", invalid="ignore"):
            K = np.exp(-kappa * r) / (4.0 * np.pi * r)
        K[r <= 16 * np.finfo(r.dtype).eps * r.max(initial=0.0)] = 0.0
        return K
    return G


def family_matrix(k, imaginary, kind="helmholtz"):
    """The kernel matrix of one family: a Helmholtz component, or the screened-Coulomb
    kernel (kind "yukawa", k = kappa; one family)."""
    return screened_matrix(k) if kind == "yukawa" else component_matrix(k, imaginary)


def damped_factors(A, eps_rel):
    U, s, Vt = np.linalg.svd(A, full_matrices=False)
    eps = eps_rel * s[0]
    return U, s / (s * s + eps * eps), Vt


def level_scale(domain_extent, level):
    return float(domain_extent) * 0.5 ** (level + 1)


def level_decodes(p, level, domain_extent, k, imaginary, eps_rel, kind="helmholtz"):
    """Only the two damped-SVD decodes of one family at one level (the kernel matrices
    are then generated on the device, hfmm_plan_set_level_decode)."""
    G = family_matrix(k, imaginary, kind)
    equiv = surface_pts(p, R_EQUIV)
    check = surface_pts(p, R_CHECK)
    s = level_scale(domain_extent, level)
    F_up = damped_factors(G(check * s, equiv * s), eps_rel)
    F_dn = damped_factors(G(equiv * s, check * s), eps_rel)
    return dict(F_up=F_up, F_dn=F_dn)


def level_tables(p, level, max_depth, domain_extent, k, imaginary, eps_rel, kind="helmholtz"):
    """Tables of one kernel family at one level, in the layout hfmm_plan_set_level takes."""
    G = family_matrix(k, imaginary, kind)
    equiv = surface_pts(p, R_EQUIV)
    check = surface_pts(p, R_CHECK)
    n_s = equiv.shape[0]
    s = level_scale(domain_extent, level)

    def Gs(x, y, sc=s):
        return G(x * sc, y * sc)

    F_up = damped_factors(Gs(check, equiv), eps_rel)
    F_dn = damped_factors(Gs(equiv, check), eps_rel)
    m2l = np.zeros((343, n_s, n_s))
    for dxi in range(7):
        for dyi in range(7):
            for dzi in range(7):
                d = (dxi - 3, dyi - 3, dzi - 3)
                if max(abs(c) for c in d) <= 1:
                    continue
                dv = np.array([2.0 * d[0], 2.0 * d[1], 2.0 * d[2]])
                m2l[dxi * 49 + dyi * 7 + dzi] = Gs(equiv + dv, equiv)
    l2l = None
    if level >= 3:
        l2l = np.stack([Gs(equiv + CHILD_OFFSETS[c], check * 2.0) for c in range(8)])
    m2m = None
    if level < max_depth:
        sc = level_scale(domain_extent, level + 1)   # parent level couples children at level+1
        m2m = np.stack([Gs(check * 2.0, equiv + CHILD_OFFSETS[c], sc) for c in range(8)])
    return dict(F_up=F_up, F_dn=F_dn, M2M_K=m2m, L2L_K=l2l, M2L_K=m2l, n_s=n_s)
