"""Oracle: KIFMM cube-surface point sets (test infrastructure only).

Restates jaxfmm/kifmm/surfaces.py:20-85: a p x p grid on each of the six faces of
a cube of half-side r, duplicate edge/corner points removed by 14-digit rounding
and ``np.unique(..., return_index=True)``, original first-occurrence order kept.
"""
import numpy as np

R_EQUIV = 1.05   # surfaces.py:21 (upward equivalent / downward check)
R_CHECK = 2.95   # surfaces.py:22 (upward check / downward equivalent)


def n_surf(p):
    """Unique surface points for p points per cube edge (surfaces.py:24-37)."""
    return 6 * p * p - 12 * p + 8


def surface_pts(p, r=1.0):
    """(n_surf(p), 3) surface points at half-side ``r`` (surfaces.py:40-85)."""
    if p < 2:
        raise ValueError(f"p must be >= 2, got {p}")
    t = np.linspace(-r, r, p)
    g0, g1 = np.meshgrid(t, t, indexing="ij")
    g0 = g0.reshape(-1)
    g1 = g1.reshape(-1)
    c = r * np.ones(p * p)
    faces = [np.stack([+c, g0, g1], 1), np.stack([-c, g0, g1], 1),
             np.stack([g0, +c, g1], 1), np.stack([g0, -c, g1], 1),
             np.stack([g0, g1, +c], 1), np.stack([g0, g1, -c], 1)]
    pts = np.vstack(faces)
    key = np.round(pts / max(r, 1e-300), 14)
    _, first = np.unique(key, axis=0, return_index=True)
    return pts[np.sort(first)]
