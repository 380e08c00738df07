"""What a per-level expansion order would buy, measured with the oracle's operators:
the error of one KIFMM far-field translation (P2M + upward decode, M2L at the nearest
face displacement, downward decode, evaluation at target points; both kernel
families, the damped pseudo-inverses of kifmm/operators.py:72-99) against the direct
sum, as a function of p and the box's k x side. Up to k x side ~ 1.25 (2.5 from p = 8
on) the error sits at its low-frequency floor for each p; above it the order must
grow with k x side. So on a deep tree at large k only the coarse levels need the
high order."""
import numpy as np

from oracle.operators import helmholtz_G_np, pinv_factors
from oracle.surfaces import surface_pts, R_EQUIV, R_CHECK


def _decode(F, v):
    U, d, Vt = F
    return ((v @ U) * d) @ Vt


def translation_error(p, k, side, seed=0):
    s = side / 2
    rng = np.random.default_rng(seed)
    src = rng.uniform(-s, s, (300, 3))
    q = rng.normal(size=300)
    c_t = np.array([2.0, 0.0, 0.0]) * side          # nearest V displacement (2, 0, 0)
    tgt = c_t + rng.uniform(-s, s, (300, 3))
    worst = 0.0
    for imag, eps in ((False, 1e-7), (True, 1e-12)):
        G = helmholtz_G_np(k, imag)
        eq_u, ck_u = surface_pts(p, R_EQUIV) * s, surface_pts(p, R_CHECK) * s
        ck_d, eq_d = surface_pts(p, R_EQUIV) * s + c_t, surface_pts(p, R_CHECK) * s + c_t
        x = _decode(pinv_factors(G(ck_u, eq_u), eps), (G(ck_u, src) @ q)[None])[0]
        y = _decode(pinv_factors(G(ck_d, eq_d), eps), (G(ck_d, eq_u) @ x)[None])[0]
        ref = G(tgt, src) @ q
        worst = max(worst, np.linalg.norm(G(tgt, eq_d) @ y - ref) / np.linalg.norm(ref))
    return worst


def test_low_frequency_levels_share_one_floor_per_order():
    """Up to k x side 1.25 an order reaches the same error at every level (within 2x of
    k x side 0.31, the finest level of 1e6 points at k = 10); at p = 8 that holds up to
    k x side 2.5, the coarsest level there, while p = 6 is already 5x off at 2.5."""
    for p in (6, 8):
        fine, mid = translation_error(p, 10.0, 2 ** -5), translation_error(p, 10.0, 2 ** -3)
        assert max(fine, mid) < 2 * min(fine, mid), (p, fine, mid)
    fine8, coarse8 = translation_error(8, 10.0, 2 ** -5), translation_error(8, 10.0, 2 ** -2)
    assert coarse8 < 2 * fine8 and coarse8 < 1.5e-6
    assert translation_error(6, 10.0, 2 ** -2) > 3 * translation_error(6, 10.0, 2 ** -5)


def test_high_frequency_levels_need_a_higher_order():
    """k x side 10 (level 2 at k = 40): p = 8 misses 1e-6 by more than an order of
    magnitude, p = 10 meets it; one level down (k x side 5) p = 9 does."""
    assert translation_error(8, 40.0, 2 ** -2) > 1e-5
    assert translation_error(10, 40.0, 2 ** -2) < 5e-7
    assert translation_error(9, 40.0, 2 ** -3) < 1e-6
