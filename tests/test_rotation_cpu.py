"""Host math of the rotation-based M2L (hfmm_b200/rotation.py), on the CPU: the
coaxial coefficients against a numerical projection of the shifted singular
solutions, the rotation blocks' unitarity, and the whole rotate - shift - rotate
operator against the dense KIFMM M2L matrix of the same level and displacement."""
import numpy as np
import pytest
from numpy.polynomial.legendre import leggauss
from scipy.special import sph_harm_y, spherical_jn, spherical_yn

from hfmm_b200 import operators as O, rotation as rot


def _sphere(nq):
    x, w = leggauss(nq)
    th = np.arccos(x)
    ph = np.linspace(0, 2 * np.pi, 2 * nq, endpoint=False)
    TH, PH = np.meshgrid(th, ph, indexing="ij")
    W = np.outer(w, np.full(2 * nq, 2 * np.pi / (2 * nq)))
    return TH, PH, W


@pytest.mark.parametrize("regular", [False, True])
def test_coaxial_coefficients_match_projection(regular):
    """Shift y_n (or j_n) Y_nm by t along z and project onto j_n' Y_n'm on a sphere of
    radius a < t: at k a = 1.5 the low orders are resolved to rounding."""
    k, t, a, P = 10.0, 0.4, 0.15, 6
    z = spherical_jn if regular else spherical_yn
    C = rot.coaxial(P, k, t, regular)
    TH, PH, W = _sphere(24)
    pts = np.stack([a * np.sin(TH) * np.cos(PH), a * np.sin(TH) * np.sin(PH), a * np.cos(TH)], -1)
    v = pts + np.array([0.0, 0.0, t])
    r = np.linalg.norm(v, axis=-1)
    th, ph = np.arccos(v[..., 2] / r), np.arctan2(v[..., 1], v[..., 0])
    for n, m, n2 in [(0, 0, 0), (1, 0, 1), (2, 1, 1), (3, -2, 4), (4, 2, 2), (5, 3, 6)]:
        f = z(n, k * r) * sph_harm_y(n, m, th, ph)
        num = np.sum(W * f * np.conj(sph_harm_y(n2, m, TH, PH))) / spherical_jn(n2, k * a)
        assert abs(C[m + P, n2, n] - num) <= 1e-11 * max(1.0, abs(num)), (n, m, n2)


def test_wigner_3j_known_values_and_orthogonality():
    """Tabulated symbols ((j j 0; m -m 0) = (-1)^(j-m) / sqrt(2j+1) and two (j1 j2 j3; 0 0 0))
    and the orthogonality sum over m1, m2 of products with equal (j1, j2)."""
    w = rot.wigner_3j
    for j in range(6):
        for m in range(-j, j + 1):
            assert abs(w(j, j, 0, m, -m, 0) - (-1) ** (j - m) / np.sqrt(2 * j + 1)) < 1e-15
    assert abs(w(1, 1, 2, 0, 0, 0) - np.sqrt(2 / 15)) < 1e-15
    assert abs(w(2, 2, 2, 0, 0, 0) + np.sqrt(2 / 35)) < 1e-15
    assert w(1, 1, 1, 0, 0, 0) == 0.0 and w(2, 3, 7, 0, 0, 0) == 0.0   # parity, triangle
    for j1, j2 in ((3, 5), (7, 4), (12, 9)):
        for j3 in range(abs(j1 - j2), j1 + j2 + 1):
            for j3b in (j3, min(j3 + 1, j1 + j2)):
                m3 = min(j3, j3b) // 2
                tot = sum(w(j1, j2, j3, m1, -m1 - m3, m3) * w(j1, j2, j3b, m1, -m1 - m3, m3)
                          for m1 in range(-j1, j1 + 1) if abs(m1 + m3) <= j2)
                assert abs(tot - (j3 == j3b) / (2 * j3 + 1)) < 1e-14, (j1, j2, j3, j3b)


@pytest.mark.parametrize("P", [0, 1, 7, 24, 40])
def test_harmonics_recurrence_matches_scipy(P):
    rng = np.random.default_rng(P)
    th = np.arccos(rng.uniform(-1, 1, 300))
    th[:2] = 0.0, np.pi   # the poles
    ph = rng.uniform(-np.pi, np.pi, 300)
    n = np.array([a for a in range(P + 1) for _ in range(-a, a + 1)])
    m = np.array([b for a in range(P + 1) for b in range(-a, a + 1)])
    ref = sph_harm_y(n[:, None], m[:, None], th[None, :], ph[None, :])
    assert np.abs(rot._harmonics(P, th, ph) - ref).max() < 1e-13


def test_rotation_blocks_are_unitary_and_rotate():
    P = 8
    d = np.array([2.0, -1.0, 3.0])
    R = rot.rotation_to_z(d)
    assert np.allclose(R @ d / np.linalg.norm(d), [0, 0, 1]) and np.isclose(np.linalg.det(R), 1)
    T = rot.rotation_blocks(P, R)
    for n, t in enumerate(T):
        assert np.allclose(t @ t.conj().T, np.eye(2 * n + 1), atol=1e-12)
    # a function's coefficients in the rotated frame reproduce it at rotated points
    rng = np.random.default_rng(0)
    a = rng.normal(size=2 * P + 1) + 1j * rng.normal(size=2 * P + 1)
    s = rng.normal(size=(5, 3))
    s /= np.linalg.norm(s, axis=1, keepdims=True)
    th, ph = np.arccos(s[:, 2]), np.arctan2(s[:, 1], s[:, 0])
    f = sum(a[i] * sph_harm_y(P, m, th, ph) for i, m in enumerate(range(-P, P + 1)))
    b = T[P] @ a
    sr = s @ R.T
    th2, ph2 = np.arccos(np.clip(sr[:, 2], -1, 1)), np.arctan2(sr[:, 1], sr[:, 0])
    g = sum(b[i] * sph_harm_y(P, m, th2, ph2) for i, m in enumerate(range(-P, P + 1)))
    assert np.allclose(f, g, atol=1e-12)


def test_slot_rotations_factor_into_real_y_rotations_and_phases():
    """Every V slot: R_y(-theta) R_z(-phi) takes the displacement to z, and its blocks
    are D_n(theta) diag(e^{i m phi}) with D_n real, the tables the device reads."""
    P = 5
    theta, tidx, phi = rot.direction_angles()
    D, Z = rot.packed_dmatrices(P), rot.pack_phases(P)
    d = rot.displacements()
    far = np.abs(d).max(1) > 1
    assert (tidx[far] >= 0).all() and (tidx[~far] == -1).all() and len(theta) < 61
    for e in np.nonzero(far)[0]:
        R = rot._rot_y(-theta[tidx[e]]) @ rot._rot_z(-phi[e])
        assert np.allclose(R @ d[e] / np.linalg.norm(d[e]), [0, 0, 1], atol=1e-14)
        full, sr = rot.rotation_blocks(P, R), rot.slot_rotation(e, P)
        off = 0
        for n in range(P + 1):
            w = 2 * n + 1
            Dn = D[tidx[e], off:off + w * w].reshape(w, w)
            off += w * w
            assert np.abs(Dn * Z[e, P - n:P + n + 1][None, :] - full[n]).max() < 1e-13
            assert np.abs(sr[n] - full[n]).max() < 1e-13


def _apply(P, Q, E, pref, T, C, x):
    M = Q @ x
    Mb = np.concatenate([T[n] @ M[n * n:(n + 1) ** 2] for n in range(P + 1)])
    Lb = np.zeros_like(Mb)
    for m in range(-P, P + 1):
        ns = list(range(abs(m), P + 1))
        rows = [n * n + n + m for n in ns]
        Lb[rows] = C[m + P][np.ix_(ns, ns)] @ Mb[rows]
    La = np.concatenate([T[n].conj().T @ Lb[n * n:(n + 1) ** 2] for n in range(P + 1)])
    return (pref * (E @ La)).real


@pytest.mark.parametrize("imag", [False, True])
def test_rotation_m2l_matches_the_dense_kifmm_operator(imag):
    """p = 6 surfaces, level 4, k = 10, P = 20: sin to rounding; cos converges with
    the separation (4.3e-5 at the nearest face displacement, where the two boxes'
    surface corners come closest, below 1e-8 beyond)."""
    p, lev, ext, k, P = 6, 4, 1.0, 10.0, 20
    s = O.level_scale(ext, lev)
    eq = O.surface_pts(p, O.R_EQUIV) * s
    Q, E, pref = rot.level_operators(p, lev, ext, k, imag, P)
    x = np.random.default_rng(1).normal(size=eq.shape[0])
    for d, bar in (((3, 1, 0), 1e-8), ((2, 2, 2), 1e-8), ((2, 0, 0), 1e-4)):
        dv = 2 * s * np.array(d, float)
        T = rot.slot_rotation((d[0] + 3) * 49 + (d[1] + 3) * 7 + d[2] + 3, P)   # D_n diag(phase)
        C = rot.coaxial(P, k, np.linalg.norm(dv), imag)
        y = _apply(P, Q, E, pref, T, C, x)
        ref = O.family_matrix(k, imag)(eq + dv, eq) @ x
        err = np.linalg.norm(y - ref) / np.linalg.norm(ref)
        assert err < (1e-12 if imag else bar), (d, err)


def test_enable_refuses_before_touching_the_plan():
    """No plan handle is needed: every refusal comes before the first library call."""
    from types import SimpleNamespace
    st = SimpleNamespace(kind="helmholtz", k=10.0, p=4, info={"domain_extent": 1.0},
                         n_families=2, max_depth=5, handle=None)
    for bad in (dict(kind="yukawa"), dict(k=0.0)):
        with pytest.raises(ValueError):
            rot.enable(SimpleNamespace(**{**vars(st), **bad}), 10)
    for order in (0, 41):
        with pytest.raises(ValueError):
            rot.enable(st, order)
    with pytest.raises(ValueError, match="overflows"):   # y_80(k 4 s) at k = 0.05
        rot.enable(SimpleNamespace(**{**vars(st), "k": 0.05}), 40)
    assert not hasattr(st, "rotation_order")


def test_disable_goes_through_the_library_signature():
    """disable() reaches the C entry point with its full argument list; a NULL plan is
    refused there before anything touches a device."""
    from types import SimpleNamespace
    with pytest.raises(ValueError, match="plan is NULL"):   # HFMM_ERR_ARG
        rot.disable(SimpleNamespace(handle=None))
