"""Rotation-based M2L of the FP64 path: rotate, shift along z, rotate back.

The reference's Helmholtz path translates with KIFMM operators only (kifmm/phases.py:
176-237); its rotation-based M2L is Laplace's (kernels/laplace/transf.py:143-250,
rotations kernels/laplace/rotation.py). This module builds the Helmholtz version of
that scheme for the two kernel families, as an alternative to the dense M2L tables
of the FP64 evaluate (``hfmm_plan_set_m2l_rotation``):

* a box's equivalent density x (n_s points on its equivalent surface, radius
  R_EQUIV x half side) becomes multipole coefficients about the box centre,
  M_nm = sum_s x_s j_n(k |y_s|) conj(Y_nm(y_s)), n <= P (orthonormal complex Y);
* per V pair with displacement d: rotate the coefficients into the frame where d is
  the z axis (T_n, per degree), shift coaxially by |d| (one matrix per order m), rotate
  back (T_n^H), accumulated over the target's V list;
* the target's check potential is Re(pref sum L_nm j_n(k |c|) Y_nm(c)) at its check
  points (the same unit point set, scaled), pref = -4 pi k for cos(kr)/r = -k y_0(kr)
  and 4 pi k for sin(kr)/r = k j_0(kr).

Coaxial coefficients (shift t along +z, multipole (n, m) -> local (n', m)), from the
addition theorem with Gaunt integrals:
    C^m_{n'n}(t) = 4 pi sum_nu i^(n'+nu-n) G(n' m; nu 0; n m) z_nu(k t) sqrt((2 nu+1)/(4 pi)),
G = int Y_{n'm} Y_{nu 0} conj(Y_{nm}), z = y for the cos family (singular), j for
the sin family (regular everywhere); i^(n'+nu-n) is real wherever G is nonzero.
The formula is pinned against numerical projection in tests/test_rotation_cpu.py.
Rotation blocks T_n[m, m''] = int Y_{nm''}(s) conj(Y_nm(R s)) d Omega are integrated
exactly (Gauss-Legendre x uniform azimuth, enough points for degree 2P).

Each slot's rotation is R_y(-theta) R_z(-phi) (theta, phi the displacement's polar
angle and azimuth), whose blocks factor as T_n = D_n(theta) diag(e^{i m phi}) with D_n
real; the shift along z commutes with rotations about z, so this gives the same
operator as any other rotation taking d to z. The 316 slots share the D tables of
their distinct polar angles.

Cost per V pair, family and charge column: two real rotations of sum (2n+1)^2 and one
coaxial shift of sum (P+1-|m|)^2 real x complex multiply-adds plus the phases, O(P^3):
at P = 20 about 30,900 (61,700 FMA), against n_s^2 = 87,616 multiply-adds of the dense
p = 8 table. Accuracy is
set by P: at p = 8 the nearest face displacement (2, 0, 0) converges slowest
(relative 2.9e-6 at P = 20, 1.1e-6 at 24, 3.8e-7 at 28); the sin family is exact to
rounding at any P used here.
"""
import math
from fractions import Fraction
from functools import lru_cache

import numpy as np
from numpy.polynomial.legendre import leggauss
from scipy.special import spherical_jn, spherical_yn

from .operators import surface_pts, level_scale, R_EQUIV

__all__ = ["gaunt", "rotation_blocks", "coaxial", "level_operators", "direction_angles",
           "slot_rotation", "packed_dmatrices", "pack_phases", "n_coeff", "pack_coaxial",
           "enable", "disable"]


def n_coeff(P):
    return (P + 1) * (P + 1)


def _sph(v):
    r = np.linalg.norm(v, axis=-1)
    th = np.arccos(np.clip(v[..., 2] / np.where(r > 0, r, 1.0), -1.0, 1.0))
    return r, th, np.arctan2(v[..., 1], v[..., 0])


@lru_cache(maxsize=None)
def _fact(n):
    return math.factorial(n)


@lru_cache(maxsize=None)
def wigner_3j(j1, j2, j3, m1, m2, m3):
    """The Wigner 3j symbol by the Racah formula in exact integer arithmetic: the
    alternating sum over k of 1 / prod(a_i!) is formed over the common denominator
    prod(max_k a_i)! (each a_i is linear in k), and the square of the result is
    rounded to a double once."""
    if m1 + m2 + m3 != 0 or j3 < abs(j1 - j2) or j3 > j1 + j2:
        return 0.0
    if abs(m1) > j1 or abs(m2) > j2 or abs(m3) > j3:
        return 0.0
    f = _fact
    pre_num = (f(j1 + j2 - j3) * f(j1 - j2 + j3) * f(-j1 + j2 + j3)
               * f(j1 + m1) * f(j1 - m1) * f(j2 + m2) * f(j2 - m2) * f(j3 + m3) * f(j3 - m3))
    pre_den = f(j1 + j2 + j3 + 1)
    terms = []
    for k in range(0, j1 + j2 + j3 + 1):
        a = (k, j3 - j2 + k + m1, j3 - j1 + k - m2, j1 + j2 - j3 - k, j1 - k - m1, j2 - k + m2)
        if min(a) >= 0:
            terms.append((k, a))
    den = 1
    for i in range(6):
        den *= f(max(a[i] for _, a in terms))
    num = 0
    for k, a in terms:
        d = f(a[0]) * f(a[1]) * f(a[2]) * f(a[3]) * f(a[4]) * f(a[5])
        num += (den // d) if k % 2 == 0 else -(den // d)
    sign = -1.0 if (j1 - j2 - m3) % 2 else 1.0
    # sqrt(pre) * s: the square pre s^2 = pre_num num^2 / (pre_den den^2) is exact and
    # Python's integer division rounds it correctly; the sign is num's
    val = math.sqrt((pre_num * num * num) / (pre_den * den * den))
    return sign * (val if num >= 0 else -val)


def gaunt(l1, m1, l2, m2, l3, m3):
    """int Y_{l1 m1} Y_{l2 m2} Y_{l3 m3} dOmega (orthonormal complex harmonics)."""
    if (l1 + l2 + l3) % 2:
        return 0.0
    return (math.sqrt((2 * l1 + 1) * (2 * l2 + 1) * (2 * l3 + 1) / (4 * math.pi))
            * wigner_3j(l1, l2, l3, 0, 0, 0) * wigner_3j(l1, l2, l3, m1, m2, m3))


@lru_cache(maxsize=None)
def _coax_table(P):
    """W[m + P, n', n, nu] = 4 pi i^(n'+nu-n) G(n' m; nu 0; n m) sqrt((2 nu+1)/(4 pi)) (real)."""
    W = np.zeros((2 * P + 1, P + 1, P + 1, 2 * P + 1))
    for m in range(0, P + 1):   # the coefficients of -m equal those of m (n' + nu + n even)
        for n2 in range(abs(m), P + 1):
            for n in range(abs(m), P + 1):
                for nu in range(abs(n - n2), n + n2 + 1, 2):
                    g = gaunt(n2, m, nu, 0, n, -m) * (-1) ** (m % 2)
                    if g == 0.0:
                        continue
                    e = (n2 + nu - n) % 4   # i^e: 0 -> 1, 2 -> -1 (odd e has g = 0)
                    W[m + P, n2, n, nu] = (1.0 if e == 0 else -1.0) * 4 * math.pi * g * \
                        math.sqrt((2 * nu + 1) / (4 * math.pi))
    W[:P] = W[:P:-1]
    return W


def coaxial(P, k, t, regular):
    """C[m + P] ((P+1) x (P+1), real): local (n', m) from multipole (n, m) for a shift t
    along +z; rows and columns below |m| are zero."""
    z = spherical_jn if regular else spherical_yn
    zs = np.array([z(nu, k * t) for nu in range(2 * P + 1)])
    return np.einsum("mabn,n->mab", _coax_table(P), zs)


def _harmonics(P, th, ph):
    """Y_nm (orthonormal, Condon-Shortley phase) at the given angles for every n <= P,
    m = -n..n, rows in (n, m) order. Column recurrence of the normalised associated
    Legendre functions, P~_mm = -sqrt((2m+1)/(2m)) sin(th) P~_(m-1)(m-1),
    P~_(m+1)m = sqrt(2m+3) cos(th) P~_mm, then
    P~_nm = a (cos(th) P~_(n-1)m - b P~_(n-2)m), a = sqrt((4n^2-1)/(n^2-m^2)),
    b = sqrt(((n-1)^2-m^2)/(4(n-1)^2-1)); Y_n(-m) = (-1)^m conj(Y_nm)."""
    th, ph = np.ravel(th), np.ravel(ph)
    x, s = np.cos(th), np.sin(th)
    out = np.empty(((P + 1) ** 2, th.size), np.complex128)
    pmm = np.full(th.size, math.sqrt(1.0 / (4 * math.pi)))
    for m in range(P + 1):
        if m > 0:
            pmm = -math.sqrt((2 * m + 1) / (2 * m)) * s * pmm
        e = np.exp(1j * m * ph)
        sign = -1.0 if m % 2 else 1.0
        p2, p1 = None, pmm
        for n in range(m, P + 1):
            if n == m + 1:
                p2, p1 = p1, math.sqrt(2 * m + 3) * x * p1
            elif n > m + 1:
                a = math.sqrt((4 * n * n - 1) / (n * n - m * m))
                b = math.sqrt(((n - 1) ** 2 - m * m) / (4 * (n - 1) ** 2 - 1))
                p2, p1 = p1, a * (x * p1 - b * p2)
            y = p1 * e
            out[n * n + n + m] = y
            if m:
                out[n * n + n - m] = sign * np.conj(y)
    return out


@lru_cache(maxsize=None)
def _rotation_quadrature(P):
    """Gauss-Legendre x uniform azimuth nodes exact for degree 2P, their weights and
    the harmonics there."""
    nq = P + 2
    x, w = leggauss(nq)
    th = np.arccos(x)
    ph = np.linspace(0, 2 * np.pi, 2 * nq + 1, endpoint=False)
    TH, PH = np.meshgrid(th, ph, indexing="ij")
    W = np.outer(w, np.full(len(ph), 2 * np.pi / len(ph))).ravel()
    S = np.stack([np.sin(TH) * np.cos(PH), np.sin(TH) * np.sin(PH), np.cos(TH)], -1).reshape(-1, 3)
    _, t1, p1 = _sph(S)
    return S, W, _harmonics(P, t1, p1)


def rotation_blocks(P, R):
    """T_n ((2n+1) x (2n+1) complex) for n <= P: coefficients in the frame R maps to."""
    S, W, A = _rotation_quadrature(P)
    _, t2, p2 = _sph(S @ R.T)
    B = _harmonics(P, t2, p2)
    return [(np.conj(B[n * n:(n + 1) ** 2]) * W) @ A[n * n:(n + 1) ** 2].T for n in range(P + 1)]


def rotation_to_z(d):
    """A proper rotation R with R d / |d| = z."""
    u = np.asarray(d, float) / np.linalg.norm(d)
    z = np.array([0.0, 0.0, 1.0])
    v = np.cross(u, z)
    c, s = float(u @ z), float(np.linalg.norm(v))
    if s < 1e-14:
        return np.eye(3) if c > 0 else np.diag([1.0, -1.0, -1.0])
    vx = np.array([[0, -v[2], v[1]], [v[2], 0, -v[0]], [-v[1], v[0], 0]])
    return np.eye(3) + vx + vx @ vx * ((1 - c) / s ** 2)


def displacements():
    """The 343 displacement slots (dx, dy, dz) in [-3, 3]^3, (dx+3)*49 + (dy+3)*7 + (dz+3)."""
    return np.array([(i // 49 - 3, (i // 7) % 7 - 3, i % 7 - 3) for i in range(343)], float)


def _rot_y(b):
    c, s = math.cos(b), math.sin(b)
    return np.array([[c, 0.0, s], [0.0, 1.0, 0.0], [-s, 0.0, c]])


def _rot_z(a):
    c, s = math.cos(a), math.sin(a)
    return np.array([[c, -s, 0.0], [s, c, 0.0], [0.0, 0.0, 1.0]])


def direction_angles():
    """The rotation of each non-adjacent slot's displacement d = target - source onto z
    as R_y(-theta) R_z(-phi) (polar angle theta, azimuth phi of d). Its blocks factor as
    T_n = D_n(theta) diag(e^{i m phi}) with D_n real (a y-rotation), so the slots share
    the D tables of their distinct polar angles. Returns (theta of each distinct polar
    angle, each slot's theta index (-1: adjacent), each slot's phi)."""
    d = displacements()
    keys, theta = {}, []
    tidx, phi = np.full(343, -1, np.int32), np.zeros(343)
    for e in range(343):
        dx, dy, dz = (int(v) for v in d[e])
        if max(abs(dx), abs(dy), abs(dz)) <= 1:
            continue
        d2 = dx * dx + dy * dy + dz * dz
        key = ((dz > 0) - (dz < 0), Fraction(dz * dz, d2))   # cos(theta) = dz / |d|
        if key not in keys:
            keys[key] = len(theta)
            theta.append(math.acos(dz / math.sqrt(d2)))
        tidx[e] = keys[key]
        phi[e] = math.atan2(dy, dx)
    return np.array(theta), tidx, phi


def slot_rotation(e, P):
    """The blocks T_n of slot e from its factors (what the device applies)."""
    theta, tidx, phi = direction_angles()
    D = rotation_blocks(P, _rot_y(-theta[tidx[e]]))
    return [D[n].real * np.exp(1j * np.arange(-n, n + 1) * phi[e])[None, :] for n in range(P + 1)]


@lru_cache(maxsize=4)
def packed_dmatrices(P):
    """[n_theta][sum (2n+1)^2] real: D_n(theta) of every distinct polar angle, each block
    row-major [m][m'']."""
    theta, _, _ = direction_angles()
    return np.ascontiguousarray(np.stack([np.concatenate([t.real.ravel() for t in
                                                          rotation_blocks(P, _rot_y(-th))])
                                          for th in theta]))


def pack_phases(P):
    """[343][2P+1] complex: e^{i m phi} of each slot, m = -P..P (zeros for adjacent slots)."""
    _, tidx, phi = direction_angles()
    out = np.exp(1j * np.outer(phi, np.arange(-P, P + 1)))
    out[tidx < 0] = 0.0
    return np.ascontiguousarray(out)


def distances():
    """Distinct |d|^2 of the non-adjacent slots (sorted) and each slot's index (-1: adjacent)."""
    d = displacements()
    d2 = (d * d).sum(1).astype(int)
    far = np.abs(d).max(1) > 1
    uniq = np.unique(d2[far])
    slot = np.where(far, np.searchsorted(uniq, d2), -1).astype(np.int32)
    return uniq, slot


def pack_coaxial(P, k, s, regular):
    """[n_dist][2P+1][P+1][P+1] real: the coaxial matrices of a level (half side s; a slot's
    shift is 2 s |d|)."""
    uniq, _ = distances()
    return np.stack([coaxial(P, k, 2 * s * math.sqrt(d2), regular) for d2 in uniq])


def level_operators(p, level, extent, k, imaginary, P):
    """(Q, E, pref) of one level and family: Q ((P+1)^2 x n_s complex) makes multipole
    coefficients from an equivalent density, E (n_s x (P+1)^2 complex) check potentials
    (times pref, real part) from local coefficients."""
    s = level_scale(extent, level)
    eq = surface_pts(p, R_EQUIV) * s
    r, th, ph = _sph(eq)
    Ys = _harmonics(P, th, ph)
    deg = np.array([n for n in range(P + 1) for _ in range(-n, n + 1)])
    Jn = spherical_jn(deg[:, None], k * r[None, :])
    Q = np.conj(Ys) * Jn
    E = (Ys * Jn).T
    pref = 4 * math.pi * k * (1.0 if imaginary else -1.0)
    return Q, E, pref


def enable(state, order):
    """Switch a plan's FP64 evaluate to the rotation-based M2L of ``order`` P (the
    Helmholtz kernel, k > 0; the dense tables stay in the plan for the other paths).
    Builds every level's operators on the host first (rotation blocks and the Gaunt
    table once per order: about 4 s at P = 20, 25 s at P = 32) and uploads them only
    when all are finite: at small k x box size with a high order the Neumann
    functions y_nu(k t), nu <= 2P, overflow, and that raises ValueError with the plan
    unchanged."""
    from . import _lib
    from ._lib import check
    if getattr(state, "kind", "helmholtz") != "helmholtz":
        raise ValueError("the rotation-based M2L is built for the Helmholtz kernel")
    P = int(order)
    if not 1 <= P <= 40:
        raise ValueError("rotation order must be in [1, 40]")
    if not float(state.k) > 0.0:
        raise ValueError("the rotation-based M2L needs k > 0 (its expansions are spherical "
                         "Bessel and Neumann functions of k r)")
    extent = state.info["domain_extent"]
    for level in range(2, state.max_depth + 1):
        # the largest Neumann value the shifts take: y_2P at the nearest V distance, 4 s
        x = state.k * 4 * level_scale(extent, level)
        if not np.isfinite(spherical_yn(2 * P, x)):
            raise ValueError(f"rotation order {P} overflows at level {level} (y_{2 * P}"
                             f"({x:.3g}) is not finite): use a lower order or the dense tables")
    levels = []
    for fam in range(state.n_families):
        for level in range(2, state.max_depth + 1):
            Q, E, pref = level_operators(state.p, level, extent, state.k, fam == 1, P)
            C = np.ascontiguousarray(pack_coaxial(P, state.k, level_scale(extent, level), fam == 1))
            Q = np.ascontiguousarray(Q.astype(np.complex128))
            E = np.ascontiguousarray(E.astype(np.complex128))
            if not (np.isfinite(C).all() and np.isfinite(Q).all() and np.isfinite(E).all()):
                raise ValueError(f"rotation order {P} overflows at level {level} (k x box side "
                                 f"{state.k * 2 * level_scale(extent, level):.3g}): use a lower "
                                 f"order or the dense tables")
            levels.append((fam, level, Q, E, C, pref))
    D = packed_dmatrices(P)
    _, tidx, _ = direction_angles()
    tidx = np.ascontiguousarray(tidx, np.int32)
    Z = pack_phases(P)
    uniq, slot = distances()
    slot = np.ascontiguousarray(slot, np.int32)
    check(_lib.lib.hfmm_plan_set_m2l_rotation(state.handle, P, D.ctypes.data, D.shape[0],
                                               tidx.ctypes.data, Z.ctypes.data, slot.ctypes.data,
                                               len(uniq)))
    for fam, level, Q, E, C, pref in levels:
        check(_lib.lib.hfmm_plan_set_rotation_level(state.handle, fam, level, Q.ctypes.data,
                                                     E.ctypes.data, C.ctypes.data, float(pref)))
    state.rotation_order = P


def disable(state):
    """Back to the dense M2L tables."""
    from . import _lib
    from ._lib import check
    check(_lib.lib.hfmm_plan_set_m2l_rotation(state.handle, 0, None, 0, None, None, None, 0))
    state.rotation_order = 0
