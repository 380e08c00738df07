"""Seeded point clouds shared by the tests (synthetic, following the reference's
test.py conventions: ``default_rng(seed + n)``, uniform in [0,1]^3, real N(0,1)
charges, and the ``--clustered`` variant of test.py:40-43)."""
import numpy as np


def uniform(n, seed=42):
    rng = np.random.default_rng(seed + n)
    pos = rng.uniform(0.0, 1.0, (n, 3))
    q = rng.normal(size=n)
    return pos, q


def clustered(n, seed=42):
    """test.py:40-43: the first half squeezed into [0.1, 0.25]^3."""
    rng = np.random.default_rng(seed + n)
    pos = rng.uniform(0.0, 1.0, (n, 3))
    pos[: n // 2] = rng.uniform(0.1, 0.25, (n // 2, 3))
    q = rng.normal(size=n)
    return pos, q


def sphere_clusters(n, seed=7):
    """Half on the sphere of radius 0.5 about (0.5,0.5,0.5), half in 8 Gaussian
    clusters with sigma 0.03 (the adaptive-tree workload shape)."""
    rng = np.random.default_rng(seed + n)
    h = n // 2
    d = rng.normal(size=(h, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    sph = 0.5 + 0.5 * d
    cen = rng.uniform(0.1, 0.9, (8, 3))
    lab = rng.integers(0, 8, n - h)
    cl = cen[lab] + 0.03 * rng.normal(size=(n - h, 3))
    pos = np.concatenate([sph, cl])
    q = rng.normal(size=n) + 1j * rng.normal(size=n)
    return pos, q


def complex_uniform(n, seed=42):
    rng = np.random.default_rng(seed + n)
    pos = rng.uniform(0.0, 1.0, (n, 3))
    q = rng.normal(size=n) + 1j * rng.normal(size=n)
    return pos, q


def with_duplicates(n, seed=3):
    """Uniform points where every 10th point repeats its predecessor exactly."""
    pos, q = uniform(n, seed)
    pos[10::10] = pos[9::10][: len(pos[10::10])]
    return pos, q


def plane(n, seed=5):
    """Quasi-2D cloud (z = 0.5): a thin film that makes the depth refinement work."""
    rng = np.random.default_rng(seed + n)
    pos = rng.uniform(0.0, 1.0, (n, 3))
    pos[:, 2] = 0.5 + 1e-3 * pos[:, 2]
    return pos, rng.normal(size=n)


def sphere_and_clusters(n, seed=11):
    """The C3 workload's shape: half uniform on the sphere of radius 0.5 about
    (0.5, 0.5, 0.5), half in 8 Gaussian clusters (sigma 0.03, centres U[0.1, 0.9]^3);
    complex N(0,1) charges. Deep and adaptive: at n = 8000 with leaf 16 the tree
    build must double its box buffer (6096 -> 12192)."""
    rng = np.random.default_rng(seed + n)
    ns = n // 2
    d = rng.normal(size=(ns, 3))
    sph = 0.5 + 0.5 * d / np.linalg.norm(d, axis=1, keepdims=True)
    c = rng.uniform(0.1, 0.9, (8, 3))
    cl = c[rng.integers(0, 8, n - ns)] + 0.03 * rng.normal(size=(n - ns, 3))
    pos = np.concatenate([sph, cl])
    q = rng.normal(size=n) + 1j * rng.normal(size=n)
    return pos, q

