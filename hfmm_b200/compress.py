"""Low-rank compression of a level's M2L operators for the mixed-precision path.

The reference applies each of the 316 non-adjacent M2L matrices K_d of a level
densely (n_s x n_s per V pair, jaxfmm/kifmm/phases.py:176-237). Those matrices
share their dominant left and right subspaces: with the Gram matrix
S = sum_d K_d K_d^T (equal to sum_d K_d^T K_d, because K_{-d} = K_d^T on the
symmetric equivalent surface), its leading r eigenvectors U give
K_d ~ U C_d U^T with C_d = U^T K_d U (r x r). r is the smallest rank whose
discarded eigenvalues stay below (eps * lambda_max): the projection error of
every K_d is then about eps relative to the largest singular value.

The M2L of a level becomes: compress the source densities (x' = U^T x), apply
the r x r matrices per V pair on the tensor cores, expand (y = U y'). For the
sin(kr)/r component the ranks are small (the kernel is smooth): at p = 8,
k x box = 0.16, r = 19 of 296 at eps = 1e-8. The plain FP64 path never uses
this; the mixed path does when a plan is built with a compression tolerance,
and its results stay certified against the direct sum like every mixed result.
"""
import numpy as np
import torch

from .operators import surface_pts, level_scale, R_EQUIV


def nonadjacent_displacements():
    """The 316 displacements (dx, dy, dz) in [-3, 3]^3 with max |d| >= 2, in
    (dx+3)*49 + (dy+3)*7 + (dz+3) order (the order of the M2L tables)."""
    out = []
    for i in range(343):
        d = (i // 49 - 3, (i // 7) % 7 - 3, i % 7 - 3)
        if max(abs(c) for c in d) > 1:
            out.append(d)
    return np.array(out, dtype=np.float64)


def level_m2l_matrices(p, level, extent, k, imaginary, device, chunk=64, kind="helmholtz"):
    """K_d = G((equiv + 2 d) s, equiv s), (316, n_s, n_s) float64 on ``device``; G a
    Helmholtz component, or exp(-k r) / (4 pi r) for kind "yukawa"."""
    eq = torch.as_tensor(surface_pts(p, R_EQUIV), dtype=torch.float64, device=device)
    s = level_scale(extent, level)
    disp = torch.as_tensor(2.0 * nonadjacent_displacements(), dtype=torch.float64, device=device)
    y = eq * s
    out = torch.empty((disp.shape[0], eq.shape[0], eq.shape[0]), dtype=torch.float64,
                      device=device)
    for c0 in range(0, disp.shape[0], chunk):
        x = (eq[None, :, :] + disp[c0:c0 + chunk, None, :]) * s
        r = torch.linalg.norm(x[:, :, None, :] - y[None, None, :, :], dim=-1)
        if kind == "yukawa":
            out[c0:c0 + chunk] = torch.exp(-float(k) * r) / (4.0 * np.pi * r)
        else:
            trig = torch.sin if imaginary else torch.cos
            out[c0:c0 + chunk] = trig(float(k) * r) / r
    return out


def compress_level(K, eps):
    """(U (n_s, r), C (316, r, r)) with K_d ~ U C_d U^T, rank chosen by ``eps``."""
    S = torch.einsum("dmk,dnk->mn", K, K)
    S = 0.5 * (S + S.T)
    w, V = torch.linalg.eigh(S)                  # ascending
    w = torch.clamp(w, min=0.0)
    r = int((w > (eps * eps) * w[-1]).sum().item())
    r = max(r, 1)
    U = V[:, -r:].flip(1).contiguous()           # leading eigenvectors first
    C = torch.matmul(torch.matmul(U.T.unsqueeze(0), K), U.unsqueeze(0)).contiguous()
    return U, C


def level_compressed(p, level, extent, k, imaginary, eps, device, kind="helmholtz"):
    K = level_m2l_matrices(p, level, extent, k, imaginary, device, kind=kind)
    U, C = compress_level(K, eps)
    del K
    return U, C
