"""Host math of the low-rank M2L (hfmm_b200/compress.py) on the CPU: its M2L
matrices are the reference's tables (operators.py:363-403, as the oracle restates
them), and the compression K_d ~ U C_d U^T keeps its stated error."""
import numpy as np
import pytest
import torch

import oracle as O
from hfmm_b200 import compress
from hfmm_b200.operators import level_scale

P, EXTENT, LEVEL = 4, 1.0, 3


def test_displacements_are_the_nonadjacent_table_entries_in_order():
    d = compress.nonadjacent_displacements()
    assert d.shape == (316, 3)
    assert (np.abs(d).max(axis=1) >= 2).all()
    idx = (d[:, 0] + 3) * 49 + (d[:, 1] + 3) * 7 + (d[:, 2] + 3)
    assert (np.diff(idx) > 0).all()


@pytest.mark.parametrize("imaginary", [False, True])
def test_m2l_matrices_equal_the_reference_tables(imaginary):
    k = 10.0
    K = compress.level_m2l_matrices(P, LEVEL, EXTENT, k, imaginary, "cpu").numpy()
    s = level_scale(EXTENT, LEVEL)
    assert s == EXTENT * 0.5 ** (LEVEL + 1)
    G = O.helmholtz_G_np(k, imaginary)
    ref = O.build_operators(P, lambda x, y: G(x * s, y * s))["M2L_K_table"]
    d = compress.nonadjacent_displacements()
    idx = ((d[:, 0] + 3) * 49 + (d[:, 1] + 3) * 7 + (d[:, 2] + 3)).astype(int)
    assert np.abs(K - ref[idx]).max() <= 1e-13 * np.abs(ref).max()


@pytest.mark.parametrize("imaginary", [False, True])
def test_compression_error_follows_eps(imaginary):
    K = compress.level_m2l_matrices(P, LEVEL, EXTENT, 10.0, imaginary, "cpu")
    kmax = max(float(torch.linalg.matrix_norm(K[i], ord=2)) for i in range(K.shape[0]))
    ranks = []
    for eps in (1e-4, 1e-7, 1e-10):
        U, C = compress.compress_level(K, eps)
        r = U.shape[1]
        ranks.append(r)
        assert torch.allclose(U.T @ U, torch.eye(r, dtype=torch.float64), atol=1e-12)
        err = max(float(torch.linalg.matrix_norm(K[i] - U @ C[i] @ U.T, ord=2))
                  for i in range(K.shape[0]))
        assert err <= 10 * eps * kmax, (eps, r, err / kmax)
    assert ranks[0] <= ranks[1] <= ranks[2] <= K.shape[1]


def test_sin_component_compresses_harder():
    r = {}
    for imaginary in (False, True):
        K = compress.level_m2l_matrices(P, LEVEL, EXTENT, 10.0, imaginary, "cpu")
        r[imaginary] = compress.compress_level(K, 1e-7)[0].shape[1]
    assert r[True] < r[False]
