"""The C-ABI boundary without a GPU: the in-tree library loads, exports every
function include/hfmm_b200.h declares, and the Python front door validates its
arguments exactly as HFMM.py:14-16 and 57-64 / 86-87 do (before touching a device)."""
import ctypes
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "hfmm_b200.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(hfmm_[a-z_0-9]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    from hfmm_b200 import _lib
    names = declared_functions()
    assert len(names) >= 14
    lib = ctypes.CDLL(_lib.LIB_PATH)
    for n in names:
        assert hasattr(lib, n), n
    bound = {s[0] for s in _lib.SIGNATURES}
    assert set(names) <= bound, set(names) - bound


def test_diagnostics_without_gpu():
    from hfmm_b200 import _lib
    assert isinstance(_lib.lib.hfmm_launch_count(), int)
    assert isinstance(_lib.lib.hfmm_last_error(), bytes)


def test_null_arguments_rejected():
    from hfmm_b200 import _lib
    h = ctypes.c_void_p()
    assert _lib.lib.hfmm_tree_build(None, 10, 16, 0, ctypes.byref(h)) == -1
    assert _lib.lib.hfmm_evaluate(None, None, None, None, None, 0, None) == -1
    assert b"NULL" in _lib.lib.hfmm_last_error() or _lib.lib.hfmm_last_error()


@pytest.mark.parametrize("bad", [
    dict(positions=np.zeros((0, 3))), dict(positions=np.zeros((4, 2))),
    dict(positions=np.array([[0.0, 0.0, np.inf]])), dict(p=1), dict(p=3.5),
    dict(N_max=0), dict(N_max=2.5), dict(max_depth=0), dict(max_depth=1.5),
    dict(k=np.nan), dict(k=np.inf)])
def test_setup_validation_matches_reference(bad):
    import hfmm_b200
    args = dict(positions=np.random.default_rng(0).uniform(size=(32, 3)), k=1.0, p=3,
                N_max=16, max_depth=None)
    args.update(bad)
    with pytest.raises(ValueError):
        hfmm_b200.setup(**args)


def test_evaluate_rejects_complex_and_wrong_shape():
    import hfmm_b200

    class Dummy:
        n = 10
        device = None
    with pytest.raises(ValueError):
        hfmm_b200.evaluate(Dummy(), np.ones(10) + 1j)
    with pytest.raises(ValueError):
        hfmm_b200.evaluate(Dummy(), np.ones(9))
    with pytest.raises(ValueError):
        hfmm_b200.evaluate_field(Dummy(), np.ones((10, 2)))


def test_no_gpu_means_loud_failure():
    import torch
    import hfmm_b200
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(RuntimeError, match="CUDA"):
        hfmm_b200.setup(np.random.default_rng(0).uniform(size=(32, 3)), 1.0, p=3)
