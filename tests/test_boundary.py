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
    assert _lib.lib.hfmm_export_densities(None, 0, 1, None, 0) == -1
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


def _fake_plan(n=4):
    """Enough of a plan for the host-side checks, which run before any launch."""
    import types
    import torch
    return types.SimpleNamespace(n=n, device=torch.device("cuda", 0), handle=None)


@pytest.mark.parametrize("which,bad,msg", [
    ("q_re", "float32", "float64"), ("q_re", "short", "shape"), ("q_im", "short", "shape"),
    ("phi_out", "float64", "complex128"), ("field_out", "flat", "shape"),
    ("phi_out", "strided", "contiguous"), ("q_re", "host", "device")])
def test_evaluate_into_refuses_buffers_that_do_not_fit_the_plan(which, bad, msg):
    """The kernels take raw pointers and trust the plan's sizes: a buffer of the
    wrong type, size, layout or device is refused before any pointer is passed."""
    import torch
    import hfmm_b200
    n = 4
    bufs = dict(q_re=torch.zeros(n, dtype=torch.float64), q_im=torch.zeros(n, dtype=torch.float64),
                phi_out=torch.zeros(n, dtype=torch.complex128),
                field_out=torch.zeros((n, 3), dtype=torch.complex128))
    if bad == "float32":
        bufs[which] = torch.zeros(n, dtype=torch.float32)
    elif bad == "short":
        bufs[which] = torch.zeros(n - 1, dtype=torch.float64)
    elif bad == "float64":
        bufs[which] = torch.zeros(n, dtype=torch.float64)
    elif bad == "flat":
        bufs[which] = torch.zeros(3 * n, dtype=torch.complex128)
    elif bad == "strided":
        bufs[which] = torch.zeros(2 * n, dtype=torch.complex128)[::2]
    with pytest.raises(ValueError, match=msg):
        hfmm_b200.evaluate_into(_fake_plan(n), bufs["q_re"], bufs["q_im"], bufs["phi_out"],
                                bufs["field_out"])


@pytest.mark.parametrize("targets", [[0, 4], [-1], [[0, 1]], [0.5]])
def test_direct_refuses_targets_outside_the_points(targets):
    import hfmm_b200
    with pytest.raises(ValueError, match="targets"):
        hfmm_b200.direct(_fake_plan(4), np.zeros(4), np.asarray(targets))


def test_direct_refuses_charges_of_another_size():
    import hfmm_b200
    with pytest.raises(ValueError, match="charges"):
        hfmm_b200.direct(_fake_plan(4), np.zeros(5), np.array([0, 1]))


def _golden_module():
    import importlib.util
    path = os.path.join(ROOT, "tests", "golden", "make_golden.py")
    spec = importlib.util.spec_from_file_location("make_golden", path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def test_invalid_inputs_raise_what_the_reference_raises():
    """Each invalid input of tests/golden/make_golden.py's error cases raises, from
    setup / evaluate here, the exception the reference's own HFMM.setup /
    HFMM.evaluate raised for it (tests/golden/errors/reference_errors.json,
    recorded by running the reference's code), before any device is touched."""
    import json
    import hfmm_b200
    with open(os.path.join(ROOT, "tests", "golden", "errors", "reference_errors.json")) as f:
        ref = json.load(f)
    good, cases = _golden_module()._error_cases()
    assert set(cases) | {"charges_complex", "charges_short", "charges_two_columns"} == set(ref)
    for name, kw in cases.items():
        args = dict(positions=good, k=1.0, p=3, N_max=16, max_depth=None)
        args.update(kw)
        with pytest.raises(Exception) as e:
            hfmm_b200.setup(**args)
        assert type(e.value).__name__ == ref[name], name

    class Plan:                     # the charge checks run before any device work
        n = 64
        device = None
    for name, q in (("charges_complex", np.ones(64) + 1j), ("charges_short", np.ones(63)),
                    ("charges_two_columns", np.ones((64, 2)))):
        with pytest.raises(Exception) as e:
            hfmm_b200.evaluate(Plan(), q)
        assert type(e.value).__name__ == ref[name], name
