"""The leaf-size autotuner's host logic (hfmm_b200/tune.py) on the CPU: the
selection rule of the reference's probe (jaxfmm/tune.py:69-120), the wisdom key's
buckets (:44-48) and the wisdom file's round trip."""
import numpy as np
import pytest

from hfmm_b200 import tune


def test_pick_takes_the_fastest_within_the_anchor_slack():
    res = [(32, 5.0, 3e-7), (64, 6.0, 2e-7), (128, 4.0, 4e-7)]
    assert tune.pick(res, 1.5, anchor=64)[0] == 32          # 128 is too inaccurate
    assert tune.pick(res, 2.0, anchor=64)[0] == 128         # within 2x of the anchor
    assert tune.pick(res, 1.0, anchor=64)[0] == 64


def test_pick_anchors_on_the_best_accuracy_without_the_default():
    res = [(32, 5.0, 3e-7), (128, 4.0, 4e-7)]
    assert tune.pick(res, 1.2, anchor=64)[0] == 32
    assert tune.pick(res, 1.5, anchor=64)[0] == 128
    assert tune.pick([(16, 1.0, 0.0), (32, 0.5, 1e-17)], 1.5)[0] == 32   # the 1e-16 floor
    with pytest.raises(RuntimeError):
        tune.pick([], 1.5, anchor=64)


def test_wisdom_key_buckets():
    k = tune.wisdom_key("helmholtz", 1_000_000, 1.0, 8, 0, "NVIDIA B200")
    assert k == "v1|helmholtz|N2^20|A2^0|p8|prec0|NVIDIA_B200"
    assert tune.wisdom_key("helmholtz", 900_000, 1.3, 8, 0, "x") == \
        tune.wisdom_key("helmholtz", 1_100_000, 1.2, 8, 0, "x")
    assert "A2^10" in tune.wisdom_key("helmholtz", 10, 1e9, 8, 0, "x")
    pos = np.array([[0, 0, 0], [4, 1, 2.0]])
    assert tune.aspect(pos) == 4.0


def test_wisdom_round_trip(tmp_path, monkeypatch):
    path = str(tmp_path / "sub" / "w.json")
    tune._save(path, {"a": {"N_max": 64}})
    assert tune._load(path) == {"a": {"N_max": 64}}
    assert tune._load(str(tmp_path / "missing.json")) == {}
    monkeypatch.setenv("HFMM_B200_WISDOM", path)
    assert tune.wisdom_path() == path
