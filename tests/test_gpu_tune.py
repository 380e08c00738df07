"""The leaf-size autotuner (hfmm_b200/tune.py, the reference's tune_kifmm at
jaxfmm/tune.py:123-172) on a B200: it probes every candidate, picks the fastest
within the accuracy slack of the N_max = 64 candidate, stores the class in the
wisdom file and takes it from there the second time; the plan it returns is the
plan a plain setup with the chosen leaf size gives."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_tune_leaf_probes_picks_and_remembers(tmp_path):
    import torch
    import hfmm_b200
    from hfmm_b200 import tune
    rng = np.random.default_rng(5)
    n = 20000
    pos = rng.random((n, 3))
    q = rng.normal(size=n) + 1j * rng.normal(size=n)
    path = str(tmp_path / "wisdom.json")
    params, st, report = tune.tune_leaf(pos, 10.0, q, p=6, wisdom=path)
    probes = {r[0]: r for r in report}
    assert set(probes) == {32, 64, 128} and all(len(r) == 3 for r in report)
    anchor = probes[64][2]
    assert params["N_max"] in probes and params["rel"] <= 1.5 * anchor
    feasible = [r for r in report if r[2] <= 1.5 * anchor]
    assert params["ms"] == min(r[1] for r in feasible)
    assert params["rel"] < 1e-4
    params2, st2, report2 = tune.tune_leaf(pos, 10.0, q, p=6, wisdom=path)
    assert report2[0][0] == "wisdom" and params2["N_max"] == params["N_max"]
    ref = hfmm_b200.setup(pos, 10.0, p=6, N_max=params["N_max"])
    qt = torch.as_tensor(q, device="cuda")
    a = hfmm_b200.evaluate_field(st, qt)[0].cpu().numpy()
    b = hfmm_b200.evaluate_field(st2, qt)[0].cpu().numpy()
    c = hfmm_b200.evaluate_field(ref, qt)[0].cpu().numpy()
    assert np.array_equal(a, c) and np.array_equal(b, c)
    for s in (st, st2, ref):
        s.close()
