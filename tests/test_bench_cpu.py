"""bench.py's CPU legs on small problems (no GPU): the oracle sampler behind
``cpu_baseline`` and the reference arm, and the timed full oracle evaluate of the
calibration, which evaluates every padded near-field slot as the reference does.
Also: the oracle's near field gives the same result with and without cutting the
padded slots."""
import numpy as np
import pytest

import oracle as O
from cases import clustered


def _small(cfg, **kw):
    out = dict(cfg)
    out.update(kw)
    return out


def test_oracle_sampler_runs_and_scales():
    import bench
    cfg = _small(bench.CONFIGS["c1"], n=3000, p=4)
    total, sample, est = bench.OracleSampler(cfg, log=lambda *a: None).sample(0.6)
    assert total > 0 and np.isfinite(total)
    assert {"p2m", "l2p", "l2p_field", "decodes", "m2m_l2l", "m2l", "p2p", "p2p_field"} <= set(est)
    assert all(v >= 0 for v in est.values())
    assert "estimate, not a timed evaluate" in sample


def test_calibration_times_the_padded_reference_near_field(monkeypatch):
    import bench
    monkeypatch.setitem(bench.CONFIGS, "c1", _small(bench.CONFIGS["c1"], n=2500, p=4))
    seen = []
    real = O.hfmm.eval_direct

    def spy(s, *args, **kw):
        seen.append(s.get("near_trim", True))
        return real(s, *args, **kw)
    monkeypatch.setattr(O.hfmm, "eval_direct", spy)
    cal = bench.calibrate_c1(0.5, log=lambda *a: None)
    assert cal["timed_evaluate_s"] > 0 and cal["estimated_evaluate_s"] > 0
    # the full evaluate's near-field calls (4: 2 components x potential and field)
    # evaluate every padded slot; the sampler's calls carry no "pil" either way
    assert seen.count(False) == 4


def test_near_field_with_and_without_padding_cut():
    pos, q = clustered(400)
    st = O.setup(pos, 6.0, p=3, N_max=8, max_depth=2)     # wide, ragged leaves
    s = st[0]
    nv = (s["pil"] >= 0).sum(1)
    assert nv.max() > 4 * nv[nv > 0].mean()
    Q = np.stack([q, np.cos(np.arange(q.size))], 1)
    ppts, pchg, rev = O.hfmm._build_padded(s["positions"], Q, s["pil"])
    for field in (False, True):
        cut = O.hfmm.eval_direct(s, s["kernel"], ppts, pchg, rev, field)
        full = O.hfmm.eval_direct(dict(s, near_trim=False), s["kernel"], ppts, pchg, rev, field)
        assert O.relative_error(cut, full) < 1e-14


def test_clock_sampler_summary_from_nvidia_smi_rows():
    """The clocks record of the JSON line from nvidia-smi rows (index, sm, max sm,
    power, active reasons, then the four reason columns): median SM clock, highest
    max, the reasons seen active, malformed rows skipped."""
    import bench

    class _Proc:
        def terminate(self): pass
        def wait(self, timeout=None): return 0
        def kill(self): pass

    class _Thread:
        def join(self, timeout=None): pass

    cs = bench.ClockSampler(0)
    cs.proc, cs.t = _Proc(), _Thread()
    row = lambda sm, pc: ["0", str(sm), "1965", "900.1", "0x0", "Not Active", "Not Active",
                          "Not Active", pc]
    cs.rows = [row(1965, "Not Active"), row(1890, "Active"), row(1965, "Not Active"),
               ["garbage"], ["0", "[N/A]", "1965", "1", "x", "Not Active", "Not Active",
                             "Not Active", "Not Active"]]
    out = cs.stop()
    assert out["sm_mhz"] == 1965.0 and out["sm_max_mhz"] == 1965.0
    assert out["reasons"] == ["sw_power_cap"] and out["samples"] == 5
    cs2 = bench.ClockSampler(0)
    assert cs2.stop() is None            # never started
