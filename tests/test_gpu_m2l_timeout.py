"""The bounded-wait failure path of the tcgen05 M2L kernel, made on purpose without
a GPU fault: a test-only switch (hfmm_debug_m2l_wait) leaves the first operand
stage of every CTA without its gather arrivals, so the MMA thread's wait, limited
here to 20 ms, runs out. The kernel must then drain the TMA loads and MMAs it
issued, free its tensor memory and return; the host reads the timeout flag (4)
through hfmm_plan_check as HFMM_ERR_DEVICE. The context stays usable: the next
evaluate, with the switch off, is bit-identical to one made before."""
import numpy as np
import pytest

from cases import complex_uniform

pytestmark = pytest.mark.gpu


def test_m2l_wait_runs_out_drains_and_reports():
    import torch
    import hfmm_b200
    from hfmm_b200 import _lib
    lib = _lib.load()
    pos, q = complex_uniform(6000)
    st = hfmm_b200.setup(pos, 4.0, p=6, N_max=32)
    qt = torch.as_tensor(q, device="cuda")
    before = hfmm_b200.evaluate_field(st, qt, precision=hfmm_b200.PREC_MIXED)
    try:
        assert lib.hfmm_debug_m2l_wait(20_000_000, 1) == 0
        with pytest.raises(hfmm_b200.HFMMError) as ei:
            hfmm_b200.evaluate_field(st, qt, precision=hfmm_b200.PREC_MIXED)
    finally:
        lib.hfmm_debug_m2l_wait(0, 0)
    assert ei.value.code == -5
    assert "device error flag 4" in str(ei.value)
    after = hfmm_b200.evaluate_field(st, qt, precision=hfmm_b200.PREC_MIXED)
    assert torch.equal(before[0], after[0]) and torch.equal(before[1], after[1])
    # the FP64 path on the same plan is unaffected as well
    a = hfmm_b200.evaluate_field(st, qt, precision=hfmm_b200.PREC_FP64)
    assert np.isfinite(a[0].cpu().numpy()).all()
    st.close()


def test_m2l_grid_mode_wait_runs_out_drains_and_reports():
    """The same failure path when the M2L reads its sources from the dense box grid
    (complete levels, complex charges, low-rank tables): stage 0 is never loaded."""
    import torch
    import hfmm_b200
    from hfmm_b200 import _lib
    lib = _lib.load()
    pos, q = complex_uniform(30000)
    st = hfmm_b200.setup(pos, 6.0, p=8, N_max=32, m2l_compress=1e-7)
    qt = torch.as_tensor(q, device="cuda")
    before = hfmm_b200.evaluate_field(st, qt, precision=hfmm_b200.PREC_MIXED)
    try:
        assert lib.hfmm_debug_m2l_wait(20_000_000, 1) == 0
        with pytest.raises(hfmm_b200.HFMMError) as ei:
            hfmm_b200.evaluate_field(st, qt, precision=hfmm_b200.PREC_MIXED)
    finally:
        lib.hfmm_debug_m2l_wait(0, 0)
    assert ei.value.code == -5
    assert "device error flag 4" in str(ei.value)
    after = hfmm_b200.evaluate_field(st, qt, precision=hfmm_b200.PREC_MIXED)
    assert torch.equal(before[0], after[0]) and torch.equal(before[1], after[1])
    st.close()
