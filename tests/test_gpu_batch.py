"""Streamed M2L tables and batched graph launches on the GPU.

Streaming regenerates each level's M2L matrices per evaluate with the same
arithmetic as the resident device tables, so results must be bit-identical.
A batch replays the same kernels with the same inputs, so each problem's result
must equal its individual evaluate bit for bit as well."""
import json

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _problem(n, k, seed, clustered=False):
    rng = np.random.default_rng(seed)
    if clustered:
        c = rng.uniform(0.2, 0.8, (3, 3))
        x = np.clip(c[rng.integers(0, 3, n)] + 0.05 * rng.standard_normal((n, 3)), 0, 1)
    else:
        x = rng.random((n, 3))
    q = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    return x, float(k), q


@pytest.mark.parametrize("p,mixed", [(4, False), (6, False), (6, True), (7, True)])
def test_streamed_tables_bit_identical(p, mixed):
    import hfmm_b200 as hf
    x, k, q = _problem(5000, 5.0, 1, clustered=True)
    prec = hf.PREC_MIXED if mixed else hf.PREC_FP64
    a = hf.setup(x, k, p=p, N_max=32)
    b = hf.setup(x, k, p=p, N_max=32, stream_tables=True)
    pa, ea = hf.evaluate_field(a, q, prec)
    pb, eb = hf.evaluate_field(b, q, prec)
    assert np.array_equal(pa, pb) and np.array_equal(ea, eb)
    # the other precision through the same streamed plan, then back
    other = hf.PREC_FP64 if mixed else hf.PREC_MIXED
    assert np.array_equal(hf.evaluate_field(a, q, other)[0], hf.evaluate_field(b, q, other)[0])
    assert np.array_equal(hf.evaluate_field(b, q, prec)[0], pa)
    a.close()
    b.close()


def test_shared_workspace_and_errors():
    import hfmm_b200 as hf
    from hfmm_b200 import _lib
    x1, k1, q1 = _problem(3000, 3.0, 2)
    x2, k2, q2 = _problem(4000, 9.0, 3)
    s1 = hf.setup(x1, k1, p=6, N_max=32, stream_tables=True)
    s2 = hf.setup(x2, k2, p=6, N_max=32, stream_tables=True)
    need = _lib.ctypes.c_int64()
    _lib.check(_lib.lib.hfmm_plan_workspace_bytes(s1.handle, _lib.ctypes.byref(need)))
    ws = torch.empty(need.value // 8, dtype=torch.float64, device="cuda")
    with pytest.raises(hf.HFMMError):      # too small
        _lib.check(_lib.lib.hfmm_plan_bind_workspace(s1.handle, ws.data_ptr(), need.value - 8))
    for s in (s1, s2):
        _lib.check(_lib.lib.hfmm_plan_bind_workspace(s.handle, ws.data_ptr(), need.value))
    r1 = hf.setup(x1, k1, p=6, N_max=32)
    r2 = hf.setup(x2, k2, p=6, N_max=32)
    for prec in (hf.PREC_FP64, hf.PREC_MIXED):
        assert np.array_equal(hf.evaluate_field(s1, q1, prec)[0], hf.evaluate_field(r1, q1, prec)[0])
        assert np.array_equal(hf.evaluate_field(s2, q2, prec)[0], hf.evaluate_field(r2, q2, prec)[0])
    # a resident plan cannot take a workspace; streaming is chosen before the tables
    with pytest.raises(hf.HFMMError):
        _lib.check(_lib.lib.hfmm_plan_bind_workspace(r1.handle, ws.data_ptr(), need.value))
    with pytest.raises(hf.HFMMError):
        _lib.check(_lib.lib.hfmm_plan_set_streaming(r1.handle, 1))
    for s in (s1, s2, r1, r2):
        s.close()


def _batch_problems():
    specs = [(20000, 2.0, 10, False, 8), (3000, 7.0, 11, True, 6), (9000, 12.0, 12, False, 7),
             (1500, 1.0, 13, True, 5), (12000, 4.0, 14, True, 4)]
    out = []
    for n, k, seed, cl, p in specs:
        x, k, q = _problem(n, k, seed, cl)
        out.append((x, k, q, p))
    return out


@pytest.mark.parametrize("n_streams,streamed", [(1, False), (3, True), (8, True)])
def test_batch_matches_individual_evaluates(n_streams, streamed):
    import hfmm_b200 as hf
    from hfmm_b200.batch import Batch
    probs = _batch_problems()
    states = [hf.setup(x, k, p=p, N_max=32, stream_tables=streamed) for x, k, q, p in probs]
    precs = [hf.PREC_MIXED, hf.PREC_FP64, hf.PREC_MIXED, hf.PREC_FP64, hf.PREC_FP64]
    qs = [torch.as_tensor(q).cuda() for _, _, q, _ in probs]
    b = Batch(states, n_streams)
    assert {b.stream_of(i) for i in range(len(states))} <= set(range(min(n_streams, 5)))
    outs = b.bind(qs, field=True, precision=precs)
    for _ in range(2):                      # relaunch: same results
        b.launch()
        torch.cuda.synchronize()
        b.check_errors()
        for st, q, prec, (phi, E) in zip(states, qs, precs, outs):
            ref = hf.setup(st.positions, st.k, p=st.p, N_max=32)
            rp, re = hf.evaluate_field(ref, q, prec)
            assert torch.equal(phi, rp) and torch.equal(E, re)
            ref.close()
    b.close()
    for st in states:
        st.close()


def test_batch_repoint_requires_capture():
    import hfmm_b200 as hf
    from hfmm_b200 import _lib
    from hfmm_b200.batch import Batch
    probs = _batch_problems()[:2]
    states = [hf.setup(x, k, p=p, N_max=32, stream_tables=True) for x, k, q, p in probs]
    qs = [torch.as_tensor(q).cuda() for _, _, q, _ in probs]
    b = Batch(states, 2)
    outs = b.bind(qs, field=False)
    b.launch()
    q2 = qs[0] * 2.0
    qr, qi = q2.real.contiguous(), q2.imag.contiguous()
    _lib.check(_lib.lib.hfmm_batch_set_problem(b._h, 0, qr.data_ptr(), qi.data_ptr(),
                                               outs[0][0].data_ptr(), None, hf.PREC_MIXED))
    with pytest.raises(hf.HFMMError):
        _lib.check(_lib.lib.hfmm_batch_launch(b._h, None))
    _lib.check(_lib.lib.hfmm_batch_capture(b._h))
    b.launch()
    torch.cuda.synchronize()
    ref = hf.evaluate_field(states[0], q2, hf.PREC_MIXED)[0]
    assert torch.equal(outs[0][0], ref)
    b.close()
    for st in states:
        st.close()


def test_autotune_writes_and_reuses_wisdom(tmp_path):
    import hfmm_b200 as hf
    from hfmm_b200.batch import autotune
    probs = _batch_problems()
    states = [hf.setup(x, k, p=p, N_max=32, stream_tables=True) for x, k, q, p in probs]
    qs = [torch.as_tensor(q).cuda() for _, _, q, _ in probs]
    w = tmp_path / "wisdom.json"
    b, times = autotune(states, qs, candidates=(1, 2, 4), wisdom=str(w), reps=2)
    store = json.loads(w.read_text())
    assert len(store) == 1
    entry = next(iter(store.values()))
    # the plans have no low-rank M2L, so the queue does not apply: "S,0" keys only
    assert entry["n_streams"] == b.n_streams and set(entry["ms"]) == {"1,0", "2,0", "4,0"}
    assert f"{b.n_streams},0" == min(times, key=times.get)
    b.close()
    b2, t2 = autotune(states, qs, candidates=(1, 2, 4), wisdom=str(w))
    assert b2.n_streams == entry["n_streams"] and t2 == entry["ms"]
    b2.close()
    for st in states:
        st.close()


def test_auto_batch_certifies_every_problem():
    from hfmm_b200.batch import AutoBatch
    probs = _batch_problems()[:3]
    ab = AutoBatch([(x, k) for x, k, _, _ in probs], tol=1e-5, net=False, n_streams=2)
    ab.bind([q for _, _, q, _ in probs], field=True)
    ab.batch.launch()
    rep = ab.certify()
    assert all(r["certified"] for r in rep)
    assert all(r["p"] == 10 for r in rep)
    ab.close()


def test_in_graph_check_matches_host_referee():
    """The direct sum and error sums captured in the graph give the errors the
    host-side referee gives for the same targets."""
    import hfmm_b200 as hf
    from hfmm_b200.batch import Batch
    probs = _batch_problems()[:3]
    states = [hf.setup(x, k, p=p, N_max=32, stream_tables=True) for x, k, q, p in probs]
    qs = [torch.as_tensor(q).cuda() for _, _, q, _ in probs]
    rng = np.random.default_rng(5)
    tgs = [torch.as_tensor(np.sort(rng.choice(st.n, 200, replace=False)).astype(np.int32)).cuda()
           for st in states]
    b = Batch(states, 2)
    outs = b.bind(qs, field=True, precision=hf.PREC_MIXED, checks=tgs)
    b.launch()
    torch.cuda.synchronize()
    b.check_errors()
    got = b.check_rel_errors()
    for st, q, tg, (phi, E), (e_phi, e_E) in zip(states, qs, tgs, outs, got):
        r_phi, r_E = hf.direct_at(st, q.real.contiguous(), q.imag.contiguous(), tg, field=True)
        want_phi = float(torch.linalg.norm(phi[tg.long()] - r_phi) / torch.linalg.norm(r_phi))
        want_E = float(torch.linalg.norm(E[tg.long()] - r_E) / torch.linalg.norm(r_E))
        assert e_phi == pytest.approx(want_phi, rel=1e-9) and e_E == pytest.approx(want_E, rel=1e-9)
        assert 0 < e_phi < 1e-3
    b.close()
    for st in states:
        st.close()


def _compressed_problems(n_probs=6):
    rng = np.random.default_rng(21)
    out = []
    for i in range(n_probs):
        n = int(np.exp(rng.uniform(np.log(4000), np.log(40000))))
        x, k, q = _problem(n, float(rng.uniform(1.0, 12.0)), 30 + i, bool(i % 2))
        out.append((x, k, q))
    return out


@pytest.mark.parametrize("n_streams", [1, 4])
def test_queued_m2l_matches_individual_evaluates(n_streams):
    """The batch's queued M2L (one persistent kernel over every problem's M2L tiles,
    hfmm_batch_set_queue) computes each tile as the per-level kernel does, so the
    batch's results equal each plan's own evaluate bit for bit, launch after launch."""
    import hfmm_b200 as hf
    from hfmm_b200.batch import Batch
    probs = _compressed_problems()
    states = [hf.setup(x, k, p=6, N_max=32, stream_tables=True, m2l_compress=1e-7)
              for x, k, _ in probs]
    qs = [torch.as_tensor(q).cuda() for _, _, q in probs]
    b = Batch(states, n_streams, queue=True)
    outs = b.bind(qs, field=True, precision=hf.PREC_MIXED)
    assert b.queued, b.queue_note
    refs = [hf.evaluate_field(st, q, hf.PREC_MIXED) for st, q in zip(states, qs)]
    for _ in range(2):
        b.launch()
        torch.cuda.synchronize()
        b.check_errors()
        for (phi, E), (rp, re) in zip(outs, refs):
            assert torch.equal(phi, rp) and torch.equal(E, re)
    b.close()
    # a problem with real charges: the column counts differ, the queue does not apply
    qs[0] = qs[0].real.contiguous()
    b = Batch(states, 2, queue=True)
    outs = b.bind(qs, field=True, precision=hf.PREC_MIXED)
    assert not b.queued
    b.launch()
    torch.cuda.synchronize()
    for st, q, (phi, E) in zip(states, qs, outs):
        rp, re = hf.evaluate_field(st, q, hf.PREC_MIXED)
        assert torch.equal(phi, rp) and torch.equal(E, re)
    b.close()
    for st in states:
        st.close()


def test_queued_m2l_wait_runs_out_and_reports():
    """The persistent queue kernel's bounded waits: a test switch starves every CTA's
    first stage (20 ms limit); the launch ends with the timeout flag (4) on the plans,
    and a graph captured again without the switch gives the plans' own results."""
    import hfmm_b200 as hf
    from hfmm_b200 import _lib
    from hfmm_b200.batch import Batch
    lib = _lib.load()
    probs = _compressed_problems(4)
    states = [hf.setup(x, k, p=6, N_max=32, stream_tables=True, m2l_compress=1e-7)
              for x, k, _ in probs]
    qs = [torch.as_tensor(q).cuda() for _, _, q in probs]
    b = Batch(states, 2, queue=True)
    try:
        lib.hfmm_debug_m2l_wait(20_000_000, 1)
        outs = b.bind(qs, field=True, precision=hf.PREC_MIXED)
        assert b.queued, b.queue_note
        b.launch()
        torch.cuda.synchronize()
    finally:
        lib.hfmm_debug_m2l_wait(0, 0)
    flagged = 0
    for st in states:
        try:
            hf.check_errors(st)
        except hf.HFMMError as e:
            assert e.code == -5 and "device error flag 4" in str(e)
            flagged += 1
    assert flagged >= 1
    outs = b.bind(qs, field=True, precision=hf.PREC_MIXED)
    b.launch()
    torch.cuda.synchronize()
    b.check_errors()
    for st, q, (phi, E) in zip(states, qs, outs):
        rp, re = hf.evaluate_field(st, q, hf.PREC_MIXED)
        assert torch.equal(phi, rp) and torch.equal(E, re)
    b.close()
    for st in states:
        st.close()


def test_solve_from_host_rescales_exactly():
    """Batch.solve runs new host charges through the captured graph (no re-capture):
    charges scaled by 2 give results scaled by 2 bit for bit (every step of the
    evaluate is linear in the charges and a power of two scales exactly), real
    charges into a complex-bound problem count as zero imaginary parts, and a wrong
    shape, count or a complex vector into a real-bound problem is refused."""
    import hfmm_b200 as hf
    from hfmm_b200.batch import Batch
    probs = _batch_problems()[:3]
    states = [hf.setup(x, k, p=p, N_max=32, stream_tables=True) for x, k, q, p in probs]
    qs = [torch.as_tensor(q).cuda() for _, _, q, _ in probs]
    qs[2] = qs[2].real.contiguous()
    precs = [hf.PREC_MIXED, hf.PREC_FP64, hf.PREC_MIXED]
    b = Batch(states, 2)
    outs = b.bind(qs, field=True, precision=precs)
    b.launch()
    torch.cuda.synchronize()
    ref = [(phi.cpu().numpy(), E.cpu().numpy()) for phi, E in outs]
    host = [2.0 * q for _, _, q, _ in probs]
    host[2] = host[2].real.copy()
    for _ in range(2):
        res = b.solve(host)
        for (phi, E), (rp, re) in zip(res, ref):
            assert np.array_equal(phi, 2.0 * rp) and np.array_equal(E, 2.0 * re)
    res = b.solve([host[0].real.copy(), host[1], host[2]])
    r0 = hf.evaluate_field(states[0], torch.as_tensor(host[0].real.copy()).cuda(), hf.PREC_MIXED)
    r0 = r0[0].cpu().numpy()   # the one-column evaluate: same values to the mixed path's rounding
    assert np.linalg.norm(res[0][0] - r0) < 1e-6 * np.linalg.norm(r0)
    with pytest.raises(ValueError):
        b.solve(host[:2])
    with pytest.raises(ValueError):
        b.solve([host[0][:-1], host[1], host[2]])
    with pytest.raises(ValueError):
        b.solve([host[0], host[1], host[2] + 1j])
    b.close()
    for st in states:
        st.close()


def test_auto_batch_raises_the_missed_orders():
    """AutoBatch.raise_missed: problems whose in-graph check missed the tolerance take
    the next order and the batch is captured again; a few rounds certify every one."""
    from hfmm_b200.batch import AutoBatch
    probs = _batch_problems()[:3]
    ab = AutoBatch([(x, k) for x, k, _, _ in probs], tol=1e-6, net=False, n_streams=2)
    ab.choice = [(6, leaf) for _, leaf in ab.choice]        # start every problem too low
    import hfmm_b200 as hf
    from hfmm_b200.learned import precision_for, compress_for
    for i, ((x, k), (p, leaf)) in enumerate(zip(ab.problems, ab.choice)):
        ab.states[i].close()
        ab.precisions[i] = precision_for(ab.tol, p)
        ab.states[i] = hf.setup(x, k, p=p, N_max=leaf, stream_tables=True,
                                m2l_compress=compress_for(ab.tol, ab.precisions[i]))
    ab.bind([q for _, _, q, _ in probs], field=True)
    raised = []
    for _ in range(8):
        ab.batch.launch()
        torch.cuda.synchronize()
        r = ab.raise_missed()
        raised += r
        if not r:
            break
    assert raised and not r
    rep = ab.certify()
    assert all(x["certified"] and not x["fallback"] for x in rep)
    assert all(c[0] >= 6 for c in ab.choice) and max(c[0] for c in ab.choice) > 6
    ab.close()
