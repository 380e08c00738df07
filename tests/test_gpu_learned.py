"""The expansion-order network's CUDA kernels against the NumPy oracle, and the
certified auto-plan (check on sampled targets, plain rerun on a miss)."""
import numpy as np
import pytest
import torch

from oracle import mlp as om

pytestmark = pytest.mark.gpu

N_IN, N_OUT = 24, 2


def _dev(a):
    return torch.as_tensor(np.ascontiguousarray(a, np.float32)).cuda()


def _data(n=300, seed=0):
    rng = np.random.default_rng(seed)
    X = rng.normal(size=(n, N_IN)).astype(np.float32)
    T = np.stack([X[:, 0] - 0.5 * X[:, 3] * X[:, 5], np.tanh(X[:, 1] + X[:, 2])], 1)
    P = rng.normal(0, 0.2, om.param_count(N_IN, N_OUT)).astype(np.float32)
    return P, X, T.astype(np.float32)


def _rel(a, b):
    return float(np.linalg.norm(np.asarray(a, np.float64) - b) / np.linalg.norm(b))


def test_forward_matches_oracle():
    from hfmm_b200 import _lib
    P, X, _ = _data()
    Pd, Xd = _dev(P), _dev(X)       # held: the call reads them
    Y = torch.empty((len(X), N_OUT), dtype=torch.float32, device="cuda")
    assert _lib.lib.hfmm_mlp_forward(Pd.data_ptr(), Xd.data_ptr(), len(X), N_IN, N_OUT,
                                     Y.data_ptr(), None) == 0
    ref, _ = om.forward(P.astype(np.float64), X, N_OUT)
    assert _rel(Y.cpu().numpy(), ref) < 1e-5


@pytest.mark.parametrize("n", [1, 300, 4097])
def test_gradient_matches_oracle(n):
    from hfmm_b200 import _lib
    P, X, T = _data(n, seed=n)
    Pd, Xd, Td = _dev(P), _dev(X), _dev(T)
    G = torch.empty(len(P), dtype=torch.float32, device="cuda")
    loss = _lib.ctypes.c_double()
    assert _lib.lib.hfmm_mlp_grad(Pd.data_ptr(), Xd.data_ptr(), Td.data_ptr(), n,
                                  N_IN, N_OUT, G.data_ptr(), _lib.ctypes.byref(loss), None) == 0
    l_ref, g_ref = om.loss_grad(P.astype(np.float64), X, T, N_OUT)
    assert loss.value == pytest.approx(l_ref, rel=1e-5)
    assert _rel(G.cpu().numpy(), g_ref) < 1e-4


def test_adam_steps_match_oracle():
    from hfmm_b200 import _lib
    P, X, T = _data(256, seed=3)
    p, m, v = _dev(P), torch.zeros(len(P), device="cuda"), torch.zeros(len(P), device="cuda")
    Xd, Td = _dev(X), _dev(T)
    loss = _lib.ctypes.c_double()
    for t0 in (0, 3):           # two calls continue one optimiser run
        assert _lib.lib.hfmm_mlp_train(p.data_ptr(), m.data_ptr(), v.data_ptr(), t0,
                                       Xd.data_ptr(), Td.data_ptr(), len(X), N_IN, N_OUT,
                                       3, 1e-3, _lib.ctypes.byref(loss), None) == 0
    P_ref, m_ref, _, l_ref = om.adam(P.astype(np.float64), X, T, N_OUT, steps=6, lr=1e-3)
    got = p.cpu().numpy()
    assert _rel(got, P_ref) < 1e-5
    # the update itself: a few parameters with near-zero gradients may take the other sign
    assert _rel(got - P, P_ref - P) < 2e-2
    assert _rel(m.cpu().numpy(), m_ref) < 1e-3
    assert loss.value == pytest.approx(l_ref, rel=1e-3)


def test_training_on_gpu_fits():
    from hfmm_b200.learned import OrderNet
    _, X, T = _data(512, seed=4)
    net = OrderNet.init(X, T, seed=0, device="cuda")
    y0 = net.predict(X)
    l0 = float(np.mean(((y0 - T) / net.t_sd) ** 2))
    l1 = net.train(X, T, steps=1500, lr=3e-3)
    assert l1 < 0.1 * l0
    y1 = net.predict(X)
    assert float(np.mean(((y1 - T) / net.t_sd) ** 2)) == pytest.approx(l1, rel=1e-3)


def _problem(n=6000, seed=0):
    rng = np.random.default_rng(seed)
    x = rng.random((n, 3))
    q = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    return x, q


def test_auto_plan_below_the_learned_range_uses_the_conservative_order():
    from hfmm_b200.learned import AutoPlan, TOL_LEARNED
    x, q = _problem(3000, seed=3)
    ap = AutoPlan(x, 3.0, tol=TOL_LEARNED / 2)       # the network is not consulted
    assert ap.feats is None and ap.p == 14
    ap.evaluate(q)
    assert ap.report["p"] == 14
    ap.close()


def test_auto_plan_beyond_the_trained_wavenumbers_starts_conservative():
    """k x extent 80 lies beyond 1.5 x the training sweep's 50: the plan starts at the
    conservative order (12 at 1e-6) in mixed precision, without the network, and its
    report agrees with its own check (at this frequency and size the conservative
    order need not meet 1e-6; the reruns then step p up to 16)."""
    from hfmm_b200.learned import AutoPlan, KD_TRUSTED
    import hfmm_b200 as hf
    x, q = _problem(20000, seed=5)
    ap = AutoPlan(x, 80.0, tol=1e-6)
    assert ap.feats is not None and ap.feats[1] > KD_TRUSTED and not ap.network_used
    assert ap.p == 12 and ap.precision == hf.PREC_MIXED
    ap.evaluate(q)
    rep = ap.report
    assert not rep["network"] and rep["certified"] == (rep["error"] <= 1e-6)
    ap.close()


def test_auto_plan_conservative_certifies():
    from hfmm_b200.learned import AutoPlan
    x, q = _problem()
    ap = AutoPlan(x, 6.0, tol=1e-5, net=False)
    phi, E = ap.evaluate_field(q)
    assert ap.report["certified"] and not ap.report["fallback"]
    assert ap.report["p"] == 10 and ap.report["error"] <= 1e-5
    assert phi.shape == (len(x),) and E.shape == (len(x), 3)
    ap.close()


def _low_net():
    """A network that asks for the lowest order (p = 4, leaf 64) whatever the problem."""
    from hfmm_b200.learned import OrderNet, N_FEATURES, N_OUTPUTS
    return OrderNet(np.zeros(om.param_count(N_FEATURES, N_OUTPUTS), np.float32),
                    np.zeros(N_FEATURES), np.ones(N_FEATURES), np.array([2.0, 6.0]),
                    np.ones(2), device="cuda")


def test_auto_plan_raises_the_order_on_a_miss_and_keeps_it():
    """A network that asks for the lowest order misses 1e-6: the plan steps its order
    up (mixed from p = 5 on) until the check passes, keeps that order, and the next
    evaluate starts there without raising again."""
    from hfmm_b200.learned import AutoPlan
    import hfmm_b200 as hf
    x, q = _problem(seed=1)
    ap = AutoPlan(x, 4.0, tol=1e-6, net=_low_net())
    assert ap.p == 4 and ap.leaf == 64 and ap.p_network == 4
    ap.evaluate(q)
    rep = ap.report
    assert rep["certified"] and not rep["fallback"] and rep["raised"] >= 1
    assert 5 <= rep["p_final"] <= 12 and rep["precision"] == hf.PREC_MIXED
    assert ap.p == rep["p_final"]
    phi = ap.evaluate(q)
    rep2 = ap.report
    assert rep2["p"] == rep["p_final"] and rep2["raised"] == 0 and rep2["certified"]
    ref = hf.evaluate_field(ap.state, q, hf.PREC_MIXED)[0]
    assert np.array_equal(phi, ref)
    ap.close()


def test_auto_plan_reruns_plainly_past_the_conservative_order():
    """With no order left to raise to (the conservative order lowered to the network's
    for the test), a miss reruns plainly in FP64, stepping p by 2 until it certifies."""
    from hfmm_b200.learned import AutoPlan
    import hfmm_b200 as hf
    x, q = _problem(seed=1)
    ap = AutoPlan(x, 4.0, tol=1e-6, net=_low_net())
    ap.p_plain = 4
    phi = ap.evaluate(q)
    rep = ap.report
    assert rep["fallback"] and rep["certified"] and rep["raised"] == 0
    assert rep["precision"] == hf.PREC_FP64 and rep["p_final"] in (6, 8, 10, 12, 14, 16)
    st = hf.setup(x, 4.0, p=rep["p_final"], N_max=64)
    ref = hf.evaluate_field(st, q)[0]
    assert np.linalg.norm(phi - ref) <= 1e-13 * np.linalg.norm(ref)
    st.close()
    ap.close()


def test_gpu_training_generalises_across_problems():
    """Cross-validation on the committed sweep with the CUDA kernels: the held-out
    p error stays well under one order (0.36 on the 198-problem sweep, k x extent 1
    to 50). The leaf label is noisier: with the low-rank M2L, leaves of 64 and 128
    points often time within a few percent of each other (0.61 correct)."""
    import os
    from hfmm_b200 import train_order as to
    data = dict(np.load(os.path.join(os.path.dirname(to.__file__), "data", "order_sweep.npz")))
    cvs = to.cross_validate(data, steps_list=(400,), device="cuda")
    r = cvs[400]
    assert r["p_mae"] < 0.5, r
    assert r["under@0.5"] < 0.08, r
    assert r["leaf_acc"] > 0.4, r


def test_bundled_network_predicts_the_regime():
    from hfmm_b200.learned import OrderNet, features_for
    net = OrderNet.load(device="cuda")
    rng = np.random.default_rng(7)
    x = rng.random((200000, 3))
    f6 = features_for(x, 10.0, 1e-6)
    f3 = features_for(x, 10.0, 1e-3)
    p6 = net.predict(f6)[0, 0]
    p3 = net.predict(f3)[0, 0]
    assert 6.0 <= p6 <= 9.5, p6          # the sweep's labels at 1e-6 span 6.6 .. 8.4
    assert p3 < p6                         # a looser tolerance needs a lower order


def _time_eval(ap, q, reps=3):
    ap.evaluate_field(q)
    s = torch.cuda.current_stream()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(s)
    for _ in range(reps):
        ap.evaluate_field(q)
    b.record(s)
    b.synchronize()
    return a.elapsed_time(b) / reps


def test_ablation_network_beats_conservative_order():
    """What the trained network gains over the method without it: the same
    certified evaluate (mixed precision, 256-target check) with the conservative
    order in place of the network's."""
    from hfmm_b200.learned import AutoPlan
    rng = np.random.default_rng(11)
    n = 200000
    x = rng.random((n, 3))
    q = torch.as_tensor(rng.standard_normal(n) + 1j * rng.standard_normal(n)).cuda()
    learned = AutoPlan(x, 10.0, tol=1e-6)
    plain = AutoPlan(x, 10.0, tol=1e-6, net=False)
    t_l = _time_eval(learned, q)
    t_c = _time_eval(plain, q)
    rl, rc = learned.report, plain.report
    assert rl["certified"] and rc["certified"], (rl, rc)
    assert not rl["fallback"], rl
    assert rl["p"] < rc["p"] == 12, (rl, rc)
    assert t_l < 0.85 * t_c, (t_l, t_c, rl, rc)
    print(f"ablation: learned p={rl['p']} leaf={rl['leaf']} {t_l:.1f} ms, err {rl['error']:.2e}; "
          f"conservative p={rc['p']} {t_c:.1f} ms, err {rc['error']:.2e}")
    learned.close()
    plain.close()
