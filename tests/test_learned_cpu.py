"""Host logic of the learned expansion order, without a GPU: the NumPy network
oracle against finite differences, the label read off an error curve, the
conservative order, the tree features, and the network entry points' argument
checks."""
import math

import numpy as np
import pytest

from oracle import mlp as om


def _rand_net(n_in, n_out, seed=0):
    rng = np.random.default_rng(seed)
    return rng.normal(0, 0.3, om.param_count(n_in, n_out))


@pytest.mark.parametrize("n_in,n_out", [(24, 2), (5, 1), (64, 4)])
def test_oracle_gradient_matches_finite_differences(n_in, n_out):
    rng = np.random.default_rng(1)
    P = _rand_net(n_in, n_out)
    X = rng.normal(size=(7, n_in))
    T = rng.normal(size=(7, n_out))
    _, G = om.loss_grad(P, X, T, n_out)
    idx = rng.choice(len(P), 40, replace=False)
    idx = np.concatenate([idx, [len(P) - 1, len(P) - n_out - 1, 0]])
    h = 1e-6
    for i in idx:
        d = np.zeros_like(P)
        d[i] = h
        num = (om.loss_grad(P + d, X, T, n_out)[0] - om.loss_grad(P - d, X, T, n_out)[0]) / (2 * h)
        assert abs(num - G[i]) <= 1e-7 + 1e-5 * abs(num), (i, num, G[i])


def test_oracle_adam_decreases_loss():
    rng = np.random.default_rng(2)
    X = rng.normal(size=(64, 6))
    T = np.stack([X[:, 0] * 2 - X[:, 1], np.sin(X[:, 2])], 1)
    P0 = _rand_net(6, 2)
    l0 = om.loss_grad(P0, X, T, 2)[0]
    _, _, _, l1 = om.adam(P0, X, T, 2, steps=200, lr=3e-3)
    assert l1 < 0.2 * l0


def test_param_count_matches_library():
    from hfmm_b200 import _lib
    for n_in, n_out in ((24, 2), (1, 1), (64, 4)):
        assert _lib.lib.hfmm_mlp_param_count(n_in, n_out) == om.param_count(n_in, n_out)
    assert _lib.lib.hfmm_mlp_param_count(0, 1) == -1
    assert _lib.lib.hfmm_mlp_param_count(65, 1) == -1
    assert _lib.lib.hfmm_mlp_param_count(8, 5) == -1


def test_network_entry_points_reject_null():
    from hfmm_b200 import _lib
    assert _lib.lib.hfmm_mlp_forward(None, None, 4, 24, 2, None, None) == -1
    assert _lib.lib.hfmm_mlp_grad(None, None, None, 4, 24, 2, None, None, None) == -1
    assert _lib.lib.hfmm_mlp_train(None, None, None, 0, None, None, 4, 24, 2, 1, 1e-3, None,
                                   None) == -1


def test_label_p():
    from hfmm_b200.learned import label_p
    ps = [4, 5, 6, 7, 8]
    errs = [1e-2, 1e-3, 1e-4, 1e-5, 1e-6]
    assert label_p(ps, errs, 1e-1) == 4.0
    assert label_p(ps, errs, 1e-4) == pytest.approx(6.0)
    assert label_p(ps, errs, 10 ** -4.5) == pytest.approx(6.5)
    assert label_p(ps, errs, 1e-7) == 9.0                      # unreachable: last + 1
    # a non-monotone curve: the label is where every higher order also passes
    assert label_p(ps, [1e-2, 1e-5, 1e-3, 1e-5, 1e-6], 1e-4) == pytest.approx(6.5)
    assert label_p([5, 6], [np.inf, 1e-8], 1e-6) == 6.0


def test_conservative_p():
    from hfmm_b200.learned import conservative_p
    assert conservative_p(1e-6) == 12
    assert conservative_p(1e-3) == 6
    assert conservative_p(1e-9) == 16
    assert conservative_p(0.5) == 4


def test_tree_features():
    from hfmm_b200.learned import tree_features, N_FEATURES
    lv = np.array([0, 1, 1, 2, 2, 2, 3])
    cnt = np.array([100, 60, 40, 30, 20, 10, 64])
    leaf = np.array([0, 0, 1, 1, 1, 1, 1], bool)
    f = tree_features(dict(lvls=lv, counts=cnt, is_leaf=leaf),
                      dict(max_depth=3, domain_extent=2.0), k=5.0, tol=1e-6, n_max=64)
    assert f.shape == (N_FEATURES,) and f.dtype == np.float32
    assert f[0] == pytest.approx(-6)
    assert f[1] == pytest.approx(10.0)
    assert f[2] == pytest.approx(math.log2(100))
    assert f[3] == 3
    assert f[4] == pytest.approx(10.0 / 8) and f[5] == pytest.approx(10.0 / 16) and f[6] == 0
    assert f[10] == pytest.approx(3 / 7) and f[11] == pytest.approx(1 / 7)
    # leaves with 40, 30, 20, 10, 64 points of 64: bins of 1/8
    assert f[16:24].sum() == pytest.approx(1.0)
    assert f[16 + 5] == pytest.approx(1 / 5)   # 40/64 = 0.625
    assert f[23] == pytest.approx(1 / 5)       # 64/64 lands in the last bin


def test_training_samples_from_sweep():
    from hfmm_b200 import train_order as to
    ps = np.arange(4, 9)
    data = dict(ps=ps, feats=np.zeros((2, 24), np.float32),
                err64=np.array([[1e-2, 1e-4, 1e-6, 1e-8, 1e-10]] * 2),
                errmx=np.array([[np.inf, 1e-4, 1e-6, 5e-7, 5e-7]] * 2),
                leaf_t=np.array([[3.0, 1.0, 2.0, 4.0], [1.0, 2.0, 3.0, 4.0]]))
    X, T = to.samples(data, tols=(1e-3, 1e-6, 1e-8))
    assert X.shape == (6, 24) and T.shape == (6, 2)
    assert X[0, 0] == pytest.approx(-3) and X[2, 0] == pytest.approx(-8)
    assert T[1, 0] == pytest.approx(6.0)          # mixed curve at 1e-6
    assert T[2, 0] == pytest.approx(7.0)          # FP64 curve at 1e-8
    assert T[0, 1] == 5.0 and T[3, 1] == 4.0      # log2 of the fastest leaf size


def test_choose_keeps_the_leaf_at_64_or_128():
    from hfmm_b200.learned import OrderNet
    assert OrderNet.choose_from([7.6, 4.0]) == (9, 64)      # p rounded up after the margin
    assert OrderNet.choose_from([7.4, 7.6]) == (8, 128)
    assert OrderNet.choose_from([2.0, 9.0]) == (4, 128)     # p clamped to [4, 16]
    assert OrderNet.choose_from([30.0, 6.4]) == (16, 64)


def test_network_is_consulted_only_in_its_range():
    from hfmm_b200.learned import network_applies, TOL_LEARNED, KD_TRUSTED
    f = np.zeros(24, np.float32)
    f[1] = 30.0                                   # the batched workload's largest k x extent
    assert network_applies(f, 1e-6)
    f[1] = 44.0                                   # 8M clustered points at k = 40: in the sweep
    assert network_applies(f, 1e-6)
    f[1] = KD_TRUSTED + 1.0                       # beyond 1.5 x the sweep's largest (50)
    assert not network_applies(f, 1e-6)
    f[1] = KD_TRUSTED
    assert network_applies(f, 1e-6)
    f[1] = 10.0
    assert not network_applies(f, TOL_LEARNED / 2)



def test_label_p_skips_orders_not_swept():
    """Merged sweeps: NaN marks an order a problem's sweep did not run; labels come
    from the orders that ran (inf still marks an order that does not apply)."""
    from hfmm_b200.learned import label_p
    ps = [4, 5, 6, 7, 8, 9]
    errs = [1e-2, 1e-3, 1e-4, 1e-5, np.nan, np.nan]        # swept 4..7 only
    assert label_p(ps, errs, 1e-4) == pytest.approx(6.0)
    assert label_p(ps, errs, 1e-6) == 8.0                    # unreachable: last run + 1
    errs = [np.nan, np.nan, 1e-4, 1e-5, 1e-6, 1e-7]          # swept 6..9 only
    assert label_p(ps, errs, 1e-3) == 6.0                    # first run order meets it
    assert label_p(ps, errs, 10 ** -5.5) == pytest.approx(7.5)


def test_merge_lays_sweeps_on_the_union_of_orders():
    from hfmm_b200 import train_order
    rng = np.random.default_rng(0)

    def sweep(ps, n):
        m = len(ps)
        return dict(feats=rng.random((n, 24)), err64=10.0 ** -rng.uniform(2, 8, (n, m)),
                    errmx=10.0 ** -rng.uniform(2, 8, (n, m)), t64=rng.random((n, m)),
                    tmx=rng.random((n, m)), leaf_t=rng.random((n, 4)), leaf_p=np.full(n, 8),
                    n=np.full(n, 1000), k=rng.random(n), kind=np.array(["uniform"] * n),
                    ps=np.asarray(ps))
    a, b = sweep(range(4, 15), 3), sweep(range(6, 17), 2)
    m = train_order.merge([a, b])
    assert list(m["ps"]) == list(range(4, 17)) and m["err64"].shape == (5, 13)
    assert np.isnan(m["err64"][:3, 11:]).all() and np.isnan(m["err64"][3:, :2]).all()
    assert np.array_equal(m["err64"][:3, :11], a["err64"])
    assert np.array_equal(m["errmx"][3:, 2:], b["errmx"])
    Xa, Ta = train_order.samples(a)
    Xm, Tm = train_order.samples(m)
    assert np.array_equal(Tm[:len(Ta)], Ta)                  # a's labels are unchanged


def test_decode_cache_stands_in_for_level_decodes():
    """The sweep swaps operators.level_decodes for a memoising wrapper: same
    parameters, same results, one computation per key."""
    import inspect
    from hfmm_b200 import operators, train_order
    cache = train_order._DecodeCache()
    mine = list(inspect.signature(cache.__call__).parameters.values())
    theirs = list(inspect.signature(operators.level_decodes).parameters.values())
    assert len(mine) == len(theirs) and [q.default for q in mine] == [q.default for q in theirs]
    a = cache(3, 2, 1.0, 2.0, False, 1e-7, "helmholtz")
    b = operators.level_decodes(3, 2, 1.0, 2.0, False, 1e-7, "helmholtz")
    assert all(np.array_equal(x, y) for x, y in zip(a, b))
    assert cache(3, 2, 1.0, 2.0, False, 1e-7, "helmholtz") is a and len(cache.memo) == 1
