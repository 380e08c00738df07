"""The NumPy stand-in for JAX that runs the reference to make the golden fixtures
(tests/golden/jax_on_numpy.py) follows JAX's documented semantics where they
differ from NumPy's: gathers clamp out-of-range indices, scatters drop them,
sorts are stable, segment reductions drop out-of-range ids, float-to-integer
conversion saturates. The module is used without installing it into
`sys.modules` here, so no other test sees a `jax` package."""
import os
import sys

import numpy as np

sys.path.insert(0, os.path.join(os.path.dirname(__file__), "golden"))
import jax_on_numpy as J  # noqa: E402


def arr(x, dtype=None):
    return J._wrap(np.asarray(x, dtype=dtype))


def test_gather_wraps_negatives_once_then_clamps():
    x = arr([10, 20, 30])
    assert x[np.array([5, -1, -7, 1])].tolist() == [30, 30, 10, 20]
    assert x.at[np.array([3])].get().tolist() == [30]
    y = arr(np.arange(12).reshape(3, 4))
    assert y[np.array([9]), 1:3].tolist() == [[9, 10]]


def test_gather_fill_mode():
    x = arr([1.0, 2.0])
    got = x.at[np.array([0, 2, -3])].get(mode="fill", fill_value=-5.0)
    assert got.tolist() == [1.0, -5.0, -5.0]
    assert np.isnan(x.at[np.array([7])].get(mode="fill")[0])


def test_scatter_drops_out_of_range_and_clip_clamps():
    x = arr([0, 0, 0])
    assert x.at[np.array([0, 5, -1, -9])].set(np.array([1, 2, 3, 4])).tolist() == [1, 0, 3]
    assert x.at[np.array([0, 5])].set(7, mode="clip").tolist() == [7, 0, 7]
    assert x.tolist() == [0, 0, 0]                       # functional update


def test_scatter_add_accumulates_repeats_and_set_keeps_the_last():
    x = arr([0, 0, 0])
    assert x.at[np.array([0, 0, 1, 4])].add(1).tolist() == [2, 1, 0]
    assert x.at[np.array([2, 2, 2])].set(np.array([5, 6, 7])).tolist() == [0, 0, 7]
    z = arr(np.zeros((2, 3)))
    got = z.at[np.array([1, 1, 3]), np.array([0, 2, 0])].add(np.array([1.0, 2.0, 4.0]))
    assert got.tolist() == [[0, 0, 0], [1, 0, 2]]


def test_sorts_are_stable():
    keys = np.array([3, 1, 3, 1, 2, 1])
    assert J._argsort(keys).tolist() == [1, 3, 5, 4, 0, 2]
    assert J._argsort(np.array([1, 2, 1]), descending=True).tolist() == [1, 0, 2]


def test_segment_reductions_drop_bad_ids():
    data = np.array([1, 2, 3, 4], np.int32)
    ids = np.array([0, 2, 2, 7])
    assert J._segment_sum(data, ids, num_segments=3).tolist() == [1, 0, 5]
    mx = J._segment_max(np.array([1.0, 5.0, 2.0]), np.array([1, 1, -1]), num_segments=3)
    assert mx[1] == 5.0 and mx[0] == -np.inf and mx[2] == -np.inf


def test_float_to_int_saturates():
    got = J._convert(np.array([np.nan, -1e30, 1e30, 2.7, -2.7]), np.int32)
    i = np.iinfo(np.int32)
    assert got.tolist() == [0, i.min, i.max, 2, -2]


def test_take_fills_by_default():
    got = J._take(np.array([1.0, 2.0, 3.0]), np.array([0, 3, -1]))
    assert got[0] == 1.0 and np.isnan(got[1]) and got[2] == 3.0


def test_control_flow_stacks_like_jax():
    xs = (np.arange(4), np.arange(4) * 2.0)
    out = J._lax_map(lambda t: (t[0] + 1, t[1] * t[0]), xs)
    assert out[0].tolist() == [1, 2, 3, 4] and out[1].tolist() == [0, 2, 8, 18]
    carry, ys = J._scan(lambda c, x: (c + x, c), 0, np.arange(5))
    assert int(carry) == 10 and ys.tolist() == [0, 0, 1, 3, 6]
    assert J._fori_loop(0, 4, lambda i, v: v + i, 0) == 6
    f = J.vmap(lambda a, b: a * b, in_axes=(0, None))
    assert f(np.arange(3), 2).tolist() == [0, 2, 4]


def test_map_over_nothing_keeps_the_element_shape():
    out = J._lax_map(lambda t: (t[0] * 2.0, t[1][:2]), (np.zeros((0, 3)), np.zeros((0, 4), np.int32)))
    assert out[0].shape == (0, 3) and out[1].shape == (0, 2) and out[1].dtype == np.int32


def test_scan_over_nothing_returns_the_carry_and_empty_outputs():
    carry, ys = J._scan(lambda c, x: (c + x.sum(), x * 2.0), 1.0, np.zeros((0, 3)))
    assert carry == 1.0 and ys.shape == (0, 3)


def test_bincount_length_drops_out_of_range_values():
    """jnp.bincount(x, weights, length=L): exactly L bins, values >= L dropped."""
    import jax_on_numpy as jn
    jnp = jn._NumpyModule("jax.numpy")
    assert np.array_equal(jnp.bincount(np.array([0, 1, 1, 5]), length=3), [1, 2, 0])
    w = np.array([0.5, 1.0, 2.0, 4.0])
    assert np.allclose(jnp.bincount(np.array([2, 2, 0, 9]), weights=w, length=4), [2.0, 0, 1.5, 0])
    assert np.array_equal(jnp.bincount(np.array([3, 1])), [0, 1, 0, 1])
