"""A NumPy stand-in for the part of JAX that the reference's Helmholtz path calls.

Test infrastructure only: `make_golden.py` (beside it) installs it into
`sys.modules` so that the reference's own Python code (`HFMM.py`, `jaxfmm/...`)
runs eagerly on the host and writes golden vectors. JAX is not installed in
this environment and there is no network, so this is the only way to execute the
reference here. Nothing in the library imports it.

What it reproduces of JAX (0.4.38, `jax_enable_x64` on, CPU backend):

* `jax.jit`, `jax.checkpoint`, `custom_vjp`: the function runs eagerly as written.
* `lax.map`, `lax.scan`, `lax.fori_loop`, `lax.while_loop`, `lax.cond`, `vmap`:
  Python loops over the mapped axis, results stacked (pure functions, so the
  values equal the vectorised ones up to floating-point summation order).
* Gathers (`x[idx]`, `x.at[idx].get()`) clamp out-of-range integer indices into
  range after wrapping negatives once; with `mode="fill"` they return the fill value.
* Scatters (`x.at[idx].set/add/min/max/mul`) drop out-of-range updates
  (`mode="clip"` clamps them instead); repeated indices under `set` keep the
  last update, as XLA's sequential CPU scatter does.
* `jnp.argsort` / `jnp.sort` are stable (JAX's default), `jnp.take` fills out of
  range, `segment_sum` / `segment_max` drop out-of-range segment ids.
* Float to integer conversion saturates and maps NaN to 0, as XLA's does.
"""
import functools
import sys
import types

import numpy as np

# ---------------------------------------------------------------------------
# the array type


def _wrap(x):
    if isinstance(x, Arr):
        return x
    if isinstance(x, np.ndarray):
        return x.view(Arr)
    if isinstance(x, np.generic):
        return np.asarray(x).view(Arr)
    if isinstance(x, tuple):
        return tuple(_wrap(v) for v in x)
    if isinstance(x, list):
        return [_wrap(v) for v in x]
    return x


def _is_int_index(c):
    if isinstance(c, (bool, np.bool_)):
        return False
    if isinstance(c, np.ndarray):
        return np.issubdtype(c.dtype, np.integer)
    return isinstance(c, np.integer)


def _expand(shape, idx):
    """Pairs (component, axis or None) for an index tuple; axis is the array axis
    an integer component addresses."""
    if not isinstance(idx, tuple):
        idx = (idx,)
    n_consumed = 0
    for c in idx:
        if c is None or c is Ellipsis:
            continue
        if isinstance(c, np.ndarray) and c.dtype == np.bool_:
            n_consumed += max(c.ndim, 1)
        else:
            n_consumed += 1
    out, ax = [], 0
    for c in idx:
        if c is None:
            out.append((c, None))
        elif c is Ellipsis:
            out.append((c, None))
            ax += len(shape) - n_consumed
        elif isinstance(c, np.ndarray) and c.dtype == np.bool_:
            out.append((c, None))
            ax += max(c.ndim, 1)
        else:
            out.append((c, ax))
            ax += 1
    return out


def _norm_index(idx, shape, how):
    """Rewrite the integer-array components of `idx`: negatives wrapped once, then
    out-of-range entries clamped (how="clip") or sent to the pad slot `n`
    (how="pad"). Returns the new index and the axes that need a pad slot."""
    parts = _expand(shape, idx)
    new, pad_axes = [], []
    for c, ax in parts:
        if ax is not None and _is_int_index(c):
            n = shape[ax]
            a = np.asarray(c).astype(np.int64)
            a = np.where(a < 0, a + n, a)
            if how == "clip":
                a = np.clip(a, 0, max(n - 1, 0))
            else:
                bad = (a < 0) | (a >= n)
                if bad.any():
                    pad_axes.append(ax)
                a = np.where(bad, n, a)
            new.append(a)
        elif isinstance(c, (list,)):
            new.append(np.asarray(c))
        else:
            new.append(c)
    return tuple(new), pad_axes


def _plain(idx):
    if isinstance(idx, tuple):
        return tuple(np.asarray(c) if isinstance(c, (Arr, list)) else c for c in idx)
    if isinstance(idx, list):
        return np.asarray(idx)
    return np.asarray(idx) if isinstance(idx, Arr) else idx


class Arr(np.ndarray):
    """ndarray with JAX's indexing rules and the `.at[]` update API."""

    def __getitem__(self, idx):
        idx = _plain(idx)
        base = self.view(np.ndarray)
        if any(_is_int_index(c) and not isinstance(c, (int,)) for c, _ in _expand(self.shape, idx)):
            idx, _ = _norm_index(idx, self.shape, "clip")
        return _wrap(base[idx])

    @property
    def at(self):
        return _At(self)

    def block_until_ready(self):
        return self

    def astype(self, dtype, *a, **k):
        return _wrap(_convert(self.view(np.ndarray), dtype))

    def __array_finalize__(self, obj):
        pass


def _convert(x, dtype):
    dt = np.dtype(dtype)
    x = np.asarray(x)
    if np.issubdtype(dt, np.integer) and np.issubdtype(x.dtype, np.floating):
        info = np.iinfo(dt)
        y = np.where(np.isnan(x), 0, x)
        y = np.clip(y, info.min, info.max)
        big = y >= float(info.max)
        out = y.astype(dt)
        return np.where(big, info.max, out).astype(dt) if big.any() else out
    return x.astype(dt)


class _At:
    def __init__(self, arr):
        self.arr = arr

    def __getitem__(self, idx):
        return _AtIdx(self.arr, _plain(idx))


class _AtIdx:
    def __init__(self, arr, idx):
        self.arr, self.idx = arr, idx

    def get(self, mode=None, fill_value=None, **_):
        base = self.arr.view(np.ndarray)
        if mode != "fill":
            idx, _ = _norm_index(self.idx, base.shape, "clip")
            return _wrap(base[idx])
        idx, pad = _norm_index(self.idx, base.shape, "pad")
        if fill_value is None:
            fill_value = (np.nan if np.issubdtype(base.dtype, np.inexact) else
                          True if base.dtype == np.bool_ else
                          np.iinfo(base.dtype).min if np.issubdtype(base.dtype, np.signedinteger)
                          else np.iinfo(base.dtype).max)
        padded = _pad_axes(base, pad, fill_value)
        return _wrap(padded[idx])

    def _scatter(self, op, v, mode):
        base = np.array(self.arr.view(np.ndarray))
        v = _convert(np.asarray(v), base.dtype)
        how = "clip" if mode == "clip" else "pad"
        idx, pad = _norm_index(self.idx, base.shape, how)
        padded = _pad_axes(base, pad, 0)
        if op is None:
            padded[idx] = v
        else:
            op.at(padded, idx, np.broadcast_to(v, padded[idx].shape))
        sl = tuple(slice(0, n) for n in base.shape)
        return _wrap(np.ascontiguousarray(padded[sl]))

    def set(self, v, mode=None, **_):
        return self._scatter(None, v, mode)

    def add(self, v, mode=None, **_):
        return self._scatter(np.add, v, mode)

    def mul(self, v, mode=None, **_):
        return self._scatter(np.multiply, v, mode)

    multiply = mul

    def min(self, v, mode=None, **_):
        return self._scatter(np.minimum, v, mode)

    def max(self, v, mode=None, **_):
        return self._scatter(np.maximum, v, mode)


def _pad_axes(base, axes, fill):
    if not axes:
        return base
    width = [(0, 1 if a in axes else 0) for a in range(base.ndim)]
    return np.pad(base, width, constant_values=fill)


# ---------------------------------------------------------------------------
# pytrees


def tree_flatten(x):
    leaves = []

    def rec(y):
        if y is None:
            return ("none",)
        if isinstance(y, tuple) and hasattr(y, "_fields"):
            return ("nt", type(y), [rec(v) for v in y])
        if isinstance(y, (tuple, list)):
            return (type(y), [rec(v) for v in y])
        if isinstance(y, dict):
            keys = sorted(y)
            return ("dict", keys, [rec(y[k]) for k in keys])
        leaves.append(y)
        return ("leaf",)

    return leaves, rec(x)


def tree_unflatten(spec, leaves):
    it = iter(leaves)

    def rec(s):
        if s[0] == "none":
            return None
        if s[0] == "leaf":
            return next(it)
        if s[0] == "nt":
            return s[1](*[rec(c) for c in s[2]])
        if s[0] == "dict":
            return {k: rec(c) for k, c in zip(s[1], s[2])}
        return s[0](rec(c) for c in s[1])

    return rec(spec)


def tree_map(f, x, *rest, is_leaf=None):
    lx, spec = tree_flatten(x)
    lr = [tree_flatten(r)[0] for r in rest]
    return tree_unflatten(spec, [f(*vals) for vals in zip(lx, *lr)])


def tree_leaves(x, is_leaf=None):
    return tree_flatten(x)[0]


def _stack_trees(outs):
    leaves0, spec = tree_flatten(outs[0])
    cols = [tree_flatten(o)[0] for o in outs]
    return tree_unflatten(spec, [_wrap(np.stack([np.asarray(c[i]) for c in cols]))
                                 for i in range(len(leaves0))])


def _index_tree(x, i):
    return tree_map(lambda a: _wrap(np.asarray(a)[i]), x)


def _lead_len(x):
    return len(np.asarray(tree_flatten(x)[0][0]))


# ---------------------------------------------------------------------------
# transformations and control flow


def jit(fun=None, **_):
    if fun is None:
        return lambda f: f
    return fun


def checkpoint(fun=None, **_):
    if fun is None:
        return lambda f: f
    return fun


remat = checkpoint


class custom_vjp:
    def __init__(self, fun, nondiff_argnums=()):
        self.fun = fun
        functools.update_wrapper(self, fun)

    def defvjp(self, fwd, bwd, **_):
        return None

    def __call__(self, *a, **k):
        return self.fun(*a, **k)


def _unsupported(name):
    def f(*a, **k):
        raise NotImplementedError(f"jax.{name} is not part of the NumPy stand-in")
    return f


def vmap(fun, in_axes=0, out_axes=0, **_):
    def mapped(*args):
        axes = in_axes if isinstance(in_axes, (tuple, list)) else (in_axes,) * len(args)
        n = None
        for a, ax in zip(args, axes):
            if ax is not None:
                n = np.asarray(tree_flatten(a)[0][0]).shape[ax]
                break
        outs = []
        for i in range(n):
            call = [a if ax is None else tree_map(lambda t: _wrap(np.take(np.asarray(t), i, axis=ax)), a)
                    for a, ax in zip(args, axes)]
            outs.append(fun(*call))
        res = _stack_trees(outs)
        if out_axes != 0:
            res = tree_map(lambda t: _wrap(np.moveaxis(np.asarray(t), 0, out_axes)), res)
        return res
    return mapped


def _empty_like_mapped(f, xs):
    """Zero-length result of mapping `f`: its structure and element shapes come
    from one call on a zero element, as JAX's tracing would give them."""
    dummy = tree_map(lambda a: _wrap(np.zeros(np.asarray(a).shape[1:], np.asarray(a).dtype)), xs)
    out = f(dummy)
    return tree_map(lambda o: _wrap(np.empty((0,) + np.asarray(o).shape, np.asarray(o).dtype)), out)


def _lax_map(f, xs, batch_size=None):
    n = _lead_len(xs)
    if n == 0:
        return _empty_like_mapped(f, xs)
    return _stack_trees([f(_index_tree(xs, i)) for i in range(n)])


def _scan(f, init, xs=None, length=None, reverse=False, **_):
    n = length if xs is None else _lead_len(xs)
    if n == 0:   # the stacked outputs' shapes come from one call, as tracing gives them
        dummy = None if xs is None else tree_map(
            lambda a: _wrap(np.zeros(np.asarray(a).shape[1:], np.asarray(a).dtype)), xs)
        _, y = f(init, dummy)
        return init, (None if y is None else tree_map(
            lambda o: _wrap(np.empty((0,) + np.asarray(o).shape, np.asarray(o).dtype)), y))
    carry, ys = init, []
    order = range(n - 1, -1, -1) if reverse else range(n)
    for i in order:
        carry, y = f(carry, None if xs is None else _index_tree(xs, i))
        ys.append(y)
    if reverse:
        ys = ys[::-1]
    if not ys or ys[0] is None:
        return carry, None
    return carry, _stack_trees(ys)


def _fori_loop(lo, hi, body, init, **_):
    v = init
    for i in range(int(lo), int(hi)):
        v = body(i, v)
    return v


def _while_loop(cond, body, init):
    v = init
    while bool(cond(v)):
        v = body(v)
    return v


def _cond(pred, tf, ff, *ops):
    return tf(*ops) if bool(pred) else ff(*ops)


def _switch(i, branches, *ops):
    return branches[int(np.clip(int(i), 0, len(branches) - 1))](*ops)


def _lax_pad(x, value, config):
    x = np.asarray(x)
    out = x
    for ax, (lo, hi, interior) in enumerate(config):
        if interior:
            raise NotImplementedError("interior padding")
        if lo < 0:
            out = np.take(out, np.arange(-lo, out.shape[ax]), axis=ax)
            lo = 0
        if hi < 0:
            out = np.take(out, np.arange(0, out.shape[ax] + hi), axis=ax)
            hi = 0
        w = [(0, 0)] * out.ndim
        w[ax] = (lo, hi)
        out = np.pad(out, w, constant_values=value)
    return _wrap(out)


def _dynamic_slice_in_dim(x, start, size, axis=0):
    x = np.asarray(x)
    s = int(np.clip(int(start), 0, x.shape[axis] - size))
    return _wrap(np.take(x, np.arange(s, s + size), axis=axis))


def _dynamic_update_slice_in_dim(x, upd, start, axis):
    x = np.array(x)
    upd = np.asarray(upd)
    s = int(np.clip(int(start), 0, x.shape[axis] - upd.shape[axis]))
    sl = [slice(None)] * x.ndim
    sl[axis] = slice(s, s + upd.shape[axis])
    x[tuple(sl)] = upd
    return _wrap(x)


def _segment(op, init_fn, data, segment_ids, num_segments, **_):
    data = np.asarray(data)
    ids = np.asarray(segment_ids).astype(np.int64)
    out = np.full((num_segments,) + data.shape[1:], init_fn(data.dtype), data.dtype)
    ok = (ids >= 0) & (ids < num_segments)
    op.at(out, ids[ok], data[ok])
    return _wrap(out)


def _segment_sum(data, segment_ids, num_segments=None, **k):
    return _segment(np.add, lambda dt: 0, data, segment_ids, num_segments, **k)


def _segment_max(data, segment_ids, num_segments=None, **k):
    def lowest(dt):
        return -np.inf if np.issubdtype(dt, np.inexact) else np.iinfo(dt).min
    return _segment(np.maximum, lowest, data, segment_ids, num_segments, **k)


# ---------------------------------------------------------------------------
# jax.numpy


def _wrapped(fn):
    @functools.wraps(fn)
    def g(*a, **k):
        for drop in ("precision", "preferred_element_type", "_dot_general", "out_sharding"):
            k.pop(drop, None)
        return _wrap(fn(*a, **k))
    return g


def _asarray(a, dtype=None, copy=None, **_):
    if isinstance(a, (list, tuple)):
        a = np.asarray([np.asarray(v) for v in a]) if any(isinstance(v, np.ndarray) for v in a) else np.asarray(a)
    x = np.asarray(a)
    if dtype is not None:
        x = _convert(x, dtype)
    elif x.dtype == np.float16 or x.dtype == object:
        raise TypeError(f"unsupported dtype {x.dtype}")
    return _wrap(np.array(x) if copy else x)


def _argsort(a, axis=-1, kind=None, order=None, stable=True, descending=False):
    a = np.asarray(a)
    if descending:
        return _wrap(np.flip(np.argsort(np.flip(a, axis), axis=axis, kind="stable"), axis) * -1
                     + (a.shape[axis] - 1))
    return _wrap(np.argsort(a, axis=axis, kind="stable"))


def _sort(a, axis=-1, kind=None, order=None, stable=True, descending=False):
    r = np.sort(np.asarray(a), axis=axis, kind="stable")
    return _wrap(np.flip(r, axis) if descending else r)


def _take(a, indices, axis=None, mode=None, fill_value=None, **_):
    a = np.asarray(a)
    if axis is None:
        a, axis = a.ravel(), 0
    idx = np.asarray(indices).astype(np.int64)
    n = a.shape[axis]
    idx = np.where(idx < 0, idx + n, idx)
    if mode in ("clip", "wrap"):
        return _wrap(np.take(a, idx, axis=axis, mode=mode))
    bad = (idx < 0) | (idx >= n)
    r = np.take(a, np.where(bad, 0, idx), axis=axis)
    if bad.any():
        fill = fill_value if fill_value is not None else (np.nan if np.issubdtype(a.dtype, np.inexact) else np.iinfo(a.dtype).min)
        shape = [1] * r.ndim
        shape[axis:axis + bad.ndim] = bad.shape
        r = np.where(bad.reshape(shape), fill, r)
    return _wrap(r)


def _take_along_axis(arr, indices, axis, mode=None, fill_value=None):
    arr = np.asarray(arr)
    idx = np.asarray(indices).astype(np.int64)
    n = arr.shape[axis]
    idx = np.where(idx < 0, idx + n, idx)
    bad = (idx < 0) | (idx >= n)
    r = np.take_along_axis(arr, np.where(bad, 0, idx), axis=axis)
    if bad.any():
        fill = fill_value if fill_value is not None else (np.nan if np.issubdtype(arr.dtype, np.inexact) else np.iinfo(arr.dtype).min)
        r = np.where(bad, fill, r)
    return _wrap(r)


def _unique(ar, return_index=False, return_inverse=False, return_counts=False, axis=None,
            size=None, fill_value=None, **_):
    res = np.unique(np.asarray(ar), return_index=return_index, return_inverse=return_inverse,
                    return_counts=return_counts, axis=axis)
    if size is not None:
        raise NotImplementedError("jnp.unique(size=...)")
    return _wrap(res)


def _nonzero(a, size=None, fill_value=None):
    res = np.nonzero(np.asarray(a))
    if size is not None:
        fv = 0 if fill_value is None else fill_value
        res = tuple(np.concatenate([r[:size], np.full(max(size - len(r), 0), fv, r.dtype)]) for r in res)
    return _wrap(res)


def _where(cond, x=None, y=None, size=None, fill_value=None):
    if x is None and y is None:
        return _nonzero(cond, size=size, fill_value=fill_value)
    return _wrap(np.where(cond, x, y))


def _cumsum(a, axis=None, dtype=None, **_):
    a = np.asarray(a)
    if dtype is None and a.dtype == np.bool_:
        dtype = np.int64
    return _wrap(np.cumsum(a, axis=axis, dtype=dtype))



def _bincount(x, weights=None, minlength=0, *, length=None):
    """jnp.bincount: with ``length`` the output has exactly that many bins and values
    at or above it are dropped (the jit-static form); without it, NumPy's."""
    x = np.asarray(x).astype(np.int64)
    w = None if weights is None else np.asarray(weights)
    if length is None:
        return _wrap(np.bincount(x, weights=w, minlength=minlength))
    keep = (x >= 0) & (x < length)
    return _wrap(np.bincount(x[keep], weights=None if w is None else w[keep], minlength=length)[:length])


def _searchsorted(a, v, side="left", sorter=None, method=None):
    return _wrap(np.searchsorted(np.asarray(a), np.asarray(v), side=side, sorter=sorter))


class _NumpyModule(types.ModuleType):
    _special = {
        "searchsorted": _searchsorted,
        "asarray": _asarray, "array": _asarray, "argsort": _argsort, "sort": _sort,
        "take": _take, "take_along_axis": _take_along_axis, "unique": _unique,
        "nonzero": _nonzero, "where": _where, "cumsum": _cumsum, "bincount": _bincount,
        "ndarray": np.ndarray,
    }

    def __getattr__(self, name):
        if name in self._special:
            return self._special[name]
        obj = getattr(np, name)
        if isinstance(obj, type) and issubclass(obj, np.generic):
            return obj
        if callable(obj) and not isinstance(obj, type):
            return _wrapped(obj)
        return obj


class _SubModule(types.ModuleType):
    def __init__(self, name, src):
        super().__init__(name)
        self._src = src

    def __getattr__(self, name):
        obj = getattr(self._src, name)
        return _wrapped(obj) if callable(obj) and not isinstance(obj, type) else obj


class _Device:
    platform = "cpu"
    device_kind = "cpu"
    id = 0

    def memory_stats(self):
        return None


class _Config:
    jax_enable_x64 = True

    def update(self, *_a, **_k):
        return None

    def __getattr__(self, name):
        return None


class _Precision:
    HIGHEST = "highest"
    HIGH = "high"
    DEFAULT = "default"


def install():
    """Register `jax`, `jax.numpy`, `jax.lax`, ... in `sys.modules`."""
    import scipy.special

    jax = types.ModuleType("jax")
    jax.__version__ = "0.4.38 (NumPy stand-in)"
    jax.__path__ = []
    jnp = _NumpyModule("jax.numpy")
    jnp.linalg = _SubModule("jax.numpy.linalg", np.linalg)
    jnp.fft = _SubModule("jax.numpy.fft", np.fft)
    lax = types.ModuleType("jax.lax")
    lax.map = _lax_map
    lax.scan = _scan
    lax.fori_loop = _fori_loop
    lax.while_loop = _while_loop
    lax.cond = _cond
    lax.switch = _switch
    lax.pad = _lax_pad
    lax.select = lambda p, a, b: _wrap(np.where(p, a, b))
    lax.stop_gradient = lambda x: x
    lax.optimization_barrier = lambda x: x
    lax.dynamic_slice_in_dim = _dynamic_slice_in_dim
    lax.dynamic_update_slice_in_dim = _dynamic_update_slice_in_dim
    lax.complex = lambda a, b: _wrap(np.asarray(a) + 1j * np.asarray(b))
    lax.Precision = _Precision
    ops = types.ModuleType("jax.ops")
    ops.segment_sum = _segment_sum
    ops.segment_max = _segment_max
    tu = types.ModuleType("jax.tree_util")
    tu.tree_map = tree_map
    tu.tree_leaves = tree_leaves
    tu.tree_flatten = tree_flatten
    tu.tree_unflatten = tree_unflatten
    tu.register_pytree_node = lambda *a, **k: None
    tu.register_pytree_node_class = lambda c: c
    jsp = types.ModuleType("jax.scipy")
    jsp.special = _SubModule("jax.scipy.special", scipy.special)
    jsp.linalg = _SubModule("jax.scipy.linalg", __import__("scipy.linalg").linalg)
    nn = types.ModuleType("jax.nn")
    nn.relu = lambda x: _wrap(np.maximum(x, 0))
    exp = types.ModuleType("jax.experimental")
    exp.__path__ = []

    jax.numpy, jax.lax, jax.ops, jax.tree_util = jnp, lax, ops, tu
    jax.scipy, jax.nn, jax.experimental = jsp, nn, exp
    jax.jit, jax.checkpoint, jax.remat, jax.custom_vjp, jax.vmap = jit, checkpoint, remat, custom_vjp, vmap
    jax.config = _Config()
    jax.Array = np.ndarray
    jax.devices = lambda *a, **k: [_Device()]
    jax.default_backend = lambda: "cpu"
    jax.device_put = lambda x, *a, **k: _wrap(np.asarray(x)) if isinstance(x, (np.ndarray, list)) else x
    jax.block_until_ready = lambda x: x
    jax.clear_caches = lambda: None
    jax.ensure_compile_time_eval = lambda: __import__("contextlib").nullcontext()
    for name in ("grad", "value_and_grad", "vjp", "jvp", "jacobian", "linear_transpose", "eval_shape"):
        setattr(jax, name, _unsupported(name))
    jax.tree_map = tree_map
    for modname, mod in (("jax", jax), ("jax.numpy", jnp), ("jax.numpy.linalg", jnp.linalg),
                         ("jax.lax", lax), ("jax.ops", ops), ("jax.tree_util", tu),
                         ("jax.scipy", jsp), ("jax.scipy.special", jsp.special),
                         ("jax.scipy.linalg", jsp.linalg), ("jax.nn", nn),
                         ("jax.experimental", exp)):
        sys.modules[modname] = mod
    return jax
