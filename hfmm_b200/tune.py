"""Leaf-size autotuner with a wisdom store: the reference's ``tune_kifmm``
(jaxfmm/tune.py:123-172) with its probe (``_probe``, :69-120) and wisdom key
(``_wisdom_key``, :44-48).

``tune_leaf(positions, k, charges, p)`` builds one plan per candidate leaf size
(``N_max`` in 32, 64, 128 by default). It times a warm evaluate on the device (CUDA
events, the faster of two calls) and measures its relative error against the FP64
direct sum on sampled targets. The winner is the fastest candidate whose error stays
within ``rel_slack`` of the anchor's: the ``N_max = 64`` candidate's error (the
reference's default), or the smallest error seen when that candidate is absent or
failed. A candidate that cannot be built or evaluated (out of memory, a refused
size) is skipped. Results are kept in a JSON wisdom file keyed by the problem class
(kernel, N rounded to a power of two, aspect-ratio bucket, p, precision, GPU name),
so a class is probed once per machine; ``force=True`` probes again.

The learned order (``hfmm_b200.learned``) picks p and the leaf size from the
problem's features without measuring; this is the measured alternative for a fixed
p, as in the reference.
"""
import json
import os

import numpy as np
import torch

__all__ = ["tune_leaf", "pick", "wisdom_key", "wisdom_path", "aspect"]

WISDOM_VERSION = 1


def wisdom_path():
    """$HFMM_B200_WISDOM, else ~/.cache/hfmm_b200/wisdom.json."""
    return os.environ.get("HFMM_B200_WISDOM") or os.path.join(
        os.path.expanduser("~"), ".cache", "hfmm_b200", "wisdom.json")


def aspect(positions):
    """Longest over shortest side of the bounding box."""
    ext = np.asarray(positions).max(0) - np.asarray(positions).min(0)
    return float(ext.max() / max(ext.min(), 1e-30))


def wisdom_key(kind, n, aspect_ratio, p, precision, device_name):
    """Problem class: N and the aspect ratio in powers of two (aspect clipped to
    [1, 2^10]), as the reference buckets them."""
    nb = int(np.round(np.log2(max(n, 1))))
    ab = int(np.clip(np.round(np.log2(max(aspect_ratio, 1.0))), 0, 10))
    return f"v{WISDOM_VERSION}|{kind}|N2^{nb}|A2^{ab}|p{p}|prec{precision}|{device_name.replace(' ', '_')}"


def pick(results, rel_slack, anchor=None):
    """The fastest (candidate, ms, rel) whose rel <= max(a rel_slack, a + 1e-16), a =
    the anchor candidate's rel if it is among the results, else the smallest rel."""
    if not results:
        raise RuntimeError("tune_leaf: every candidate failed")
    a = min(r for _, _, r in results)
    for c, _, r in results:
        if anchor is not None and c == anchor:
            a = r
            break
    ok = [x for x in results if x[2] <= max(a * rel_slack, a + 1e-16)]
    return min(ok, key=lambda x: x[1])


def _load(path):
    try:
        with open(path) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def _save(path, store):
    try:
        os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
        tmp = path + ".tmp"
        with open(tmp, "w") as f:
            json.dump(store, f, indent=1, sort_keys=True)
        os.replace(tmp, path)
    except OSError:
        pass   # the tuned plan is still returned; only the memory of it is lost


def _timed_evaluate(st, q, precision):
    """Warm evaluate of complex or real charges on the device: (ms of the faster of two
    timed calls, potential as NumPy)."""
    from . import evaluate_into, check_errors
    dev = st.device
    with torch.cuda.device(dev):
        qt = torch.as_tensor(q).to(dev)
        q_re = (qt.real if qt.is_complex() else qt).to(torch.float64).contiguous()
        q_im = qt.imag.to(torch.float64).contiguous() if qt.is_complex() else None
        phi = torch.empty(st.n, dtype=torch.complex128, device=dev)
        s = torch.cuda.current_stream(dev)
        evaluate_into(st, q_re, q_im, phi, None, precision)
        best = float("inf")
        for _ in range(2):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(s)
            evaluate_into(st, q_re, q_im, phi, None, precision)
            e1.record(s)
            e1.synchronize()
            best = min(best, e0.elapsed_time(e1))
        check_errors(st)
        return best, phi.cpu().numpy()


def tune_leaf(positions, k, charges, p=8, candidates=(32, 64, 128), rel_slack=1.5, n_ref=500,
              force=False, wisdom=None, precision=None, setup_kw=None, verbose=False):
    """Returns (params, state, report): the winning {"N_max", "ms", "rel"}, its plan
    (the caller closes it) and the probe report [(N_max, ms, rel) or (N_max, error)],
    or [("wisdom", params)] when the wisdom file already held the class."""
    from . import setup, direct, HFMMError, PREC_FP64
    pos = np.ascontiguousarray(positions, dtype=np.float64)
    if pos.ndim != 2 or pos.shape[1] != 3 or pos.shape[0] == 0:
        raise ValueError("positions: expected a nonempty (N, 3) array")
    q = np.asarray(charges)
    if q.shape != (pos.shape[0],):
        raise ValueError(f"charges must have shape ({pos.shape[0]},)")
    if not candidates:
        raise ValueError("candidates: at least one leaf size")
    precision = PREC_FP64 if precision is None else int(precision)
    setup_kw = dict(setup_kw or {})
    path = wisdom or wisdom_path()
    key = wisdom_key("helmholtz", pos.shape[0], aspect(pos), int(p), precision,
                     torch.cuda.get_device_name(setup_kw.get("device")))
    store = _load(path)
    if not force and key in store:
        params = store[key]
        return params, setup(pos, k, p=p, N_max=int(params["N_max"]), **setup_kw), [("wisdom", params)]
    idx = np.sort(np.random.default_rng(0).choice(pos.shape[0], min(n_ref, pos.shape[0]),
                                                  replace=False))
    ref, results, states, report = None, [], {}, []
    for nm in dict.fromkeys(int(c) for c in candidates):   # each leaf size once, in order
        st = None
        try:
            st = setup(pos, k, p=p, N_max=nm, **setup_kw)
            if ref is None:
                ref = direct(st, q, idx)
            ms, phi = _timed_evaluate(st, q, precision)
            rel = float(np.linalg.norm(phi[idx] - ref) / np.linalg.norm(ref))
            if not np.isfinite(rel):
                raise ValueError("non-finite error against the direct sum")
            results.append((nm, ms, rel))
            report.append((nm, ms, rel))
            states[nm] = st
            if verbose:
                print(f"tune_leaf: N_max {nm}: {ms:.2f} ms, rel {rel:.2e}", flush=True)
        except (ValueError, HFMMError, RuntimeError) as e:   # torch's OOM is a RuntimeError
            if st is not None:
                st.close()
            report.append((nm, f"{type(e).__name__}: {e}"))
            if verbose:
                print(f"tune_leaf: N_max {nm}: failed ({type(e).__name__})", flush=True)
    best = pick(results, rel_slack, anchor=64)   # raises when every candidate failed
    for nm, st in states.items():
        if nm != best[0]:
            st.close()
    params = {"N_max": best[0], "ms": best[1], "rel": best[2]}
    store[key] = params
    _save(path, store)
    return params, states[best[0]], report
