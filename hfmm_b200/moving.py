"""Moving geometry: certified evaluates of point clouds that move between calls.

Replaces, for the Helmholtz path, the reference's fully-jit moving-geometry KIFMM
(kifmm/fulljit.py:57-328: tree and lists rebuilt inside one compiled function
against frozen buffer caps, the realised counts certifying each call) and its
guarded driver (driver.py:64-640, ``kifmm_fulljit_driver``: reject and rebuild on
a violated certificate).

There the caps exist because JAX needs static shapes, and the operators are the
Laplace unit-scale set rescaled by box size. Here the device rebuilds the tree
and lists in place (``hfmm_plan_rebuild``) and its buffers follow the realised
sizes, so the certificate is about the operator tables instead: Helmholtz tables
depend on the absolute box size, so the plan is built in a fixed domain cube
(the reference geometry's bounding cube widened by ``headroom``) at a fixed depth,
and the tables stay valid for every geometry inside that cube. A call whose
points leave the cube is rejected before anything changes; the evaluator then
refits the cube around the new points and builds a new plan (new tables), up to
``max_attempts`` times per call. The realised counts (boxes, widest leaf, list
lengths) are reported per call beside the caps fitted at the last build, in the
reference's certificate vocabulary.
"""
import math

import numpy as np

from . import HFMMError, PREC_FP64, evaluate, evaluate_field, rebuild, setup

__all__ = ["MovingPlan", "fit_domain", "auto_depth"]

_CAP_KEYS = (("maxleaf", "pil_cap"), ("n_near", "dir_cap"), ("n_v", "v_cap"),
             ("n_w", "w_cap"), ("n_x", "x_cap"))


def fit_domain(positions, headroom):
    """The cube around ``positions`` (N, 3), widened by ``headroom`` on its side:
    ``(pmin (3,), extent)``."""
    x = np.asarray(positions, dtype=np.float64)
    lo, hi = x.min(0), x.max(0)
    ext = float((hi - lo).max())
    if not ext > 0:
        ext = 1.0
    ext *= 1.0 + float(headroom)
    return (lo + hi) / 2 - ext / 2, ext


def auto_depth(n, N_max):
    """The reference's automatic depth before refinement (trees/cubic.py:577-585)."""
    ratio = max(n / max(N_max, 1), 1.0)
    return max(2, int(math.ceil(math.log(ratio) / math.log(8.0))))


def _fit_cap(used, headroom):
    return int(math.ceil(max(used, 1) * (1.0 + headroom)))


class MovingPlan:
    """Certified moving-geometry evaluator: ``evaluate(positions, charges)``.

    positions: (N, 3) of the reference geometry (N stays fixed). k, p, N_max,
    max_depth (None: the automatic depth at N / N_max), precision and
    m2l_compress as in ``hfmm_b200.setup``. headroom: spare fraction of the
    domain cube's side and of every cap. Attributes: ``state`` (the current
    plan), ``builds`` (plans built, tables included), ``moves`` (in-place
    rebuilds), ``certificate`` (the last call's realised counts, caps and
    verdicts).
    """

    def __init__(self, positions, k, p=4, N_max=16, max_depth=None, headroom=0.15,
                 precision=PREC_FP64, m2l_compress=None, device=None, max_attempts=3):
        x = np.asarray(positions, dtype=np.float64)
        self.n = x.shape[0]
        self.k, self.p, self.N_max = float(k), int(p), int(N_max)
        self.depth = int(max_depth) if max_depth is not None else auto_depth(self.n, self.N_max)
        self.headroom = float(headroom)
        self.precision = precision
        self.m2l_compress = m2l_compress
        self.device = device
        self.max_attempts = int(max_attempts)
        self.state = None
        self.builds = 0
        self.moves = 0
        self.certificate = None
        self._build(x)

    def _build(self, x):
        if self.state is not None:
            self.state.close()
            self.state = None
        self.domain = fit_domain(x, self.headroom)
        self.state = setup(x, self.k, p=self.p, N_max=self.N_max, max_depth=self.depth,
                           device=self.device, m2l_compress=self.m2l_compress,
                           domain=self.domain)
        self.builds += 1
        info = self.state.info
        self.caps = {cap: _fit_cap(info[used], self.headroom) for used, cap in _CAP_KEYS}

    def inside(self, positions):
        """True when every point lies in the current plan's domain cube."""
        x = np.asarray(positions, dtype=np.float64)
        lo, ext = self.domain
        return bool(((x >= lo) & (x <= lo + ext)).all())

    def move(self, positions):
        """Rebuild the current plan for ``positions``; refit and rebuild the plan when
        they leave its domain. Returns the certificate of the geometry in use."""
        x = np.asarray(positions, dtype=np.float64)
        if x.shape != (self.n, 3):
            raise ValueError("positions must keep the shape (N, 3) of the reference geometry")
        rebuilt = 0
        for _ in range(self.max_attempts):
            try:
                rebuild(self.state, x)
                self.moves += 1
                break
            except HFMMError as e:
                if getattr(e, "code", None) != -4:
                    raise
                self._build(x)   # the points left the domain: new cube, new tables
                rebuilt += 1
                break
        else:
            raise RuntimeError("moving plan: no certified geometry after max_attempts")
        info = self.state.info
        used = {u: int(info[u]) for u, _ in _CAP_KEYS}
        within = all(used[u] <= self.caps[c] for u, c in _CAP_KEYS)
        if not within:   # grow-only refit of the caps (buffers already follow the tree)
            self.caps = {c: max(self.caps[c], _fit_cap(used[u], self.headroom))
                         for u, c in _CAP_KEYS}
        self.certificate = dict(inside_domain=True, plan_rebuilt=rebuilt > 0,
                                within_caps=within, counts=used, caps=dict(self.caps),
                                n_boxes=int(info["n_boxes"]), adaptive=bool(info["adaptive"]),
                                max_depth=int(info["max_depth"]))
        return self.certificate

    def evaluate(self, positions, charges):
        """HFMM.evaluate at the moved points (real charges)."""
        self.move(positions)
        return evaluate(self.state, charges, self.precision)

    def evaluate_field(self, positions, charges):
        """Potential and field at the moved points (real or complex charges)."""
        self.move(positions)
        return evaluate_field(self.state, charges, self.precision)

    def close(self):
        if self.state is not None:
            self.state.close()
            self.state = None
