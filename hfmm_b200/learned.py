"""Learned expansion order and leaf size, certified against a sampled direct sum.

The reference takes ``p`` and ``N_max`` from the caller (HFMM.py:55-80) and
never checks the result. Here a 3 x 64 FP32 network (the CUDA kernels of
``csrc/mlp.cu``) reads features of the problem's tree and predicts

* output 0: the smallest expansion order ``p`` (surface points per cube edge)
  whose evaluate meets the requested tolerance, as a real number;
* output 1: log2 of the fastest leaf size ``N_max`` (automatic depth), used as 64
  or 128 (``OrderNet.choose_from``).

The mixed-precision plans also get a low-rank M2L (``hfmm_b200.compress``) at a
tenth of the tolerance.

Features (``features``) are: log10(tol), k times the domain extent, log2 N,
the depth, k times the box size at levels 2..7 (0 where the tree is shallower),
the fraction of boxes on levels 2..7, and an 8-bin histogram of leaf occupancy
relative to ``N_max`` -- all from the tree that ``hfmm_tree_build`` makes, so
no operator table is built before ``p`` is known.

``AutoPlan`` is the certified front door (the design precedent is the
reference's Laplace-only tune.AutoEvaluator, jaxfmm/tune.py:375-516): every
evaluate checks ``n_check`` random targets against the FP64 direct sum on the
GPU (the referee of test.py:11-18) and, when the relative L2 error of the
potential misses the tolerance, reruns with the plain conservative order in
FP64, stepping ``p`` up by 2 while the check still fails.
"""
import math
import os

import numpy as np
import torch

from . import _lib
from ._lib import check as _check

N_FEATURES = 24
N_OUTPUTS = 2
P_MIN, P_MAX = 4, 16
LEAVES = (16, 32, 64, 128)
FEATURE_LEAF = 64          # the tree the features are read from
TOL_MIXED = 1e-6           # the mixed-precision path is used at tolerances >= this
TOL_LEARNED = 3e-7         # below this the network is not consulted (outside its training range)
KD_TRAINED = 50.0          # largest k x domain extent of the committed training sweep
KD_TRUSTED = 1.5 * KD_TRAINED   # beyond this the network is not consulted either
DEFAULT_WEIGHTS = os.path.join(os.path.dirname(__file__), "data", "order_net.npz")


def conservative_p(tol):
    """The plain order: two surface points per edge for each decade of tolerance,
    clamped to [4, 16] (1e-6 -> 12, the order of the plain path's 1M-point config)."""
    return int(min(P_MAX, max(P_MIN, math.ceil(-2.0 * math.log10(tol)))))


def network_applies(feats, tol):
    """Whether the network's order may be used for these features: the tolerance is
    in its training range and k x extent at most 1.5 times the largest one it saw
    (50 in the sweep). Measured with an earlier network trained up to 24: at 44 (8M
    clustered points, k = 40) its p = 9 missed 1e-6 and every step fell back to the
    plain FP64 rerun, which is what the guard is for."""
    return tol >= TOL_LEARNED and float(feats[1]) <= KD_TRUSTED


def precision_for(tol, p):
    from . import PREC_FP64, PREC_MIXED
    return PREC_MIXED if (tol >= TOL_MIXED and p >= 5) else PREC_FP64


def compress_for(tol, precision):
    """Low-rank M2L tolerance of the mixed path: a tenth of the requested tolerance,
    at most 1e-7; None for the FP64 path. Measured on 1M points at p = 8: the dense
    mixed M2L gives 4.5e-7 / 6.9e-7 (potential / field), eps 1e-8 gives 5.5e-7 /
    6.9e-7 and eps 1e-7 5.3e-7 / 7.1e-7 (its truncation stays under the TF32
    rounding), with the evaluate at 76, 47 and 43.5 ms."""
    from . import PREC_MIXED
    return min(1e-7, 1e-1 * tol) if precision == PREC_MIXED else None


def tree_features(tree, info, k, tol, n_max=FEATURE_LEAF):
    """Feature vector (float32, N_FEATURES) from exported tree arrays and plan info."""
    lv = np.asarray(tree["lvls"])
    cnt = np.asarray(tree["counts"])
    leaf = np.asarray(tree["is_leaf"]).astype(bool)
    md = int(info["max_depth"])
    D = float(info["domain_extent"])
    n = int(cnt[lv == 0].sum()) if np.any(lv == 0) else int(cnt[leaf].sum())
    f = np.zeros(N_FEATURES, np.float64)
    f[0] = math.log10(tol)
    f[1] = k * D
    f[2] = math.log2(max(n, 1))
    f[3] = md
    for j, l in enumerate(range(2, 8)):
        if l <= md:
            f[4 + j] = k * D * 0.5 ** (l + 1)
        f[10 + j] = np.count_nonzero(lv == l) / max(len(lv), 1)
    occ = cnt[leaf & (cnt > 0)] / float(n_max)
    if occ.size:
        h = np.histogram(np.minimum(occ, 0.999999), bins=8, range=(0.0, 1.0))[0]
        f[16:24] = h / occ.size
    return f.astype(np.float32)


def features_for(positions, k, tol, device=None):
    """Build the feature tree for ``positions`` on the GPU and return its features."""
    from . import _validate_setup, _device, HFMMState
    x, kf = _validate_setup(positions, k, 4, FEATURE_LEAF, None)
    dev = _device(device)
    with torch.cuda.device(dev):
        pos = torch.as_tensor(x, dtype=torch.float64).to(dev).contiguous()
        h = _lib.ctypes.c_void_p()
        _check(_lib.lib.hfmm_tree_build(pos.data_ptr(), pos.shape[0], FEATURE_LEAF, 0,
                                        _lib.ctypes.byref(h)))
        st = HFMMState(h.value, pos, kf, 4, FEATURE_LEAF, dev)
        try:
            return tree_features(st.tree(), st.info, kf, tol)
        finally:
            st.close()


def label_p(ps, errs, tol):
    """Smallest (fractional) p from which every swept order meets ``tol``.

    ``errs[i]`` is the error at ``ps[i]`` (ascending); NaN marks an order the sweep
    did not run (merged sweeps cover different orders) and is left out, inf an order
    that does not apply (the mixed path below p = 5). Between the last miss and the
    first hit the crossing is interpolated linearly in log10(error); when no order
    meets ``tol`` the label is one above the largest order run.
    """
    ps = np.asarray(ps, np.float64)
    e = np.asarray(errs, np.float64)
    run = ~np.isnan(e)
    ps, e = ps[run], e[run]
    ok = np.isfinite(e) & (e <= tol)
    if not ok[-1]:
        return float(ps[-1] + 1)
    i = len(ok) - 1
    while i > 0 and ok[i - 1]:
        i -= 1
    if i == 0:
        return float(ps[0])
    if not np.isfinite(e[i - 1]):         # the order below was not run (no crossing to read)
        return float(ps[i])
    la, lb, lt = math.log10(max(e[i - 1], 1e-300)), math.log10(max(e[i], 1e-300)), math.log10(tol)
    t = (la - lt) / (la - lb) if la != lb else 1.0
    return float(ps[i - 1] + min(max(t, 0.0), 1.0) * (ps[i] - ps[i - 1]))


class OrderNet:
    """The 3 x 64 network with its feature normalisation, on one GPU.

    ``params`` is the flat FP32 parameter vector (layout of hfmm_mlp_param_count);
    ``mu``/``sd`` normalise the features, ``t_mu``/``t_sd`` the targets.
    """

    def __init__(self, params, mu, sd, t_mu, t_sd, device=None):
        from . import _device
        self.device = _device(device)
        n = _lib.lib.hfmm_mlp_param_count(N_FEATURES, N_OUTPUTS)
        _check(min(n, 0))
        if len(params) != n:
            raise ValueError(f"expected {n} parameters, got {len(params)}")
        self.params = torch.as_tensor(np.asarray(params, np.float32)).to(self.device)
        self.mu = np.asarray(mu, np.float32)
        self.sd = np.asarray(sd, np.float32)
        self.t_mu = np.asarray(t_mu, np.float32)
        self.t_sd = np.asarray(t_sd, np.float32)
        self.m = torch.zeros_like(self.params)
        self.v = torch.zeros_like(self.params)
        self.step = 0

    @classmethod
    def init(cls, X, T, seed=0, device=None):
        """Fresh network (Glorot-uniform weights, zero biases) normalised to the data."""
        rng = np.random.default_rng(seed)
        parts = []
        for fan_in, fan_out in ((N_FEATURES, 64), (64, 64), (64, 64), (64, N_OUTPUTS)):
            lim = math.sqrt(6.0 / (fan_in + fan_out))
            parts += [rng.uniform(-lim, lim, fan_in * fan_out), np.zeros(fan_out)]
        X = np.asarray(X, np.float64)
        T = np.asarray(T, np.float64).reshape(len(X), N_OUTPUTS)
        sd = X.std(0)
        sd[sd < 1e-6] = 1.0
        tsd = T.std(0)
        tsd[tsd < 1e-6] = 1.0
        return cls(np.concatenate(parts), X.mean(0), sd, T.mean(0), tsd, device)

    @classmethod
    def load(cls, path=DEFAULT_WEIGHTS, device=None):
        z = np.load(path)
        return cls(z["params"], z["mu"], z["sd"], z["t_mu"], z["t_sd"], device)

    def save(self, path, **extra):
        np.savez(path, params=self.params.cpu().numpy(), mu=self.mu, sd=self.sd, t_mu=self.t_mu,
                 t_sd=self.t_sd, **extra)

    def _x(self, X):
        X = (np.asarray(X, np.float32).reshape(-1, N_FEATURES) - self.mu) / self.sd
        return torch.as_tensor(np.ascontiguousarray(X, np.float32)).to(self.device)

    def _t(self, T):
        T = (np.asarray(T, np.float32).reshape(-1, N_OUTPUTS) - self.t_mu) / self.t_sd
        return torch.as_tensor(np.ascontiguousarray(T, np.float32)).to(self.device)

    def predict(self, X):
        """(n, 2) outputs in target units: fractional p and log2 of the leaf size."""
        x = self._x(X)
        y = torch.empty((x.shape[0], N_OUTPUTS), dtype=torch.float32, device=self.device)
        s = torch.cuda.current_stream(self.device)
        with torch.cuda.device(self.device):
            _check(_lib.lib.hfmm_mlp_forward(self.params.data_ptr(), x.data_ptr(), x.shape[0],
                                             N_FEATURES, N_OUTPUTS, y.data_ptr(), s.cuda_stream))
        return y.cpu().numpy() * self.t_sd + self.t_mu

    def train(self, X, T, steps, lr=1e-3):
        """Full-batch Adam on the GPU; returns the normalised loss after the last step."""
        x, t = self._x(X), self._t(T)
        loss = _lib.ctypes.c_double()
        s = torch.cuda.current_stream(self.device)
        with torch.cuda.device(self.device):
            _check(_lib.lib.hfmm_mlp_train(self.params.data_ptr(), self.m.data_ptr(),
                                           self.v.data_ptr(), self.step, x.data_ptr(),
                                           t.data_ptr(), x.shape[0], N_FEATURES, N_OUTPUTS,
                                           int(steps), float(lr), _lib.ctypes.byref(loss),
                                           s.cuda_stream))
        self.step += int(steps)
        return loss.value

    def choose(self, feats, margin=0.5):
        """(p, N_max) for one feature vector: p rounded up after adding ``margin``."""
        return self.choose_from(self.predict(feats)[0], margin)

    @staticmethod
    def choose_from(y, margin=0.5):
        """(p, N_max) from one output row (fractional p, log2 leaf size).

        The leaf size is kept to 64 or 128: p is predicted from the tree at leaf 64,
        and a smaller leaf can deepen the tree beyond what that prediction saw (on a
        1M-point cloud, outside the sweep's sizes, leaf 16 gave a depth-6 tree whose
        mixed evaluate missed 1e-6 at the predicted p)."""
        p = int(min(P_MAX, max(P_MIN, math.ceil(float(y[0]) + margin))))
        leaf = int(2 ** min(7, max(6, round(float(y[1])))))
        return p, leaf


def _rel_l2(a, b):
    a = np.asarray(a).reshape(len(b), -1)
    b = np.asarray(b).reshape(len(b), -1)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


class AutoPlan:
    """Certified evaluate at a requested tolerance (one-knob front door).

    ``net``: an OrderNet, None for the bundled weights, or False for the
    conservative order in place of the network's (the ablation: the same
    precision rule, leaf size and certification, only the network removed). ``n_check`` random
    targets (seeded) are compared against the FP64 direct sum on every evaluate.
    When the network's order misses the tolerance, the plan steps its order up (in
    mixed precision while it applies, up to the conservative order) and keeps the
    order that certified; past that the plain FP64 rerun decides. After a call,
    ``report`` holds the order, leaf, precision, measured error, the steps raised and
    whether the plain rerun was taken.
    """

    def __init__(self, positions, k, tol=1e-6, net=None, n_check=256, seed=0, device=None,
                 margin=0.5):
        from . import setup, _device
        if not (0 < tol < 1):
            raise ValueError("tol must be in (0, 1)")
        self.tol = float(tol)
        self.k = float(k)
        self.device = _device(device)
        self.positions = positions
        self.p_plain = conservative_p(self.tol)
        self.p, self.leaf, self.feats = self.p_plain, FEATURE_LEAF, None
        self.network_used = False
        if net is not False and self.tol >= TOL_LEARNED:
            self.feats = features_for(positions, k, tol, self.device)
            if network_applies(self.feats, self.tol):
                net = OrderNet.load(device=self.device) if net is None else net
                self.p, self.leaf = net.choose(self.feats, margin)
                self.network_used = True
        self.p_network = self.p if self.network_used else None
        self.precision = precision_for(self.tol, self.p)
        self.m2l_compress = compress_for(self.tol, self.precision)
        self.state = setup(positions, k, p=self.p, N_max=self.leaf, device=self.device,
                           m2l_compress=self.m2l_compress)
        rng = np.random.default_rng(seed)
        n = self.state.n
        self.check_idx = np.sort(rng.choice(n, size=min(n_check, n), replace=False)).astype(np.int32)
        self._check_dev = torch.as_tensor(self.check_idx).to(self.device)
        self._plain = {}
        self._pin = {}
        self._side = None
        self.report = {}

    def _direct(self, q_re, q_im, field):
        """FP64 direct sum at the check targets (hfmm_direct_async into buffers kept by
        the plan), on a side stream so that it overlaps the evaluate: it needs only
        the charges. Device tensors."""
        dev = self.device
        main = torch.cuda.current_stream(dev)
        m, n = self._check_dev.shape[0], self.state.n
        if self._side is None:
            self._side = torch.cuda.Stream(device=dev)
            nbytes = int(_lib.lib.hfmm_direct_scratch_bytes(n, m))
            _check(min(nbytes, 0))
            self._scratch = torch.empty(nbytes // 8, dtype=torch.float64, device=dev)
            self._ref_phi = torch.empty(m, dtype=torch.complex128, device=dev)
            self._ref_E = torch.empty((m, 3), dtype=torch.complex128, device=dev)
            self._derr = torch.zeros(1, dtype=torch.int32, device=dev)
        self._side.wait_stream(main)           # the charges are ready on the main stream
        _check(_lib.lib.hfmm_direct_async(
            self.state.positions.data_ptr(), q_re.data_ptr(),
            None if q_im is None else q_im.data_ptr(), n, self._check_dev.data_ptr(), m, self.k,
            self._ref_phi.data_ptr(), self._ref_E.data_ptr() if field else None,
            self._scratch.data_ptr(), self._scratch.numel() * 8, self._derr.data_ptr(),
            self._side.cuda_stream))
        for t in (q_re, q_im):
            if t is not None:
                t.record_stream(self._side)
        return self._ref_phi, (self._ref_E if field else None)

    def _error_async(self, phi, E, ref):
        """The relative L2 error at the check targets (potential, and field when
        computed) as a device scalar, enqueued behind the side stream's direct sum:
        nothing waits on the host, so the GPU runs it right after the evaluate."""
        torch.cuda.current_stream(self.device).wait_stream(self._side)
        if getattr(self, "_check_long", None) is None:
            self._check_long = self._check_dev.long()
        i = self._check_long
        rel = lambda a, b: torch.linalg.norm(a - b) / torch.clamp(torch.linalg.norm(b), min=1e-300)
        err = rel(phi[i], ref[0])
        if E is not None:
            err = torch.maximum(err, rel(E[i], ref[1]))
        return err

    def _error_value(self, err):
        if int(self._derr.item()):
            raise RuntimeError("direct-sum check: a target index is out of range")
        return float(err.item())

    def _error(self, phi, E, ref):
        """Relative L2 error at the check targets; waits for the side stream."""
        return self._error_value(self._error_async(phi, E, ref))

    def _raise_order(self, p):
        """Rebuild the plan at order ``p`` (same leaf size, the precision rule of p)."""
        from . import setup
        self.state.close()
        self.p = int(p)
        self.precision = precision_for(self.tol, self.p)
        self.m2l_compress = compress_for(self.tol, self.precision)
        self.state = setup(self.positions, self.k, p=self.p, N_max=self.leaf, device=self.device,
                           m2l_compress=self.m2l_compress)

    def _plain_state(self, p):
        from . import setup
        if p not in self._plain:
            self._plain[p] = setup(self.positions, self.k, p=p, N_max=FEATURE_LEAF,
                                   device=self.device)
        return self._plain[p]

    def evaluate_field(self, charges, field=True):
        """Certified (phi, E) (E is None with field=False); complex or real charges (N,).

        The error checked is the relative L2 error over the check targets of the
        potential, and of the field when it is computed (the larger of the two)."""
        from . import evaluate_into, check_errors, PREC_FP64, _stage_charges, _to_host
        numpy_in = not isinstance(charges, torch.Tensor)
        dev = self.device
        with torch.cuda.device(dev):
            if numpy_in:
                qn = np.asarray(charges)
                if qn.shape != (self.state.n,):
                    raise ValueError(f"charges must have shape ({self.state.n},)")
                q = _stage_charges(self, qn, np.iscomplexobj(qn), dev)
            else:
                if tuple(charges.shape) != (self.state.n,):
                    raise ValueError(f"charges must have shape ({self.state.n},)")
                q = charges.to(dev)
            if q.is_complex():
                q_re, q_im = q.real.double().contiguous(), q.imag.double().contiguous()
            else:
                q_re, q_im = q.double().contiguous(), None
            n = self.state.n
            phi = torch.empty(n, dtype=torch.complex128, device=dev)
            E = torch.empty((n, 3), dtype=torch.complex128, device=dev) if field else None
            ref = self._direct(q_re, q_im, field)
            evaluate_into(self.state, q_re, q_im, phi, E, self.precision)
            err_t = self._error_async(phi, E, ref)   # enqueued before the first host wait
            check_errors(self.state)
            err = self._error_value(err_t)
            rep = dict(p=self.p, leaf=self.leaf, precision=int(self.precision), error=err,
                       fallback=False, p_final=self.p, network=self.network_used, raised=0)
            # a miss at the network's order: the next orders in the plan's own precision
            # first (up to the conservative one); the plan keeps the order that certified,
            # so later evaluates start there (the network's p stays in p_network)
            while err > self.tol and self.network_used and self.p < self.p_plain:
                self._raise_order(self.p + 1)
                evaluate_into(self.state, q_re, q_im, phi, E, self.precision)
                check_errors(self.state)
                err = self._error(phi, E, ref)
                rep.update(p_final=self.p, error=err, precision=int(self.precision),
                           raised=rep["raised"] + 1)
            p = self.p_plain
            while err > self.tol and p <= P_MAX:
                st = self._plain_state(p)
                evaluate_into(st, q_re, q_im, phi, E, PREC_FP64)
                check_errors(st)
                err = self._error(phi, E, ref)
                rep.update(fallback=True, p_final=p, error=err, precision=int(PREC_FP64))
                p += 2
            rep["certified"] = bool(err <= self.tol)
            self.report = rep
        if numpy_in:
            php = _to_host(phi)
            Ep = _to_host(E) if E is not None else None
            torch.cuda.current_stream(dev).synchronize()
            return php.numpy(), (Ep.numpy() if E is not None else None)
        return phi, E

    def _pinned(self, name, shape, dtype):
        """A reused page-locked host buffer (the staging of NumPy charges)."""
        t = self._pin.get(name)
        if t is None or tuple(t.shape) != tuple(shape) or t.dtype != dtype:
            t = torch.empty(tuple(shape), dtype=dtype, pin_memory=True)
            self._pin[name] = t
        return t

    def evaluate(self, charges):
        return self.evaluate_field(charges, field=False)[0]

    def close(self):
        self.state.close()
        for st in self._plain.values():
            st.close()
        self._plain.clear()
