"""Batched evaluate of many independent problems in one CUDA-graph launch.

No counterpart in the reference (one problem per ``HFMM.evaluate`` call,
HFMM.py:83-91). ``Batch`` binds finalized plans to the native batch runtime
(``hfmm_batch_*`` in include/hfmm_b200.h): the plans are spread over CUDA
streams by their work estimate, streaming plans share one M2L-table workspace
per stream, and the whole batch is captured into one graph.

``autotune`` measures the graph time for each candidate stream count and keeps
the fastest in a JSON "wisdom" file keyed by the batch's shape (the design
precedent is the reference's Laplace autotuner, jaxfmm/tune.py:123-172).

``AutoBatch`` is the certified front door for a list of (positions, k): the
expansion-order network picks each problem's p and leaf size from one batched
forward pass, the problems run as one graph, and each result is checked on
256 sampled targets against the FP64 direct sum, with a plain rerun of the
problems that miss.
"""
import hashlib
import json
import os

import numpy as np
import torch

from . import _lib
from ._lib import check as _check


class Batch:
    """Finalized plans evaluated together; ``bind`` sets the inputs and captures."""

    def __init__(self, states, n_streams=4, queue=True):
        """``queue``: run the problems' low-rank mixed M2L as one persistent kernel
        over a queue of all their work (hfmm_batch_set_queue) when they allow it."""
        if not states:
            raise ValueError("a batch needs at least one plan")
        self.states = list(states)
        self.n_streams = int(n_streams)
        self.queue = bool(queue)
        arr = (_lib.ctypes.c_void_p * len(states))(*[s.handle for s in states])
        h = _lib.ctypes.c_void_p()
        with torch.cuda.device(states[0].device):
            _check(_lib.lib.hfmm_batch_create(arr, len(states), self.n_streams,
                                              _lib.ctypes.byref(h)))
        self._h = h.value
        _check(_lib.lib.hfmm_batch_set_queue(self._h, int(bool(queue))))
        self.outputs = None

    def stream_of(self, i):
        r = _lib.lib.hfmm_batch_stream_of(self._h, i)
        _check(min(r, 0))
        return r

    def bind(self, charges, field=True, precision=None, checks=None):
        """Device charge tensors (complex128 or float64, one per plan); allocates the
        outputs, sets every problem and captures the graph. ``precision``: one value
        or one per problem (default mixed). ``checks``: None, or per problem a device
        int32 tensor of target indices checked in the graph against the FP64 direct
        sum (``check_sums`` then holds each problem's squared-norm sums)."""
        from . import PREC_MIXED
        if len(charges) != len(self.states):
            raise ValueError("one charge vector per plan")
        precs = precision if isinstance(precision, (list, tuple)) else \
            [PREC_MIXED if precision is None else precision] * len(self.states)
        self._keep, self.outputs, self._q_dev, self._stage = [], [], [], None
        for i, (st, q) in enumerate(zip(self.states, charges)):
            if tuple(q.shape) != (st.n,):
                raise ValueError(f"charges of problem {i} must have shape ({st.n},)")
            q = q.to(st.device)                 # the graph reads them through device pointers
            if q.is_complex():
                q_re, q_im = q.real.double().contiguous(), q.imag.double().contiguous()
            else:
                q_re, q_im = q.double().contiguous(), None
            phi = torch.empty(st.n, dtype=torch.complex128, device=st.device)
            E = torch.empty((st.n, 3), dtype=torch.complex128, device=st.device) if field else None
            _check(_lib.lib.hfmm_batch_set_problem(
                self._h, i, q_re.data_ptr(), None if q_im is None else q_im.data_ptr(),
                phi.data_ptr(), None if E is None else E.data_ptr(), int(precs[i])))
            self._keep.append((q_re, q_im))
            self._q_dev.append((q_re, q_im))
            self.outputs.append((phi, E))
        self.check_sums = None
        if checks is not None:
            dev = self.states[0].device
            self.check_sums = torch.zeros((len(self.states), 4), dtype=torch.float64, device=dev)
            for i, (st, tg) in enumerate(zip(self.states, checks)):
                tg = tg.to(device=dev, dtype=torch.int32).contiguous()
                if tg.ndim != 1 or (tg.numel() and (int(tg.min()) < 0 or int(tg.max()) >= st.n)):
                    raise ValueError(f"check targets of problem {i} must be indices in [0, {st.n})")
                self._keep.append((tg,))
                _check(_lib.lib.hfmm_batch_set_check(
                    self._h, i, st.positions.data_ptr(), tg.data_ptr(), tg.shape[0],
                    self.check_sums[i].data_ptr()))
        with torch.cuda.device(self.states[0].device):
            before = _lib.launch_count()
            _check(_lib.lib.hfmm_batch_capture(self._h))
            self.kernels_per_launch = _lib.launch_count() - before   # kernels in the graph
        self.queued = bool(_lib.lib.hfmm_batch_queued(self._h))
        self.queue_note = _lib.lib.hfmm_batch_queue_note(self._h).decode(errors="replace")
        return self.outputs

    def solve(self, charges):
        """One launch on new charges from the host, without re-capturing: ``charges``
        are NumPy arrays, one per problem with the bound shape (complex, or real where
        the problem was bound with real charges). They are copied through page-locked
        staging buffers (kept by the batch) into the device buffers the graph reads,
        the graph runs on the current stream, and each output comes back into a fresh
        page-locked host block. Returns [(phi, E or None), ...] as NumPy arrays."""
        from . import _to_host
        if self.outputs is None:
            raise RuntimeError("bind the batch before solve")
        if len(charges) != len(self.states):
            raise ValueError("one charge vector per plan")
        dev = self.states[0].device
        with torch.cuda.device(dev):
            s = torch.cuda.current_stream(dev)
            if self._stage is None:   # page-locked staging, one complex128 vector a problem
                self._stage = [(torch.empty(st.n, dtype=torch.complex128, pin_memory=True),
                                torch.empty(st.n, dtype=torch.complex128, device=dev))
                               for st in self.states]
            for i, (q, (q_re, q_im), (h, d)) in enumerate(zip(charges, self._q_dev, self._stage)):
                q = np.asarray(q)
                if q.shape != (self.states[i].n,):
                    raise ValueError(f"charges of problem {i} must have shape ({self.states[i].n},)")
                if q_im is None and np.iscomplexobj(q):
                    raise ValueError(f"problem {i} was bound with real charges")
                if q.dtype == np.complex128 and q.flags.c_contiguous and q.flags.writeable:
                    h.copy_(torch.from_numpy(q))   # torch's threaded host copy
                else:
                    h.numpy()[...] = q
                d.copy_(h, non_blocking=True)
                q_re.copy_(d.real)
                if q_im is not None:
                    q_im.copy_(d.imag)
            self.launch(s)
            out = [(_to_host(phi), None if E is None else _to_host(E)) for phi, E in self.outputs]
            s.synchronize()
        return [(a.numpy(), None if b is None else b.numpy()) for a, b in out]

    def launch(self, stream=None):
        s = stream if stream is not None else torch.cuda.current_stream(self.states[0].device)
        _check(_lib.lib.hfmm_batch_launch(self._h, s.cuda_stream))

    def check_errors(self):
        from . import check_errors
        for st in self.states:
            check_errors(st)

    def check_rel_errors(self):
        """Per problem (rel-L2 of phi, rel-L2 of E or 0) from the last launch's check."""
        s = self.check_sums.cpu().numpy()
        rel = lambda a, b: float(np.sqrt(a / b)) if b > 0 else 0.0
        return [(rel(r[0], r[1]), rel(r[2], r[3])) for r in s]

    def time_ms(self, reps=3, warmup=1):
        """Mean CUDA-event time of one graph launch."""
        s = torch.cuda.current_stream(self.states[0].device)
        for _ in range(warmup):
            self.launch(s)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(s)
        for _ in range(reps):
            self.launch(s)
        b.record(s)
        b.synchronize()
        return a.elapsed_time(b) / reps

    def close(self):
        if getattr(self, "_h", None) is not None:
            _lib.lib.hfmm_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def signature(states):
    """Key of a batch's shape for the wisdom file: sizes, orders and depths."""
    desc = sorted((s.n, s.p, s.max_depth, s.N_max, round(s.k, 6)) for s in states)
    dev = torch.cuda.get_device_name(states[0].device)
    return dev + ":" + hashlib.sha1(repr(desc).encode()).hexdigest()[:16]


def autotune(states, charges, candidates=(1, 2, 4, 8), wisdom=None, reps=3, field=True,
             precision=None, checks=None, queue_modes=(True, False)):
    """Pick the launch configuration with the lowest graph time: the stream count and
    whether the M2L runs as one queued persistent kernel or per plan on the streams.
    Returns (Batch, timings keyed "S,queue"). (The plans' leaf sizes are the learned
    order's choice, made per problem before this.)

    With ``wisdom`` (a JSON path) a previous result for the same signature is
    reused without measuring, and new measurements are stored there (the precedent is
    jaxfmm/tune.py:123-172's wisdom store)."""
    key = signature(states)
    store = {}
    if wisdom and os.path.exists(wisdom):
        with open(wisdom) as f:
            store = json.load(f)
    if key in store and "queue" in store[key]:
        b = Batch(states, store[key]["n_streams"], store[key]["queue"])
        b.bind(charges, field, precision, checks)
        return b, store[key]["ms"]
    times = {}
    for S in candidates:                 # a plan belongs to one batch at a time
        if S > len(states) and S != candidates[0]:
            continue
        for qm in queue_modes:
            b = Batch(states, S, qm)
            b.bind(charges, field, precision, checks)
            k = (S, bool(b.queued))      # the queue may not apply: then both modes are one
            if k not in times:
                times[k] = b.time_ms(reps)
            b.close()
    best = min(times, key=times.get)
    if wisdom:
        store[key] = {"n_streams": best[0], "queue": best[1],
                      "ms": {f"{k[0]},{int(k[1])}": v for k, v in times.items()}}
        tmp = wisdom + ".tmp"
        with open(tmp, "w") as f:
            json.dump(store, f, indent=1, sort_keys=True)
        os.replace(tmp, wisdom)
    b = Batch(states, best[0], best[1])
    b.bind(charges, field, precision, checks)
    return b, {f"{k[0]},{int(k[1])}": v for k, v in times.items()}


class AutoBatch:
    """Certified batched evaluate of problems [(positions, k), ...] at one tolerance.

    ``net``: an OrderNet, None for the bundled weights, or False for the
    conservative order (the ablation). Every problem's plan streams its dense M2L
    tables (only an FP64 evaluate would read them) and keeps the low-rank M2L of
    the mixed path, so the batch holds no dense M2L table at all.
    """

    def __init__(self, problems, tol=1e-6, net=None, n_streams=None, n_check=256, seed=0,
                 device=None, margin=0.5, wisdom=None):
        from . import setup, _device
        from .learned import (OrderNet, features_for, conservative_p, precision_for,
                              compress_for, network_applies, FEATURE_LEAF, TOL_LEARNED)
        self.tol = float(tol)
        self.device = _device(device)
        self.problems = problems
        if net is False or self.tol < TOL_LEARNED:
            choice = [(conservative_p(self.tol), FEATURE_LEAF)] * len(problems)
        else:
            net = OrderNet.load(device=self.device) if net is None else net
            feats = np.stack([features_for(x, k, self.tol, self.device) for x, k in problems])
            Y = net.predict(feats)
            plain = (conservative_p(self.tol), FEATURE_LEAF)
            choice = [net.choose_from(y, margin) if network_applies(f, self.tol) else plain
                      for f, y in zip(feats, Y)]
        self.choice = choice
        self.precisions = [precision_for(self.tol, p) for p, _ in choice]
        self.states = [setup(x, k, p=p, N_max=leaf, device=self.device, stream_tables=True,
                             m2l_compress=compress_for(self.tol, prec))
                       for (x, k), (p, leaf), prec in zip(problems, choice, self.precisions)]
        rng = np.random.default_rng(seed)
        self.checks = [torch.as_tensor(np.sort(rng.choice(st.n, min(n_check, st.n), replace=False))
                                       .astype(np.int32)).to(self.device) for st in self.states]
        self.n_streams = n_streams
        self.wisdom = wisdom
        self.batch = None
        self.report = []

    def bind(self, charges, field=True):
        qs = [torch.as_tensor(np.asarray(q)).to(self.device) if not isinstance(q, torch.Tensor)
              else q.to(self.device) for q in charges]
        self._q = qs
        self._field = field
        if self.n_streams is None:
            self.batch, self.tune_ms = autotune(self.states, qs, wisdom=self.wisdom, field=field,
                                                precision=self.precisions, checks=self.checks)
        else:
            self.batch = Batch(self.states, self.n_streams)
            self.batch.bind(qs, field, self.precisions, checks=self.checks)
        return self.batch.outputs

    def solve(self, charges):
        """The batched evaluate from the host: NumPy charges in (one array per problem),
        one graph launch, NumPy (phi, E) out, and each problem's checked relative
        errors (phi, E) from the launch's in-graph direct-sum check. Problems whose
        error misses the tolerance are not rerun here; ``certify`` does that."""
        outs = self.batch.solve(charges)
        return outs, self.batch.check_rel_errors()

    def raise_missed(self, field=None):
        """After a launch: every problem whose in-graph check missed the tolerance moves
        to the next order (same leaf size, the precision rule of that order, up to
        P_MAX), and the batch is captured again with the same stream count and queue
        setting. Returns the indices raised (empty: every problem certified)."""
        from . import setup
        from .learned import P_MAX, precision_for, compress_for
        field = self._field if field is None else field
        errs = self.batch.check_rel_errors()
        missed = [i for i, (a, b) in enumerate(errs)
                  if max(a, b if field else 0.0) > self.tol and self.choice[i][0] < P_MAX]
        if not missed:
            return []
        S, queue = self.batch.n_streams, self.batch.queue
        self.batch.close()
        for i in missed:
            p, leaf = self.choice[i]
            p += 1
            prec = precision_for(self.tol, p)
            x, k = self.problems[i]
            self.states[i].close()
            self.states[i] = setup(x, k, p=p, N_max=leaf, device=self.device, stream_tables=True,
                                   m2l_compress=compress_for(self.tol, prec))
            self.choice[i] = (p, leaf)
            self.precisions[i] = prec
        self.batch = Batch(self.states, S, queue)
        self.batch.bind(self._q, self._field, self.precisions, checks=self.checks)
        return missed

    def certify(self):
        """Read the in-graph check of the last launch (the direct sum at each problem's
        sampled targets ran inside the graph) and rerun the misses plainly (FP64,
        conservative order, stepping p by 2). Returns the per-problem reports."""
        from . import direct_at, evaluate_into, check_errors, setup, PREC_FP64
        from .learned import conservative_p, P_MAX, FEATURE_LEAF, _rel_l2
        self.batch.check_errors()
        errs = self.batch.check_rel_errors()
        rep = []
        for i, (st, tg) in enumerate(zip(self.states, self.checks)):
            phi, E = self.batch.outputs[i]
            err = max(errs[i]) if E is not None else errs[i][0]
            r = dict(p=self.choice[i][0], leaf=self.choice[i][1], error=err, fallback=False)
            if err > self.tol:   # the referee's values, once more, for the reruns
                q = self._q[i]
                q_re = q.real.double().contiguous() if q.is_complex() else q.double().contiguous()
                q_im = q.imag.double().contiguous() if q.is_complex() else None
                r_phi, r_E = direct_at(st, q_re, q_im, tg, field=E is not None)
                ref = (r_phi.cpu().numpy(), None if r_E is None else r_E.cpu().numpy())

            def err_of():
                e = _rel_l2(phi[tg].cpu().numpy(), ref[0])
                if E is not None:
                    e = max(e, _rel_l2(E[tg].cpu().numpy(), ref[1]))
                return e
            p = conservative_p(self.tol)
            while err > self.tol and p <= P_MAX:
                x, k = self.problems[i]
                plain = setup(x, k, p=p, N_max=FEATURE_LEAF, device=self.device)
                evaluate_into(plain, q_re, q_im, phi, E, PREC_FP64)
                check_errors(plain)
                plain.close()
                err = err_of()
                r.update(fallback=True, p_final=p, error=err)
                p += 2
            r["certified"] = bool(err <= self.tol)
            rep.append(r)
        self.report = rep
        return rep

    def close(self):
        if self.batch is not None:
            self.batch.close()
        for st in self.states:
            st.close()
