"""hfmm_b200 -- Helmholtz KIFMM evaluate path on B200 (sm_100a).

Drop-in for the reference's Python API (HFMM.py:55-91):

    state = setup(positions, k, p=4, N_max=16, max_depth=None)
    phi = evaluate(state, charges)            # real charges -> complex128 (N,)

plus the complex-charge / field form the reference reaches only by combining
four real evaluates (``kifmm.evaluate_setup(..., field=True)``,
kifmm/setup.py:229-261):

    phi, E = evaluate_field(state, charges)   # complex charges; E = -grad(phi), (N, 3)

Positions, charges and results may be NumPy arrays or torch tensors; NumPy in,
NumPy out. The tree, the interaction lists and every evaluate phase run as CUDA
kernels of the in-tree library ``_lib/libhfmm_b200.so``; there is no CPU path.
"""
import numpy as np
import torch

from . import _lib
from ._lib import check as _check, HFMMError, launch_count
from .operators import level_tables, level_decodes, surface_pts, R_EQUIV, R_CHECK, n_surf

__all__ = ["setup", "evaluate", "evaluate_field", "evaluate_into", "direct", "direct_at",
           "HFMMState", "kernel_setup", "kernel_evaluate", "rebuild",
           "HFMMError", "launch_count", "PREC_FP64", "PREC_MIXED"]

PREC_FP64 = _lib.HFMM_PREC_FP64
PREC_MIXED = _lib.HFMM_PREC_MIXED


def _device(device):
    if device is None:
        if not torch.cuda.is_available():
            raise RuntimeError("hfmm_b200 needs a CUDA device (no CPU fallback)")
        return torch.device("cuda", torch.cuda.current_device())
    return torch.device(device)


class HFMMState:
    """A built plan: the octree, lists, operator tables and evaluate buffers on one GPU.

    Plays the role of the reference's ``(real_state, imag_state)`` tuple
    (HFMM.py:65-80). ``info`` holds the sizes the reference's setup dict reports
    (max_depth, maxleaf, max_boxes, domain_extent, list lengths).
    """

    def __init__(self, handle, positions, k, p, N_max, device, kernel=None):
        from .kernels import helmholtz
        self._h = handle
        self.positions = positions          # (N, 3) float64 on the device
        self.n = positions.shape[0]
        self.kernel = kernel if kernel is not None else helmholtz(k)
        self.kind = self.kernel.kind
        self.k = float(self.kernel.param)
        self.p = int(p)
        self.N_max = int(N_max)
        self.device = device
        self.n_families = self.kernel.families
        self._pin = {}
        self._refresh()

    def _refresh(self):
        info = _lib.HfmmInfo()
        _check(_lib.lib.hfmm_plan_info(self._h, info))
        self.info = info.as_dict()
        self.max_depth = self.info["max_depth"]

    @property
    def handle(self):
        if self._h is None:
            raise RuntimeError("HFMMState was closed")
        return self._h

    def _pinned(self, name, shape, dtype):
        """A reused page-locked host buffer (the staging of NumPy charges)."""
        t = self._pin.get(name)
        if t is None or tuple(t.shape) != tuple(shape) or t.dtype != dtype:
            t = torch.empty(tuple(shape), dtype=dtype, pin_memory=True)
            self._pin[name] = t
        return t

    def close(self):
        if getattr(self, "_h", None) is not None:
            _lib.lib.hfmm_plan_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---- inspection (tests) ----
    def tree(self):
        """Tree arrays of the active boxes, as NumPy (the build_fmm_tree outputs)."""
        nb, n = self.info["n_boxes"], self.n
        out = dict(m_id=np.empty(nb, np.uint64), p_id=np.empty(nb, np.int32),
                   lvls=np.empty(nb, np.int32), counts=np.empty(nb, np.int32),
                   is_leaf=np.empty(nb, np.uint8), sort_idx=np.empty(n, np.int32))
        _check(_lib.lib.hfmm_export_tree(self.handle, *(out[k].ctypes.data for k in
                                                         ("m_id", "p_id", "lvls", "counts",
                                                          "is_leaf", "sort_idx"))))
        out["is_leaf"] = out["is_leaf"].astype(bool)
        return out

    def pil(self):
        nb, w = self.info["n_boxes"], self.info["maxleaf"]
        out = np.empty((nb, w), np.int32)
        _check(_lib.lib.hfmm_export_pil(self.handle, out.ctypes.data))
        return out

    def densities(self, which, columns=1):
        """Upward equivalent ("up", after P2M and M2M) or downward local ("down", after
        M2L, P2L and L2L) densities of the last FP64 evaluate, which had ``columns``
        charge columns: (n_families, n_boxes, columns, n_s) float64, the boxes of
        levels 2..max_depth filled (hfmm_export_densities)."""
        nf, nb, ns = self.n_families, self.info["n_boxes"], self.info["n_s"]
        out = np.empty((nf, nb, int(columns), ns), np.float64)
        _check(_lib.lib.hfmm_export_densities(self.handle, {"up": 0, "down": 1}[which],
                                              int(columns), out.ctypes.data, out.size))
        return out

    def pairs(self, which):
        """Interaction list as (len, 2) int32: 'V', 'U', 'W', 'X' or 'near'."""
        idx = {"V": 0, "U": 1, "W": 2, "X": 3, "near": 4}[which]
        n = self.info[{"V": "n_v", "U": "n_u", "W": "n_w", "X": "n_x", "near": "n_near"}[which]]
        out = np.empty((max(n, 1), 2), np.int32)
        _check(_lib.lib.hfmm_export_list(self.handle, idx, out.ctypes.data, max(n, 1)))
        return out[:n]


def _validate_setup(positions, k, p, N_max, max_depth):
    """HFMM.py:14-16 and 57-64."""
    if isinstance(positions, torch.Tensor):
        x = positions.detach().to(torch.float64)
        ok_shape = x.ndim == 2 and x.shape[1] == 3 and x.shape[0] > 0
        if not ok_shape or not bool(torch.isfinite(x).all()):
            raise ValueError("positions must be a nonempty finite (N,3) array")
    else:
        x = np.asarray(positions, dtype=np.float64)
        if x.ndim != 2 or x.shape[1] != 3 or len(x) == 0 or not np.isfinite(x).all():
            raise ValueError("positions must be a nonempty finite (N,3) array")
    if p < 2 or int(p) != p or N_max < 1 or int(N_max) != N_max:
        raise ValueError("p must be an integer >=2; N_max must be a positive integer")
    if max_depth is not None and (max_depth < 1 or int(max_depth) != max_depth):
        raise ValueError("max_depth must be a positive integer or None")
    kf = float(k)
    if not np.isfinite(kf):
        raise ValueError("k must be a finite real number")
    return x, kf


def setup(positions, k, p=4, N_max=16, max_depth=None, device=None, tables="device",
          stream_tables=False, m2l_compress=None, domain=None, kernel=None):
    """Build the plan for ``positions`` and wavenumber ``k`` (HFMM.setup, HFMM.py:55-80).

    ``p`` is the number of surface points per cube edge, ``N_max`` the leaf
    size and ``max_depth`` an optional depth cap (``None``: the reference's
    automatic depth with refinement, trees/cubic.py:577-600).
    ``tables``: "device" evaluates the M2M/L2L/M2L kernel matrices on the GPU
    (the decodes still come from the host SVD); "host" assembles every table in
    NumPy with the reference's expressions, bit for bit.
    ``stream_tables``: keep no M2L table resident; each evaluate regenerates a
    level's 316 M2L matrices on the device right before its M2L (bit-identical
    to the resident "device" tables; memory per plan drops to one level's worth).
    ``m2l_compress``: a relative tolerance (e.g. 1e-8) to give the mixed-precision
    evaluate a low-rank M2L (``hfmm_b200.compress``); the FP64 evaluate is unchanged.
    ``domain``: ``(pmin (3,), extent)``, a fixed domain cube instead of the points'
    bounding box (moving geometry, ``hfmm_b200.moving``); needs ``max_depth``. Every
    point must lie inside it; ``rebuild`` then moves the points within it.
    ``kernel``: a ``hfmm_b200.kernels`` specification in place of the Helmholtz
    components of ``k`` (``kernel_setup`` is the entry point for it).
    """
    if tables not in ("device", "host"):
        raise ValueError('tables must be "device" or "host"')
    if stream_tables and tables != "device":
        raise ValueError('stream_tables needs tables="device"')
    x, kf = _validate_setup(positions, k, p, N_max, max_depth)
    if domain is not None:
        lo, ext = np.asarray(domain[0], dtype=np.float64).reshape(3), float(domain[1])
        if max_depth is None:
            raise ValueError("a fixed domain needs max_depth")
        if not (np.isfinite(lo).all() and np.isfinite(ext) and ext > 0):
            raise ValueError("domain must be (finite corner (3,), positive extent)")
    dev = _device(device)
    with torch.cuda.device(dev):
        pos = torch.as_tensor(x, dtype=torch.float64).to(dev).contiguous()
        h = _lib.ctypes.c_void_p()
        if domain is None:
            _check(_lib.lib.hfmm_tree_build(pos.data_ptr(), pos.shape[0], int(N_max),
                                            int(max_depth) if max_depth is not None else 0,
                                            _lib.ctypes.byref(h)))
        else:
            lo_c = (_lib.ctypes.c_double * 3)(*lo.tolist())
            _check(_lib.lib.hfmm_tree_build_in_domain(pos.data_ptr(), pos.shape[0], int(N_max),
                                                      int(max_depth), lo_c, ext,
                                                      _lib.ctypes.byref(h)))
        state = HFMMState(h.value, pos, kf, p, N_max, dev, kernel)
        try:
            _load_tables(state, tables, stream_tables)
            if m2l_compress is not None:
                _load_compressed(state, float(m2l_compress))
            _check(_lib.lib.hfmm_plan_finalize(state.handle))
        except Exception:
            state.close()
            raise
        state._refresh()
    return state


def rebuild(state, positions):
    """Move a fixed-domain plan's points (hfmm_plan_rebuild): the tree, lists and
    schedules are rebuilt in place on the device for ``positions`` (same N), the
    operator tables are kept. A point outside the plan's domain raises HFMMError
    (HFMM_ERR_CAPACITY, -4) before anything changes."""
    x, _ = _validate_setup(positions, state.k, state.p, state.N_max, None)
    if x.shape[0] != state.n:
        raise ValueError("rebuild keeps the number of points")
    with torch.cuda.device(state.device):
        pos = torch.as_tensor(x, dtype=torch.float64).to(state.device).contiguous()
        _check(_lib.lib.hfmm_plan_rebuild(state.handle, pos.data_ptr()))
        state.positions = pos
        state._refresh()
    return state


def _load_tables(state, mode="device", streamed=False):
    p, md = state.p, state.max_depth
    extent = state.info["domain_extent"]
    eq = np.ascontiguousarray(surface_pts(p, R_EQUIV))
    ch = np.ascontiguousarray(surface_pts(p, R_CHECK))
    yuk = state.kind == "yukawa"
    _check(_lib.lib.hfmm_plan_set_kernel_kind(state.handle, 1 if yuk else 0))
    _check(_lib.lib.hfmm_plan_set_kernel(state.handle, state.k, p, state.n_families,
                                         eq.ctypes.data, ch.ctypes.data))
    _check(_lib.lib.hfmm_plan_set_streaming(state.handle, int(bool(streamed))))
    state.streamed = bool(streamed)
    for fam in range(state.n_families):
        # HFMM.py:75-77; another kernel: build_operators_leveled's default (operators.py:572)
        eps_rel = 1e-7 if fam == 0 else 1e-12
        for level in range(2, md + 1):
            if mode == "device":
                t = level_decodes(p, level, extent, state.k, fam == 1, eps_rel, state.kind)
                arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in
                        (t["F_up"][0], t["F_up"][1], t["F_up"][2], t["F_dn"][0], t["F_dn"][1],
                         t["F_dn"][2])]
                _check(_lib.lib.hfmm_plan_set_level_decode(state.handle, fam, level,
                                                           *[a.ctypes.data for a in arrs]))
                continue
            t = level_tables(p, level, md, extent, state.k, fam == 1, eps_rel, state.kind)
            arrs = [t["F_up"][0], t["F_up"][1], t["F_up"][2], t["F_dn"][0], t["F_dn"][1],
                    t["F_dn"][2], t["M2M_K"], t["L2L_K"], t["M2L_K"]]
            arrs = [None if a is None else np.ascontiguousarray(a, dtype=np.float64) for a in arrs]
            ptrs = [None if a is None else a.ctypes.data for a in arrs]
            _check(_lib.lib.hfmm_plan_set_level(state.handle, fam, level, *ptrs))
            del arrs, t


def _load_compressed(state, eps):
    """Low-rank M2L of every level and family (hfmm_plan_set_m2l_compressed)."""
    from .compress import level_compressed
    extent = state.info["domain_extent"]
    state.m2l_ranks = {}
    with torch.cuda.device(state.device):
        for fam in range(state.n_families):
            for level in range(2, state.max_depth + 1):
                U, C = level_compressed(state.p, level, extent, state.k, fam == 1, eps, state.device,
                                        state.kind)
                r = U.shape[1]
                _check(_lib.lib.hfmm_plan_set_m2l_compressed(state.handle, fam, level, r,
                                                              U.data_ptr(), C.data_ptr()))
                state.m2l_ranks[(fam, level)] = r
                del U, C


def _need_tensors(state, specs):
    """The kernels take raw pointers and trust the sizes of the plan, so a buffer of
    the wrong size, type, layout or device is refused before any pointer is passed.
    ``specs``: (tensor, name, dtype, shape) per buffer; sizes are checked for all
    of them first, then devices."""
    for t, name, dtype, shape in specs:
        if not isinstance(t, torch.Tensor):
            raise ValueError(f"{name} must be a torch tensor")
        if t.dtype != dtype or tuple(t.shape) != shape:
            raise ValueError(f"{name} must be {dtype} of shape {shape}, "
                             f"got {t.dtype} {tuple(t.shape)}")
        if not t.is_contiguous():
            raise ValueError(f"{name} must be contiguous")
    for t, name, _, _ in specs:
        if not t.is_cuda or (state.device.index is not None
                             and t.device.index != state.device.index):
            raise ValueError(f"{name} must be on the plan's device {state.device}, got {t.device}")


def evaluate_into(state, q_re, q_im, phi_out, field_out=None, precision=PREC_FP64, stream=None):
    """Allocation-free evaluate on device tensors (float64 charges, complex128 outputs).

    ``q_im`` may be None (real charges). ``stream`` is a torch.cuda.Stream or
    None (the current stream). Asynchronous; call ``check_errors`` to read the
    device error flag. Raises ValueError, before launching anything, for a buffer
    that is not a contiguous tensor of the plan's size and type on its device:
    charges float64 (N,), ``phi_out`` complex128 (N,), ``field_out`` complex128 (N, 3).
    """
    n = state.n
    specs = [(q_re, "q_re", torch.float64, (n,)), (phi_out, "phi_out", torch.complex128, (n,))]
    if q_im is not None:
        specs.append((q_im, "q_im", torch.float64, (n,)))
    if field_out is not None:
        specs.append((field_out, "field_out", torch.complex128, (n, 3)))
    _need_tensors(state, specs)
    if int(precision) not in (PREC_FP64, PREC_MIXED):
        raise ValueError("precision must be PREC_FP64 or PREC_MIXED")
    s = stream if stream is not None else torch.cuda.current_stream(state.device)
    _check(_lib.lib.hfmm_evaluate(
        state.handle, q_re.data_ptr(), None if q_im is None else q_im.data_ptr(),
        phi_out.data_ptr(), None if field_out is None else field_out.data_ptr(),
        int(precision), s.cuda_stream))


def check_errors(state, stream=None):
    s = stream if stream is not None else torch.cuda.current_stream(state.device)
    _check(_lib.lib.hfmm_plan_check(state.handle, s.cuda_stream))


def _stage_charges(owner, q, is_cplx, dev):
    """NumPy charges -> device tensor, through the owner's reused page-locked buffer
    (pageable copies run far slower); the host copy into it is torch's threaded one
    where the array allows. The owner's previous call has synchronised, so the
    buffer is free."""
    dt = torch.complex128 if is_cplx else torch.float64
    qp = owner._pinned("q", q.shape, dt)
    if q.dtype == (np.complex128 if is_cplx else np.float64) and q.flags.c_contiguous \
            and q.flags.writeable:
        qp.copy_(torch.from_numpy(q))
    else:
        qp.numpy()[...] = q
    return qp.to(dev, non_blocking=True)


def _to_host(t):
    """Start the copy of device tensor ``t`` into a new page-locked host tensor from
    torch's caching host allocator; ``.numpy()`` of it, after a synchronise, is the
    result handed to the caller. No host-side copy and no page faults on fresh
    memory: the array keeps its block, which goes back to the cache (and to a later
    call) only when the caller drops the array."""
    h = torch.empty(tuple(t.shape), dtype=t.dtype, pin_memory=True)
    h.copy_(t, non_blocking=True)
    return h


def _run(state, charges, complex_ok, field, precision):
    numpy_in = not isinstance(charges, torch.Tensor)
    if numpy_in:
        q = np.asarray(charges)
        is_cplx = np.iscomplexobj(q)
    else:
        q = charges
        is_cplx = q.is_complex()
    if tuple(q.shape) != (state.n,) or (is_cplx and not complex_ok):
        raise ValueError("charges must be a real array of shape (N,)")
    dev = state.device
    with torch.cuda.device(dev):
        if numpy_in:
            q = _stage_charges(state, q, is_cplx, dev)
        else:
            q = q.detach().to(dev)
        if is_cplx:
            q_re = q.real.to(torch.float64).contiguous()
            q_im = q.imag.to(torch.float64).contiguous()
        else:
            q_re = q.to(torch.float64).contiguous()
            q_im = None
        phi = torch.empty(state.n, dtype=torch.complex128, device=dev)
        E = torch.empty((state.n, 3), dtype=torch.complex128, device=dev) if field else None
        evaluate_into(state, q_re, q_im, phi, E, precision)
        check_errors(state)
        if numpy_in:
            php = _to_host(phi)
            Ep = _to_host(E) if E is not None else None
            torch.cuda.current_stream(dev).synchronize()
            phi = php.numpy()
            E = Ep.numpy() if E is not None else None
    return (phi, E) if field else phi


def evaluate(state, charges, precision=PREC_FP64):
    """HFMM.evaluate (HFMM.py:83-91): real charges (N,) -> complex128 potential (N,)
    in the input point order; complex charges raise ValueError."""
    return _run(state, charges, complex_ok=False, field=False, precision=precision)


def evaluate_field(state, charges, precision=PREC_FP64):
    """Potential and field E = -grad(phi) for real or complex charges (N,).
    Returns (phi (N,), E (N, 3)), both complex128."""
    return _run(state, charges, complex_ok=True, field=True, precision=precision)


def direct_at(state, q_re, q_im, targets, field=False, stream=None):
    """Device form of ``direct``: float64 charge tensors (``q_im`` may be None) and
    int32 target indices, all on the plan's device; returns device tensors
    (phi (T,), E (T, 3) or None). The indices must lie in [0, N): they are read
    on the device without a check (``direct`` checks them on the host)."""
    if not isinstance(targets, torch.Tensor) or targets.ndim != 1:
        raise ValueError("targets must be a 1-D torch tensor")
    specs = [(q_re, "q_re", torch.float64, (state.n,)),
             (targets, "targets", torch.int32, (targets.shape[0],))]
    if q_im is not None:
        specs.append((q_im, "q_im", torch.float64, (state.n,)))
    _need_tensors(state, specs)
    m = targets.shape[0]
    dev = state.device
    phi = torch.empty(m, dtype=torch.complex128, device=dev)
    E = torch.empty((m, 3), dtype=torch.complex128, device=dev) if field else None
    s = stream if stream is not None else torch.cuda.current_stream(dev)
    _check(_lib.lib.hfmm_direct_kernel(_kind_code(state), state.positions.data_ptr(),
                                       q_re.data_ptr(), None if q_im is None else q_im.data_ptr(),
                                       state.n, targets.data_ptr(), m, state.k, phi.data_ptr(),
                                       None if E is None else E.data_ptr(), s.cuda_stream))
    return phi, E


def _kind_code(state):
    return 1 if getattr(state, "kind", "helmholtz") == "yukawa" else 0


def direct(state, charges, targets, field=False):
    """GPU direct sum sum_{s: r>0} q_s e^{ikr}/r (and -grad) at ``targets`` (indices),
    the referee of test.py:11-18. Returns NumPy complex arrays."""
    tg_h = np.asarray(targets)
    if tg_h.ndim != 1 or not (np.issubdtype(tg_h.dtype, np.integer) or tg_h.size == 0):
        raise ValueError("targets must be a 1-D array of point indices")
    if tg_h.size and (tg_h.min() < 0 or tg_h.max() >= state.n):
        raise ValueError(f"targets must lie in [0, {state.n})")
    if tuple(np.shape(charges)) != (state.n,):
        raise ValueError(f"charges must have shape ({state.n},)")
    dev = state.device
    with torch.cuda.device(dev):
        q = torch.as_tensor(np.asarray(charges)).to(dev) if not isinstance(charges, torch.Tensor) \
            else charges.to(dev)
        q_re = q.real.to(torch.float64).contiguous() if q.is_complex() else q.to(torch.float64).contiguous()
        q_im = q.imag.to(torch.float64).contiguous() if q.is_complex() else None
        tg = torch.as_tensor(tg_h.astype(np.int32)).to(dev)
        phi = torch.empty(tg.shape[0], dtype=torch.complex128, device=dev)
        E = torch.empty((tg.shape[0], 3), dtype=torch.complex128, device=dev) if field else None
        s = torch.cuda.current_stream(dev)
        _check(_lib.lib.hfmm_direct_kernel(_kind_code(state), state.positions.data_ptr(),
                                           q_re.data_ptr(), None if q_im is None else q_im.data_ptr(),
                                           state.n, tg.data_ptr(), tg.shape[0], state.k,
                                           phi.data_ptr(), None if E is None else E.data_ptr(),
                                           s.cuda_stream))
        phi = phi.cpu().numpy()
        E = E.cpu().numpy() if E is not None else None
    return (phi, E) if field else phi


def kernel_setup(positions, kernel, p=4, N_max=16, max_depth=None, device=None, tables="device",
                 m2l_compress=None, domain=None):
    """The reference's ``kifmm.setup(positions, p, N_max, max_depth, kernel=...)``
    (kifmm/setup.py:19-226) for a kernel of ``hfmm_b200.kernels`` (``yukawa(kappa)``,
    ``LAPLACE``, ``helmholtz(k)``): the same plan, with that kernel in every particle
    kernel, table and referee. Evaluate with ``kernel_evaluate`` (real charges, real
    result, like ``kifmm.evaluate_setup``) or ``evaluate_field`` (complex charges by
    linearity)."""
    from .kernels import KernelSpec
    if not isinstance(kernel, KernelSpec):
        raise ValueError("kernel must be a hfmm_b200.kernels specification")
    return setup(positions, kernel.param, p=p, N_max=N_max, max_depth=max_depth, device=device,
                 tables=tables, m2l_compress=m2l_compress, domain=domain, kernel=kernel)


def kernel_evaluate(state, charges, field=False, precision=PREC_FP64):
    """kifmm.evaluate_setup(s, charges, field) (kifmm/setup.py:229-261) of a real
    kernel plan: real charges (N,) -> potential (N,) or field -grad phi (N, 3), float64."""
    if state.kind != "yukawa":
        raise ValueError("kernel_evaluate is for the real kernels (yukawa, LAPLACE); "
                         "use evaluate / evaluate_field for Helmholtz")
    q = charges if isinstance(charges, torch.Tensor) else np.asarray(charges)
    if (q.is_complex() if isinstance(q, torch.Tensor) else np.iscomplexobj(q)):
        raise ValueError("charges must be real")
    phi, E = _run(state, q, complex_ok=False, field=True, precision=precision)
    out = E if field else phi
    return out.real.copy() if isinstance(out, np.ndarray) else out.real.contiguous()
