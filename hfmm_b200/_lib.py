"""ctypes binding of the hfmm_b200 C ABI (include/hfmm_b200.h).

The shared library is built in-tree by ``hfmm_b200.build``. There is no CPU or
pure-Python fallback: if the library is missing or fails to load, importing
this module raises.
"""
import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_lib", "libhfmm_b200.so")

HFMM_OK = 0
HFMM_PREC_FP64 = 0
HFMM_PREC_MIXED = 1
N_PHASES = 15
PHASES = ("gather", "p2m", "m2m_gemm", "up_decode", "m2l_l2l_gemm", "p2l", "down_decode",
          "p2p", "l2p", "m2p", "combine", "tf32_split", "m2l_tables", "l2l_gemm",
          "m2l_compress")

_c_i32, _c_i64, _c_dbl, _c_vp = ctypes.c_int32, ctypes.c_int64, ctypes.c_double, ctypes.c_void_p


class HfmmInfo(ctypes.Structure):
    _fields_ = [
        ("n_points", _c_i64), ("max_depth", _c_i32), ("maxleaf", _c_i32),
        ("max_boxes", _c_i64), ("n_boxes", _c_i64), ("n_leaves", _c_i64),
        ("adaptive", _c_i32), ("level_lo", _c_i32 * 16), ("level_hi", _c_i32 * 16),
        ("domain_extent", _c_dbl), ("pmin", _c_dbl * 3),
        ("n_v", _c_i64), ("n_u", _c_i64), ("n_w", _c_i64), ("n_x", _c_i64), ("n_near", _c_i64),
        ("n_s", _c_i32), ("p", _c_i32),
    ]

    def as_dict(self):
        md = self.max_depth
        return dict(
            n_points=self.n_points, max_depth=md, maxleaf=self.maxleaf,
            max_boxes=self.max_boxes, n_boxes=self.n_boxes, n_leaves=self.n_leaves,
            adaptive=bool(self.adaptive),
            level_ranges={l: (self.level_lo[l], self.level_hi[l]) for l in range(1, md + 1)},
            domain_extent=self.domain_extent, pmin=tuple(self.pmin),
            n_v=self.n_v, n_u=self.n_u, n_w=self.n_w, n_x=self.n_x, n_near=self.n_near,
            n_s=self.n_s, p=self.p)


# (name, restype, argtypes) for every symbol of include/hfmm_b200.h
SIGNATURES = [
    ("hfmm_tree_build", _c_i32, [_c_vp, _c_i64, _c_i32, _c_i32, ctypes.POINTER(_c_vp)]),
    ("hfmm_plan_info", _c_i32, [_c_vp, ctypes.POINTER(HfmmInfo)]),
    ("hfmm_tree_build_in_domain", _c_i32, [_c_vp, _c_i64, _c_i32, _c_i32, _c_vp, _c_dbl,
                                           ctypes.POINTER(_c_vp)]),
    ("hfmm_plan_rebuild", _c_i32, [_c_vp, _c_vp]),
    ("hfmm_plan_set_kernel_kind", _c_i32, [_c_vp, _c_i32]),
    ("hfmm_plan_set_kernel", _c_i32, [_c_vp, _c_dbl, _c_i32, _c_i32, _c_vp, _c_vp]),
    ("hfmm_plan_set_level", _c_i32, [_c_vp, _c_i32, _c_i32] + [_c_vp] * 9),
    ("hfmm_plan_set_level_decode", _c_i32, [_c_vp, _c_i32, _c_i32] + [_c_vp] * 6),
    ("hfmm_plan_set_streaming", _c_i32, [_c_vp, _c_i32]),
    ("hfmm_plan_workspace_bytes", _c_i32, [_c_vp, ctypes.POINTER(_c_i64)]),
    ("hfmm_plan_bind_workspace", _c_i32, [_c_vp, _c_vp, _c_i64]),
    ("hfmm_plan_finalize", _c_i32, [_c_vp]),
    ("hfmm_evaluate", _c_i32, [_c_vp, _c_vp, _c_vp, _c_vp, _c_vp, _c_i32, _c_vp]),
    ("hfmm_plan_check", _c_i32, [_c_vp, _c_vp]),
    ("hfmm_plan_destroy", None, [_c_vp]),
    ("hfmm_debug_m2l_wait", _c_i32, [ctypes.c_uint64, _c_i32]),
    ("hfmm_debug_m2l_grid", _c_i32, [_c_i32]),
    ("hfmm_export_tree", _c_i32, [_c_vp] * 7),
    ("hfmm_export_pil", _c_i32, [_c_vp, _c_vp]),
    ("hfmm_export_list", _c_i32, [_c_vp, _c_i32, _c_vp, _c_i64]),
    ("hfmm_export_densities", _c_i32, [_c_vp, _c_i32, _c_i32, _c_vp, _c_i64]),
    ("hfmm_direct", _c_i32, [_c_vp, _c_vp, _c_vp, _c_i64, _c_vp, _c_i64, _c_dbl, _c_vp, _c_vp,
                             _c_vp]),
    ("hfmm_direct_kernel", _c_i32, [_c_i32, _c_vp, _c_vp, _c_vp, _c_i64, _c_vp, _c_i64, _c_dbl,
                                    _c_vp, _c_vp, _c_vp]),
    ("hfmm_direct_scratch_bytes", _c_i64, [_c_i64, _c_i64]),
    ("hfmm_direct_async", _c_i32, [_c_vp, _c_vp, _c_vp, _c_i64, _c_vp, _c_i64, _c_dbl, _c_vp, _c_vp,
                                   _c_vp, _c_i64, _c_vp, _c_vp]),
    ("hfmm_direct_noalloc", _c_i32, [_c_vp, _c_vp, _c_vp, _c_i64, _c_vp, _c_i64, _c_dbl, _c_vp,
                                     _c_vp, _c_vp]),
    ("hfmm_plan_set_profiling", _c_i32, [_c_vp, _c_i32]),
    ("hfmm_plan_phase_times", _c_i32, [_c_vp, _c_vp]),
    ("hfmm_plan_set_m2l_compressed", _c_i32, [_c_vp, _c_i32, _c_i32, _c_i32, _c_vp, _c_vp]),
    ("hfmm_batch_create", _c_i32, [ctypes.POINTER(_c_vp), _c_i32, _c_i32, ctypes.POINTER(_c_vp)]),
    ("hfmm_batch_stream_of", _c_i32, [_c_vp, _c_i32]),
    ("hfmm_batch_set_queue", _c_i32, [_c_vp, _c_i32]),
    ("hfmm_batch_queued", _c_i32, [_c_vp]),
    ("hfmm_batch_queue_note", ctypes.c_char_p, [_c_vp]),
    ("hfmm_plan_set_m2l_queue", _c_i32, [_c_vp, _c_i32]),
    ("hfmm_plan_set_m2l_rotation", _c_i32, [_c_vp, _c_i32, _c_vp, _c_i32, _c_vp, _c_vp, _c_vp, _c_i32]),
    ("hfmm_plan_set_rotation_level", _c_i32, [_c_vp, _c_i32, _c_i32, _c_vp, _c_vp, _c_vp, _c_dbl]),
    ("hfmm_batch_set_problem", _c_i32, [_c_vp, _c_i32, _c_vp, _c_vp, _c_vp, _c_vp, _c_i32]),
    ("hfmm_batch_set_check", _c_i32, [_c_vp, _c_i32, _c_vp, _c_vp, _c_i32, _c_vp]),
    ("hfmm_batch_capture", _c_i32, [_c_vp]),
    ("hfmm_batch_launch", _c_i32, [_c_vp, _c_vp]),
    ("hfmm_batch_destroy", None, [_c_vp]),
    ("hfmm_mlp_param_count", _c_i32, [_c_i32, _c_i32]),
    ("hfmm_mlp_forward", _c_i32, [_c_vp, _c_vp, _c_i32, _c_i32, _c_i32, _c_vp, _c_vp]),
    ("hfmm_mlp_grad", _c_i32, [_c_vp, _c_vp, _c_vp, _c_i32, _c_i32, _c_i32, _c_vp,
                               ctypes.POINTER(_c_dbl), _c_vp]),
    ("hfmm_mlp_train", _c_i32, [_c_vp, _c_vp, _c_vp, _c_i64, _c_vp, _c_vp, _c_i32, _c_i32, _c_i32,
                                _c_i32, ctypes.c_float, ctypes.POINTER(_c_dbl), _c_vp]),
    ("hfmm_last_error", ctypes.c_char_p, []),
    ("hfmm_launch_count", _c_i64, []),
]


class HFMMError(RuntimeError):
    """A C-ABI call returned a non-zero status."""

    def __init__(self, code, msg):
        super().__init__(f"hfmm_b200 error {code}: {msg}")
        self.code = code


def load():
    """Load (once) and return the library; raises ImportError when it is missing."""
    global _handle
    if _handle is not None:
        return _handle
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"hfmm_b200: CUDA library not built ({LIB_PATH} missing); run "
            "`python -m hfmm_b200.build` (there is no CPU fallback)")
    lib = ctypes.CDLL(LIB_PATH)
    for name, res, args in SIGNATURES:
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _handle = lib
    return lib


class _Lazy:
    """Resolves symbols on first use, so building the library never needs an old copy."""

    def __getattr__(self, name):
        return getattr(load(), name)


_handle = None
lib = _Lazy()


def check(code):
    """Raise HFMMError (or ValueError for argument errors) on a non-zero status."""
    if code != HFMM_OK:
        msg = lib.hfmm_last_error().decode(errors="replace")
        if code == -1:
            raise ValueError(msg)
        raise HFMMError(code, msg)


def launch_count():
    return int(lib.hfmm_launch_count())
