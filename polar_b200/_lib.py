"""ctypes binding of libpolar.so (the sm_100a kernels; C ABI declared in include/polar.h).

The library is built in-tree by polar_b200/csrc/build.py.  There is no fallback: if the
shared object is missing, or no CUDA device is present when a kernel is requested,
importing the binding raises.
"""
import ctypes
import os
from pathlib import Path

_HERE = Path(__file__).resolve().parent
LIB_PATH = Path(os.environ.get("POLAR_LIB", _HERE / "libpolar.so"))

POLAR_OK = 0
POLAR_ERR_ITER_CAP = 1
POLAR_ERR_NONFINITE = 2
POLAR_ERR_BAD_ARG = 3
POLAR_ERR_WORKSPACE = 4
POLAR_ERR_TIMEOUT = 5
POLAR_ERR_CUDA = 6
POLAR_ERR_UNSUPPORTED = 7
POLAR_FP64 = 0
POLAR_MIXED = 1

STATUS_NAMES = {0: "OK", 1: "ITER_CAP", 2: "NONFINITE", 3: "BAD_ARG", 4: "WORKSPACE", 5: "TIMEOUT",
                6: "CUDA", 7: "UNSUPPORTED"}


class PolarError(RuntimeError):
    """A libpolar call returned a non-zero status."""

    def __init__(self, status, msg):
        self.status = status
        super().__init__(msg)


class PolarGraph(ctypes.Structure):
    _fields_ = [
        ("n", ctypes.c_int32), ("nnz", ctypes.c_int32),
        ("d_indptr", ctypes.c_void_p), ("d_indices", ctypes.c_void_p),
        ("d_wts", ctypes.c_void_p), ("d_diag", ctypes.c_void_p),
        ("sigma", ctypes.c_double),
        ("nx", ctypes.c_int32),
        ("d_xbits", ctypes.c_void_p), ("d_xrow", ctypes.c_void_p), ("d_xoff", ctypes.c_void_p),
        ("d_xnbr", ctypes.c_void_p), ("d_xwt", ctypes.c_void_p),
        ("heavy_thresh", ctypes.c_int32), ("nheavy", ctypes.c_int32), ("nchunks", ctypes.c_int32),
        ("d_hrow", ctypes.c_void_p), ("d_hchunk_off", ctypes.c_void_p), ("d_chunk_row", ctypes.c_void_p),
        ("d_chunk_lo", ctypes.c_void_p), ("d_chunk_hi", ctypes.c_void_p),
        ("nrb", ctypes.c_int32), ("d_rowblk", ctypes.c_void_p),
        ("nsl", ctypes.c_int32), ("sell_s", ctypes.c_int32),
        ("d_sl_off", ctypes.c_void_p), ("d_sl_rows", ctypes.c_void_p), ("d_sl_idx", ctypes.c_void_p),
    ]


class MsolveInfo(ctypes.Structure):
    _fields_ = [("status", ctypes.c_int32), ("ld", ctypes.c_int32), ("grid", ctypes.c_int32),
                ("block", ctypes.c_int32), ("iterations", ctypes.c_int64), ("flushes", ctypes.c_int64),
                ("error_where", ctypes.c_int32), ("pad", ctypes.c_int32), ("phase_ns", ctypes.c_int64 * 6)]


_P = ctypes.c_void_p
_I = ctypes.c_int
_D = ctypes.c_double
_S = ctypes.c_size_t
_I64 = ctypes.c_int64
_GP = ctypes.POINTER(PolarGraph)


class MsolveProblem(ctypes.Structure):
    """polar_msolve_problem: one solve of a polar_msolve_batch call (polar_msolve's arguments)."""
    _fields_ = [
        ("g", _GP), ("d_W", _P), ("d_tau", _P), ("d_active", _P), ("d_active_pos", _P), ("d_X_out", _P),
        ("d_h_out", _P), ("d_iters_out", _P), ("d_workspace", _P), ("workspace_bytes", _S),
        ("tol", _D), ("maxit", _I64), ("cost", _D),
        ("ldw", ctypes.c_int32), ("R", ctypes.c_int32), ("p", ctypes.c_int32), ("nA", ctypes.c_int32),
        ("track", ctypes.c_int32), ("x_f32", ctypes.c_int32), ("ldx", ctypes.c_int32), ("pad", ctypes.c_int32),
    ]


# name -> (restype, argtypes)
SIGNATURES = {
    "polar_last_error": (ctypes.c_char_p, []),
    "polar_version": (_I, []),
    "polar_launch_count": (ctypes.c_longlong, []),
    "polar_set_kernel_timing": (None, [_I]),
    "polar_kernel_timing": (_I, [_I, ctypes.POINTER(ctypes.c_longlong), ctypes.POINTER(ctypes.c_double),
                                 ctypes.POINTER(ctypes.c_double)]),
    "polar_spmm_scratch_bytes": (_S, [_GP, _I, _I]),
    "polar_spmm_scratch_init": (_I, [_GP, _I, _I, _P, _P]),
    "polar_spmm": (_I, [_GP, _I, _I, _D, _P, _I, _P, _I, _P, _P]),
    "polar_spmm_noalloc": (_I, [_GP, _I, _I, _D, _P, _I, _P, _I, _P]),
    "polar_msolve_workspace_bytes": (_S, [_GP, _I, _I, _I, _I]),
    "polar_msolve": (_I, [_GP, _I, _P, _I, _I, _P, _I, _P, _P, _I, _D, _I64, _I, _P, _I, _I, _P, _P, _P, _S, _P]),
    "polar_msolve_finish": (_I, [_P, _P, ctypes.POINTER(MsolveInfo)]),
    "polar_set_barrier_timeout_ns": (None, [ctypes.c_uint64]),
    "polar_set_solver_mode": (_I, [_I]),
    "polar_heavy_threshold": (_I, [_I, _I]),
    "polar_sell_rows": (_I, [_I, _I]),
    "polar_set_spmm_lane_bytes": (None, [_I]),
    "polar_set_sell": (None, [_I]),
    "polar_set_l2_policy": (_I, [_I, _S]),
    "polar_set_mixed_residual": (_I, [_I]),
    "polar_msolve_batch_workspace_bytes": (_S, [_GP, _I, _I, _I, _I]),
    "polar_msolve_batch": (_I, [ctypes.POINTER(MsolveProblem), _I, _I, _P]),
    "polar_block_orth": (_I, [_P, _I64, _I, _P, _P, _I, _P]),
    "polar_center_columns_tmp_bytes": (_S, [_I]),
    "polar_center_columns": (_I, [_P, _I64, _I, _I, _P, _S, _P]),
    "polar_incidence_apply": (_I, [_I, _P, _P, _P, _P, _I, _I, _P, _I, _P]),
    "polar_fill_incidence": (_I, [_I, _I, _P, _P, _P, _P, _I, _P, _P, _P]),
    "polar_pair_norms": (_I, [_P, _I, _I, _I, _I, _I, _I, _P, _P, _I, _P, _P]),
    "polar_topb_tmp_bytes": (_S, [_I, _I]),
    "polar_score_topb": (_I, [_P, _P, _P, _P, _D, _I, _I, _P, _I, _I, _P, _P, _P, _P, _P]),
    "polar_rerank": (_I, [_P, _I, _I, _I, _I, _P, _P, _I, _P, _P, _I, _P, _P, _P]),
    "polar_select": (_I, [_P, _P, _P, _P, _P, _P]),
    "polar_maintain_tmp_bytes": (_S, [_I, _I, _I]),
    "polar_maintain": (_I, [_P, _I, _P, _I, _I, _I, _I, _I, _P, _I, _I, _P, _P, _P, _I, _P, _P, _P, _P]),
    "polar_maintain_split": (_I, [_P, _I, _P, _I, _I, _I, _I, _I, _P, _I, _I, _P, _P, _P, _I, _P, _P, _P, _P]),
    "polar_cache_apply": (_I, [_P, _P, _P, _P, _I64, _P]),
    "polar_rank1_rows": (_I, [_P, _I, _I, _P, _P, _P, _P]),
}

_lib = None


def load(path=None):
    """Load libpolar.so and bind every entry point of include/polar.h."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = Path(path) if path else LIB_PATH
    if not p.exists():
        raise ImportError(f"libpolar.so not found at {p}; build it with `python -m polar_b200.csrc.build`")
    lib = ctypes.CDLL(str(p))
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if path is None:
        _lib = lib
    return lib


KERNEL_CLASSES = {0: "spmm", 6: "spmm_heavy", 1: "resid", 2: "dir", 3: "flush", 4: "init"}


def kernel_timing():
    """{class name: (launches, device ms, algorithmic bytes)} since polar_set_kernel_timing(1)."""
    lib = load()
    out = {}
    for cls, name in KERNEL_CLASSES.items():
        n = ctypes.c_longlong()
        ms = ctypes.c_double()
        b = ctypes.c_double()
        lib.polar_kernel_timing(cls, ctypes.byref(n), ctypes.byref(ms), ctypes.byref(b))
        out[name] = (n.value, ms.value, b.value)
    return out


def check(status, what=""):
    if status != POLAR_OK:
        msg = load().polar_last_error().decode(errors="replace")
        if status == POLAR_ERR_ITER_CAP:
            raise PolarError(status, "multi-shift CG iteration cap")
        raise PolarError(status, f"{what}: {STATUS_NAMES.get(status, status)}: {msg}")
    return status
