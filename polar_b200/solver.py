"""Multi-shift CG front end: realworld/polar_gpu.py:88-133 (msolve) on the persistent
sm_100a kernel of libpolar (polar_msolve).

    X, h, iters = msolve(op, W, tau, active, tol, maxit=100000, track=False, counter=None)

X[p, nA, R] holds the solutions of (M + tau_j I) U = W on the `active` rows, h[p, R] the
tracked squared norms ||U_j[:, c]||^2 (track=True), iters[R] (host int64) the seed
iterations per column.  Keyword-only extensions: precision ('fp64' | 'mixed'), out /
out_col (write X into columns of an existing [p, nA, ld] tensor), and pre-uploaded device
arrays (tau, active, active_pos) to avoid repeated host->device copies.
"""
import numpy as np
import torch

from . import _lib

__all__ = ["msolve", "Counter", "precision_code", "max_columns", "prepare_active", "set_solver_mode"]


def set_solver_mode(mode):
    """'graph' (default): one kernel per phase, M iterations per CUDA-graph launch;
    'persistent': a single cooperative kernel with bounded grid barriers."""
    code = {"graph": 0, "persistent": 1}[mode]
    _lib.check(_lib.load().polar_set_solver_mode(code), "set_solver_mode")


class Counter:
    def __init__(self):
        self.spmv = 0
        self.rhs = 0


def precision_code(precision):
    if precision in ("fp64", "float64", _lib.POLAR_FP64):
        return _lib.POLAR_FP64
    if precision in ("mixed", "fp32", _lib.POLAR_MIXED):
        return _lib.POLAR_MIXED
    raise ValueError(f"unknown precision {precision!r}")


def max_columns(prec):
    return 128 if prec == _lib.POLAR_MIXED else 64


_WS = {}


def tuned_layouts(G):
    """The graph's SpMM layouts recorded by autotune.tune_msolve, keyed by (precision,
    padded width): (lane bytes, sliced-ELL on/off, heavy-row threshold)."""
    d = getattr(G, "_spmm_tuned", None)
    if d is None:
        d = {}
        G._spmm_tuned = d
    return d


def _padded(prec, R):
    """The solver's padded width for R columns: next power of two, at least one vector."""
    ld = 1
    while ld < R:
        ld *= 2
    return max(ld, 4 if prec == _lib.POLAR_MIXED else 2)


LARGE_GRAPH_ROWS = 1_000_000
LARGE_GRAPH_HEAVY = 512


def heavy_threshold(G, prec, R):
    """Degree above which a row goes to the SpMM's warp chunks for an R-column solve: the
    library's width rule, raised to 512 on graphs of a million rows or more, where the
    sliced-ELL slices handle mid-degree rows with less overhead per row (measured on the
    4M-vertex graph: R = 16 mixed 1.215 -> 1.070 ms, FP64 1.619 -> 1.481 ms, R = 128 mixed
    6.50 -> 5.93 ms per SpMM launch, threshold 32 -> 512)."""
    t = _lib.load().polar_heavy_threshold(prec, R)
    return max(t, LARGE_GRAPH_HEAVY) if G.n >= LARGE_GRAPH_ROWS else t


def workspace(nbytes, device):
    """Grow-only device workspace per (device); shared by consecutive solves."""
    key = device.index
    buf = _WS.get(key)
    if buf is None or buf.numel() < nbytes:
        _WS.pop(key, None)
        buf = torch.empty(int(nbytes), dtype=torch.uint8, device=device)
        _WS[key] = buf
    return buf


def prepare_active(active, n, device):
    """(active int32 device tensor, active_pos int32[n]: row -> active index or -1)."""
    if isinstance(active, torch.Tensor):
        a_h = active.detach().cpu().numpy()
    else:
        a_h = np.asarray(active)
    a_h = a_h.astype(np.int64).ravel()
    if len(a_h) == 0:
        raise ValueError("active must be non-empty")
    if np.any(np.diff(a_h) <= 0):
        raise ValueError("active rows must be strictly increasing")
    pos = np.full(n, -1, dtype=np.int32)
    pos[a_h] = np.arange(len(a_h), dtype=np.int32)
    return (torch.as_tensor(a_h.astype(np.int32)).to(device), torch.as_tensor(pos).to(device))


def msolve(op, W, tau, active, tol, maxit=100000, track=False, counter=None, *, precision="fp64", out=None,
           out_col=0, active_pos=None, x_dtype=None, info=None):
    G = op.G
    dev = G.device
    prec = precision_code(precision)
    if not isinstance(W, torch.Tensor):
        W = torch.as_tensor(np.asarray(W, dtype=np.float64))
    if W.dim() == 1:
        W = W[:, None]
    W = W.to(device=dev, dtype=torch.float64)
    if W.stride(1) != 1:
        W = W.contiguous()
    n, R = W.shape
    if n != G.n:
        raise ValueError("W must have n rows")
    ldw = W.stride(0) if R > 1 else max(1, W.stride(0))
    if isinstance(tau, torch.Tensor):
        tau_d = tau.to(device=dev, dtype=torch.float64).contiguous()
    else:
        tau_d = torch.as_tensor(np.asarray(tau, dtype=np.float64)).to(dev)
    p = tau_d.numel()
    if active_pos is None:
        act_d, pos_d = prepare_active(active, n, dev)
    else:
        act_d = active.to(device=dev, dtype=torch.int32)
        pos_d = active_pos
    nA = act_d.numel()
    if x_dtype is None:
        x_dtype = torch.float32 if prec == _lib.POLAR_MIXED else torch.float64
    if out is None:
        out = torch.empty((p, nA, R), dtype=x_dtype, device=dev)
        out_col = 0
    if out.shape[0] != p or out.shape[1] != nA or out.stride(2) != 1 or out_col + R > out.shape[2]:
        raise ValueError("out has the wrong shape")
    x_f32 = 1 if out.dtype == torch.float32 else 0
    h = torch.zeros((p, R), dtype=torch.float64, device=dev) if track else None
    iters = torch.zeros(R, dtype=torch.int64, device=dev)
    lib = _lib.load()
    stream = torch.cuda.current_stream(dev).cuda_stream
    maxc = max_columns(prec)
    info_list = []
    for lo in range(0, R, maxc):
        hi = min(R, lo + maxc)
        r = hi - lo
        cfg = tuned_layouts(G).get((int(prec), _padded(prec, r)))
        if cfg is not None:
            lib.polar_set_spmm_lane_bytes(cfg[0])
            lib.polar_set_sell(cfg[1])
        try:
            thresh = cfg[2] if cfg is not None else heavy_threshold(G, prec, r)
            g = op.struct(heavy_thresh=thresh, sell_rows=lib.polar_sell_rows(prec, r))
            need = lib.polar_msolve_workspace_bytes(g, prec, r, p, nA)
            ws = workspace(need, dev)
            hpart = torch.zeros((p, r), dtype=torch.float64, device=dev) if track else None
            xo = out[:, :, out_col + lo:]
            st = lib.polar_msolve(g, prec, W[:, lo:].data_ptr(), ldw, r, tau_d.data_ptr(), p, act_d.data_ptr(),
                                  pos_d.data_ptr(), nA, float(tol), int(maxit), 1 if track else 0, xo.data_ptr(),
                                  x_f32, out.shape[2], hpart.data_ptr() if track else None, iters[lo:].data_ptr(),
                                  ws.data_ptr(), ws.numel(), stream)
        finally:
            if cfg is not None:  # back to the automatic layout
                lib.polar_set_spmm_lane_bytes(0)
                lib.polar_set_sell(1)
        _lib.check(st, "polar_msolve")
        inf = _lib.MsolveInfo()
        st = lib.polar_msolve_finish(ws.data_ptr(), stream, inf)
        info_list.append(inf)
        _lib.check(st, "polar_msolve")
        if track:
            h[:, lo:hi] = hpart
    it_h = iters.cpu().numpy()
    if counter is not None:
        counter.spmv += int(it_h.sum())
        counter.rhs += R
    if info is not None:
        info.extend(info_list)
    return out[:, :, out_col:out_col + R], h, it_h
