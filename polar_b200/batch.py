"""Many graphs' multi-shift solves at once (polar_msolve_batch).

The reference solves one graph per msolve call (realworld/polar_gpu.py:88-133); a study
over many graphs calls it once per graph.  Here a batch of independent problems — each
with its own graph operator, right-hand sides, pole set, active rows and tolerance — is
handed to the library in one call.  With the default kernel-per-phase driver every solve
runs on its own stream with grids sized to its graph, and the host relaunches each
solve's captured iteration block as soon as the previous one drains, so solves of small
graphs, which cannot fill the GPU alone, run side by side with the large ones.  With the
persistent driver (solver.set_solver_mode('persistent')) the whole batch is ONE
cooperative launch: problem b gets a share of the CTAs in proportion to its estimated
work and its CTAs synchronise only among themselves.

    out = msolve_batch(ops, Ws, taus, actives, tol, maxit=100000, track=False,
                       precision='mixed')

returns one (X[p, nA, R], h[p, R] or None, iters[R] host int64) per problem, the same
triple msolve returns.  tol and maxit may be one value or one per problem.  All problems
share the precision and the padded width (next power of two of R, so e.g. all R in
33..64); at most 64 problems.
"""
import ctypes

import numpy as np
import torch

from . import _lib
from .solver import max_columns, precision_code, prepare_active

__all__ = ["msolve_batch", "batch_cost"]

_WS = {}


def _workspace(slot, nbytes, device):
    """Grow-only device workspace per (device, batch slot)."""
    key = (device.index, slot)
    buf = _WS.get(key)
    if buf is None or buf.numel() < nbytes:
        _WS.pop(key, None)
        buf = torch.empty(int(nbytes), dtype=torch.uint8, device=device)
        _WS[key] = buf
    return buf


def batch_cost(G, R, tau0):
    """Relative work of one solve: per-iteration traffic (nnz + 2n) x R times the CG
    iteration scale sqrt(kappa) of the seed system, kappa = (2 dmax + sigma + tau0) /
    (sigma + tau0)."""
    lo = G.sigma + float(tau0)
    kappa = (2.0 * G.dmax + lo) / lo if lo > 0 else 1e6
    return float(G.nnz + 2 * G.n) * R * np.sqrt(kappa)


def msolve_batch(ops, Ws, taus, actives, tol, maxit=100000, track=False, *, precision="mixed", costs=None,
                 x_dtype=None, info=None):
    prec = precision_code(precision)
    nb = len(ops)
    if not (len(Ws) == len(taus) == len(actives) == nb) or nb == 0:
        raise ValueError("ops, Ws, taus and actives must have the same non-zero length")
    tols = list(tol) if np.ndim(tol) else [float(tol)] * nb
    maxits = list(maxit) if np.ndim(maxit) else [int(maxit)] * nb
    lib = _lib.load()
    dev = ops[0].G.device
    stream = torch.cuda.current_stream(dev).cuda_stream
    probs = (_lib.MsolveProblem * nb)()
    keep = []  # host structs and device tensors that must outlive the call
    outs = []
    maxc = max_columns(prec)
    for b in range(nb):
        G = ops[b].G
        if G.device != dev:
            raise ValueError("all graphs of a batch must live on one device")
        W = Ws[b]
        if not isinstance(W, torch.Tensor):
            W = torch.as_tensor(np.asarray(W, dtype=np.float64))
        if W.dim() == 1:
            W = W[:, None]
        W = W.to(device=dev, dtype=torch.float64).contiguous()
        n, R = W.shape
        if n != G.n:
            raise ValueError(f"problem {b}: W must have n rows")
        if R > maxc:
            raise ValueError(f"problem {b}: at most {maxc} columns per batched problem in this precision")
        tau_d = torch.as_tensor(np.asarray(taus[b], dtype=np.float64)).to(dev)
        p = tau_d.numel()
        act_d, pos_d = prepare_active(actives[b], n, dev)
        nA = act_d.numel()
        xdt = x_dtype or (torch.float32 if prec == _lib.POLAR_MIXED else torch.float64)
        X = torch.empty((p, nA, R), dtype=xdt, device=dev)
        h = torch.zeros((p, R), dtype=torch.float64, device=dev) if track else None
        iters = torch.zeros(R, dtype=torch.int64, device=dev)
        gs = ops[b].struct(heavy_thresh=lib.polar_heavy_threshold(prec, R), sell_rows=lib.polar_sell_rows(prec, R))
        need = lib.polar_msolve_batch_workspace_bytes(gs, prec, R, p, nA)
        ws = _workspace(b, need, dev)
        q = probs[b]
        q.g = ctypes.pointer(gs)
        q.d_W = W.data_ptr()
        q.d_tau = tau_d.data_ptr()
        q.d_active = act_d.data_ptr()
        q.d_active_pos = pos_d.data_ptr()
        q.d_X_out = X.data_ptr()
        q.d_h_out = h.data_ptr() if track else None
        q.d_iters_out = iters.data_ptr()
        q.d_workspace = ws.data_ptr()
        q.workspace_bytes = ws.numel()
        q.tol = float(tols[b])
        q.maxit = int(maxits[b])
        q.cost = float(costs[b]) if costs is not None else batch_cost(G, R, float(np.min(taus[b])))
        q.ldw = W.stride(0) if R > 1 else max(1, W.stride(0))
        q.R = R
        q.p = p
        q.nA = nA
        q.track = 1 if track else 0
        q.x_f32 = 1 if X.dtype == torch.float32 else 0
        q.ldx = R
        keep.append((gs, W, tau_d, act_d, pos_d, ws))
        outs.append((X, h, iters))
    _lib.check(lib.polar_msolve_batch(probs, nb, prec, stream), "polar_msolve_batch")
    infos = []
    err = None
    for b in range(nb):
        inf = _lib.MsolveInfo()
        st = lib.polar_msolve_finish(probs[b].d_workspace, stream, inf)
        infos.append(inf)
        if st != _lib.POLAR_OK and err is None:
            err = (st, b)
    if info is not None:
        info.extend(infos)
    if err is not None:
        _lib.check(err[0], f"polar_msolve_batch (problem {err[1]})")
    del keep
    return [(X, h, iters.cpu().numpy()) for X, h, iters in outs]
