"""Autotuner for the solver's SpMM layout: lanes per row, rows per warp and the heavy-row
split, picked per (graph, precision, width) by timing short solves on the device.

The reference launches its CSR kernel with one fixed shape (realworld/spmm.py:19-25: one
warp per row, 32 columns per pass).  Here the multi-shift CG's SpMM has three knobs:

* lane bytes (16, 32 or 64): each lane of a row group owns that many bytes of a row, so a
  row of R columns takes R * elem / bytes lanes and a warp holds 32 / lanes rows;
* the sliced-ELL copy of the light rows (on: warps read the neighbour lists of their rows
  slice-wise; off: CSR row loop);
* the heavy-row threshold, as a multiple (4, 8, 16, 32 or 128) of the lanes per row: rows
  above it are cut into chunks of at most 256 neighbours, one warp each.

tune_msolve times `iters` iterations of the real solver (kernel-per-phase driver, CUDA
graph blocks) for every combination and records the fastest; msolve then applies the
recorded choice (kept on the Graph object) whenever it solves that graph at that width.  Results are identical up to
summation order (the heavy split changes which partial sums are formed).
"""
import time

import numpy as np
import torch

from . import _lib
from . import solver as _solver

__all__ = ["tune_msolve", "tuned", "record", "clear"]

LANE_BYTES = (16, 32, 64)
HEAVY_MULT = (4, 8, 16, 32, 128)


def _ld(prec, R):
    return _solver._padded(prec, R)


def tuned(G, precision, R):
    """The recorded (lane_bytes, sell, heavy_thresh) for this graph and width, or None."""
    prec = _solver.precision_code(precision)
    return _solver.tuned_layouts(G).get((int(prec), _ld(prec, R)))


def record(G, precision, R, layout):
    """Use `layout` = (lane_bytes, sell, heavy_thresh) for this graph's R-column solves."""
    prec = _solver.precision_code(precision)
    _solver.tuned_layouts(G)[(int(prec), _ld(prec, R))] = tuple(int(x) for x in layout)


def clear(G):
    """Forget the graph's recorded layouts (the solver's automatic layout applies)."""
    _solver.tuned_layouts(G).clear()


def _lanes(prec, ld, lb):
    """Lanes per row for `lb` lane bytes, as the solver resolves it (at least one vector
    per lane, at most the row, at most 32 lanes)."""
    elem = 4 if prec == _lib.POLAR_MIXED else 8
    vec = min(ld, 4 if prec == _lib.POLAR_MIXED else 2)
    cpl = min(max(lb // elem, vec), ld)
    while ld // cpl > 32:
        cpl *= 2
    return ld // cpl


def tune_msolve(op, R, precision="mixed", p=8, iters=64, reps=2, lane_bytes=LANE_BYTES, heavy_mult=HEAVY_MULT,
                sells=(1, 0), seed=0):
    """Time every layout for R-column solves of `op`'s graph and record the fastest.

    Returns {"best": (lane_bytes, sell, heavy_thresh), "us_per_iter": float,
             "table": [(lane_bytes, sell, heavy_thresh, us_per_iter), ...]}."""
    G = op.G
    prec = _solver.precision_code(precision)
    ld = _ld(prec, R)
    dev = G.device
    rng = np.random.default_rng(seed)
    W = torch.as_tensor(rng.normal(size=(G.n, R))).to(dev)
    tau = np.concatenate([[0.0], np.geomspace(1e-2, 1e2, p - 1)])
    active = np.arange(0, G.n, max(1, G.n // 1024))
    act_d, pos_d = _solver.prepare_active(active, G.n, dev)
    reg = _solver.tuned_layouts(G)
    key = (int(prec), ld)
    saved = reg.pop(key, None)
    table = []
    seen = set()
    try:
        for lb in lane_bytes:
            lanes = _lanes(prec, ld, lb)
            if lanes in seen:
                continue  # same effective layout as a smaller lane width already timed
            seen.add(lanes)
            for sell in sells:
                if sell and G.weighted:
                    continue
                for hm in heavy_mult:
                    thresh = max(16, hm * lanes)
                    reg[key] = (lb, sell, thresh)
                    best = None
                    for _ in range(reps + 1):
                        torch.cuda.synchronize()
                        t0 = time.perf_counter()
                        try:
                            _solver.msolve(op, W, tau, act_d, 0.0, maxit=iters, precision=prec, active_pos=pos_d)
                        except _lib.PolarError as e:
                            if e.status != _lib.POLAR_ERR_ITER_CAP:
                                raise
                            # tol 0: every run stops at the iteration cap
                        torch.cuda.synchronize()
                        dt = (time.perf_counter() - t0) / iters * 1e6
                        best = dt if best is None else min(best, dt)
                    table.append((lb, sell, thresh, best))
    finally:
        reg.pop(key, None)
        if saved is not None:
            reg[key] = saved
    lb, sell, thresh, us = min(table, key=lambda t: t[3])
    reg[key] = (lb, sell, thresh)
    return {"best": (lb, sell, thresh), "us_per_iter": us, "table": table}
