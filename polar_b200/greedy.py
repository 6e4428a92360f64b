"""Greedy POLAR driver on the device: realworld/polar_gpu.py:180-254 (polar) and
:273-291 (true_marginals), with every per-round step in libpolar kernels.

Round structure (one host<->device synchronisation per round, to learn the winner):
  polar_score_topb   proxy G^_e for all candidates + stable top-B shortlist
  polar_fill_incidence + polar_msolve   B incidence solves (all poles, tracked norms)
  polar_rerank       G_q(e) = sum_j om_j hh_j / (1 + b^T u_j) and its first maximum
  polar_select       winner record, live mask
  polar_maintain     Sherman–Morrison update of the X/Y banks and the h/t caches
  polar_rank1_rows   F[a] += Gc[e]; F[b] -= Gc[e]
"""
import time

import numpy as np
import torch

from . import _lib
from .graph import Op
from .quadrature import poles
from .sketch import sketches
from .solver import Counter, max_columns, msolve, precision_code, prepare_active

__all__ = ["polar", "true_marginals", "degree_greedy", "random_set"]

_OBJ = {"frac": 0, "er": 0, "logdet": 1}


def _sync(dev):
    torch.cuda.synchronize(dev)


class _Phase:
    """CUDA-event timing of the greedy's phases (bank / shortlist solves / other)."""

    def __init__(self, enabled):
        self.enabled = enabled
        self.events = []

    def mark(self, name):
        if self.enabled:
            ev = torch.cuda.Event(enable_timing=True)
            ev.record()
            self.events.append((name, ev))

    def summary(self):
        if not self.enabled or len(self.events) < 2:
            return {}
        torch.cuda.synchronize()
        out = {}
        for (n0, e0), (_, e1) in zip(self.events[:-1], self.events[1:]):
            out[n0] = out.get(n0, 0.0) + e0.elapsed_time(e1) / 1e3
        return out


def _f64_on(x, dev):
    """A sketch array (host NumPy, or a device tensor from sketches(..., device=True)) as
    a float64 tensor on `dev`."""
    if isinstance(x, torch.Tensor):
        return x.to(device=dev, dtype=torch.float64)
    return torch.as_tensor(np.ascontiguousarray(x, dtype=np.float64)).to(dev)


def polar(G, cand, k, s, q=128, B=16, eps=1e-2, tol=1e-7, obj="frac", sketch=None, naive=False, seed=2026,
          kind="block", trace=None, time_limit=None, *, K=None, precision="fp64", width=None, maxit=100000,
          phases=False):
    """Greedy POLAR (realworld/polar_gpu.py:180-254).  Returns the reference keys
    (sequence, seconds, spmv, rhs, p, rounds, truncated) plus `marginals`: the re-rank value
    G_q(e*) of each round's winner (naive rounds: the proxy value), and `precision`."""
    if obj not in _OBJ:
        raise ValueError(f"unknown objective {obj!r}")
    dev = G.device
    prec = precision_code(precision)
    xdt = torch.float32 if prec == _lib.POLAR_MIXED else torch.float64
    x_f32 = 1 if xdt == torch.float32 else 0
    cand = np.asarray(cand, dtype=np.int64)
    n, N = G.n, len(cand)
    sigma = G.sigma
    tau, om, _ = poles(obj, s, sigma, G.Lam(k), eps, K=K)
    p = len(tau)
    if sketch is None:
        sketch = sketches(G, cand, q, seed, kind)
    Z, F, Gc = sketch
    q = int(Z.shape[1])
    lib = _lib.load()
    stream = torch.cuda.current_stream(dev).cuda_stream

    # ---- uploads (outside the timed region, as in the reference) ----
    active_h = np.unique(cand)
    es_h = np.searchsorted(active_h, cand).astype(np.int32)
    nA = len(active_h)
    act_d, pos_d = prepare_active(active_h, n, dev)
    tau_d = torch.as_tensor(tau, dtype=torch.float64).to(dev)
    om_d = torch.as_tensor(om, dtype=torch.float64).to(dev)
    cand_d = torch.as_tensor(cand).to(dev)
    es_d = torch.as_tensor(es_h).to(dev).contiguous()
    ea_d = es_d[:, 0].contiguous()
    eb_d = es_d[:, 1].contiguous()
    RHS = torch.empty((n, 2 * q), dtype=torch.float64, device=dev)
    RHS[:, :q] = _f64_on(Z, dev)
    RHS[:, q:] = _f64_on(F, dev)
    Gd = _f64_on(Gc, dev).contiguous()
    live_d = torch.ones(N, dtype=torch.uint8, device=dev)
    XY = torch.empty((p, nA, 2 * q), dtype=xdt, device=dev)
    h = torch.empty((p, N), dtype=torch.float64, device=dev)
    t = torch.empty((p, N), dtype=torch.float64, device=dev)
    Bmax = max(1, min(B, N))
    short_d = torch.empty(Bmax, dtype=torch.int64, device=dev)
    sscore_d = torch.empty(Bmax, dtype=torch.float64, device=dev)
    topb_tmp = torch.empty(lib.polar_topb_tmp_bytes(N, Bmax), dtype=torch.uint8, device=dev)
    Wb = torch.empty((n, Bmax), dtype=torch.float64, device=dev)
    ia_d = torch.empty(Bmax, dtype=torch.int32, device=dev)
    ib_d = torch.empty(Bmax, dtype=torch.int32, device=dev)
    U = torch.empty((p, nA, Bmax), dtype=xdt, device=dev)
    gq_d = torch.empty(Bmax, dtype=torch.float64, device=dev)
    best_d = torch.zeros(1, dtype=torch.int32, device=dev)
    win_d = torch.zeros(6, dtype=torch.int32, device=dev)
    mtmp = torch.empty(lib.polar_maintain_tmp_bytes(p, nA, q), dtype=torch.uint8, device=dev)
    op = Op(G)
    cnt = Counter()
    live_h = np.ones(N, bool)
    seq, marg = [], []
    solves = []  # (columns, seed iterations) of every multi-shift solve
    ph = _Phase(phases)
    wd = int(width) if width else min(2 * q, max_columns(prec))
    if wd > max_columns(prec):
        raise ValueError("width above the kernel's column limit")
    _sync(dev)
    t0 = time.perf_counter()
    ph.mark("bank")

    def bank():
        for lo in range(0, 2 * q, wd):
            w = min(wd, 2 * q - lo)
            inf = []
            msolve(op, RHS[:, lo:lo + w], tau_d, act_d, tol, maxit=maxit, counter=cnt, precision=prec, out=XY,
                   out_col=lo, active_pos=pos_d, info=inf)
            solves.extend((w, int(i.iterations)) for i in inf)
        _lib.check(lib.polar_pair_norms(XY.data_ptr(), x_f32, p, nA, 2 * q, 0, q, ea_d.data_ptr(), eb_d.data_ptr(), N,
                                        h.data_ptr(), stream), "pair_norms")
        _lib.check(lib.polar_pair_norms(XY.data_ptr(), x_f32, p, nA, 2 * q, q, q, ea_d.data_ptr(), eb_d.data_ptr(), N,
                                        t.data_ptr(), stream), "pair_norms")

    bank()
    ob = _OBJ[obj]
    for rnd in range(k):
        if rnd and time_limit is not None and time.perf_counter() - t0 > time_limit:
            break
        if naive and rnd:
            ph.mark("bank")
            bank()
        ph.mark("score")
        Br = 1 if naive else min(B, int(live_h.sum()))
        _lib.check(lib.polar_score_topb(h.data_ptr(), t.data_ptr(), tau_d.data_ptr(), om_d.data_ptr(), sigma, p, N,
                                        live_d.data_ptr(), ob, Br, short_d.data_ptr(), sscore_d.data_ptr(), None,
                                        topb_tmp.data_ptr(), stream), "score_topb")
        if naive:
            _lib.check(lib.polar_select(short_d.data_ptr(), None, es_d.data_ptr(), live_d.data_ptr(), win_d.data_ptr(),
                                        stream), "select")
            win = win_d.cpu().numpy()
            e = int(win[4:6].view(np.int64)[0])
            marg.append(float(sscore_d[0].item()))
            short = [e]
        else:
            ph.mark("shortlist")
            _lib.check(lib.polar_fill_incidence(n, Br, cand_d.data_ptr(), short_d.data_ptr(), es_d.data_ptr(),
                                                Wb.data_ptr(), Bmax, ia_d.data_ptr(), ib_d.data_ptr(), stream),
                       "fill_incidence")
            inf = []
            Uv, hh, _ = msolve(op, Wb[:, :Br], tau_d, act_d, tol, maxit=maxit, track=(obj != "logdet"),
                               counter=cnt, precision=prec, out=U, out_col=0, active_pos=pos_d, info=inf)
            solves.extend((Br, int(i.iterations)) for i in inf)
            ph.mark("select")
            _lib.check(lib.polar_rerank(U.data_ptr(), x_f32, p, nA, Bmax, ia_d.data_ptr(), ib_d.data_ptr(), Br,
                                        hh.data_ptr() if hh is not None else None, om_d.data_ptr(), ob,
                                        gq_d.data_ptr(), best_d.data_ptr(), stream), "rerank")
            _lib.check(lib.polar_select(short_d.data_ptr(), best_d.data_ptr(), es_d.data_ptr(), live_d.data_ptr(),
                                        win_d.data_ptr(), stream), "select")
            win = win_d.cpu().numpy()
            e = int(win[4:6].view(np.int64)[0])
            marg.append(float(gq_d[int(win[0])].item()))
            short = short_d[:Br].cpu().tolist() if trace is not None else None
        if trace is not None:
            trace.append(dict(shortlist=[int(x) for x in short], chosen=e))
        seq.append(e)
        live_h[e] = False
        a, b = int(cand[e, 0]), int(cand[e, 1])
        if not naive and rnd + 1 < k:
            ph.mark("maintain")
            _lib.check(lib.polar_maintain(XY.data_ptr(), 2 * q, XY[:, :, q:].data_ptr(), 2 * q, x_f32, p, nA, q,
                                          U.data_ptr(), x_f32, Bmax, win_d.data_ptr(), Gd.data_ptr(), es_d.data_ptr(),
                                          N, h.data_ptr(), t.data_ptr(), mtmp.data_ptr(), stream), "maintain")
        _lib.check(lib.polar_rank1_rows(RHS[:, q:].data_ptr(), 2 * q, q, Gd.data_ptr(), cand_d.data_ptr(),
                                        win_d[4:].data_ptr(), stream), "rank1_rows")
        op.add(a, b)
    ph.mark("end")
    _sync(dev)
    seconds = time.perf_counter() - t0
    out = dict(sequence=seq, seconds=seconds, spmv=cnt.spmv, rhs=cnt.rhs, p=p, rounds=len(seq),
               truncated=len(seq) < k, marginals=marg, precision="mixed" if prec == _lib.POLAR_MIXED else "fp64",
               solves=solves)
    if phases:
        out["phases"] = ph.summary()
    return out


def true_marginals(G, cand, seq, s, obj="frac", eps=1e-9, tol=1e-10, kmax=None, *, K=None, precision="fp64",
                   maxit=100000):
    """Certified marginals along a sequence (realworld/polar_gpu.py:273-291): one
    single-column multi-shift solve per edge with the eps quadrature, then
    g = sum_j om_j hh_j / (1 + b^T u_j); the edge then joins the operator."""
    dev = G.device
    cand = np.asarray(cand, dtype=np.int64)
    kmax = kmax or len(seq)
    tau, om, qerr = poles(obj, s, G.sigma, G.Lam(kmax), eps, K=K)
    tau_d = torch.as_tensor(tau, dtype=torch.float64).to(dev)
    om_d = torch.as_tensor(om, dtype=torch.float64).to(dev)
    op = Op(G)
    cnt = Counter()
    out = []
    lib = _lib.load()
    stream = torch.cuda.current_stream(dev).cuda_stream
    prec = precision_code(precision)
    x_f32 = 1 if prec == _lib.POLAR_MIXED else 0
    W = torch.empty((G.n, 1), dtype=torch.float64, device=dev)
    ia = torch.zeros(1, dtype=torch.int32, device=dev)
    ib = torch.ones(1, dtype=torch.int32, device=dev)
    gq = torch.empty(1, dtype=torch.float64, device=dev)
    best = torch.empty(1, dtype=torch.int32, device=dev)
    cand_d = torch.as_tensor(cand).to(dev)
    sel = torch.empty(1, dtype=torch.int64, device=dev)
    for e in seq:
        a, b = int(cand[e, 0]), int(cand[e, 1])
        sel.fill_(int(e))
        _lib.check(lib.polar_fill_incidence(G.n, 1, cand_d.data_ptr(), sel.data_ptr(), None, W.data_ptr(), 1, None,
                                            None, stream), "fill_incidence")
        act = np.array(sorted((a, b)), dtype=np.int64)
        U, hh, _ = msolve(op, W, tau_d, act, tol, maxit=maxit, track=obj != "logdet", counter=cnt, precision=prec)
        if a > b:  # active rows are sorted; b^T u = u[a] - u[b]
            ia.fill_(1)
            ib.fill_(0)
        else:
            ia.fill_(0)
            ib.fill_(1)
        _lib.check(lib.polar_rerank(U.data_ptr(), x_f32, len(tau), 2, 1, ia.data_ptr(), ib.data_ptr(), 1,
                                    hh.data_ptr() if hh is not None else None, om_d.data_ptr(), _OBJ[obj],
                                    gq.data_ptr(), best.data_ptr(), stream), "rerank")
        out.append(float(gq.item()))
        op.add(a, b)
    rho = tol * float(np.max((G.Lam(kmax) + tau) / (G.sigma + tau)))
    return np.array(out), dict(quadrature_bound=qerr, residual_rho=rho, p=len(tau), spmv=cnt.spmv)


def degree_greedy(G, cand, k):
    """Degree-sum baseline (realworld/polar_gpu.py:258-265); host-side, not on the hot path."""
    deg = np.bincount(G.edges[:, 0], G.weights, G.n) + np.bincount(G.edges[:, 1], G.weights, G.n)
    cand = np.asarray(cand)
    live = np.ones(len(cand), bool)
    seq = []
    for _ in range(k):
        val = np.where(live, deg[cand[:, 0]] + deg[cand[:, 1]], np.inf)
        e = int(np.argmin(val))
        seq.append(e)
        live[e] = False
        deg[cand[e, 0]] += 1
        deg[cand[e, 1]] += 1
    return seq


def random_set(cand, k, seed):
    """Random baseline (realworld/polar_gpu.py:268-269)."""
    return np.random.default_rng(seed).choice(len(cand), k, replace=False).tolist()
