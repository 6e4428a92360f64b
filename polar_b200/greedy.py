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

__all__ = ["polar", "Greedy", "true_marginals", "degree_greedy", "random_set"]

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


class Greedy:
    """One greedy POLAR run on the device (realworld/polar_gpu.py:180-254), advanced a round
    at a time.  The constructor does the uploads the reference does before its timer starts
    (:186-196); `bank()` is :200-206 (the 2q-column solve and the h/t caches); `step()` is one
    pass of the round loop :214-251 and returns the winner's candidate index; `result()`
    gives polar()'s dict.  polar() is the loop over these; a caller that wants per-round
    control (a time budget of its own, timing single rounds) drives it directly."""

    def __init__(self, G, cand, k, s, q=128, B=16, eps=1e-2, tol=1e-7, obj="frac", sketch=None, naive=False,
                 seed=2026, kind="block", trace=None, *, K=None, precision="fp64", width=None, maxit=100000,
                 phases=False):
        if obj not in _OBJ:
            raise ValueError(f"unknown objective {obj!r}")
        self.G = G
        dev = self.dev = G.device
        prec = self.prec = precision_code(precision)
        xdt = torch.float32 if prec == _lib.POLAR_MIXED else torch.float64
        self.x_f32 = 1 if xdt == torch.float32 else 0
        cand = self.cand = np.asarray(cand, dtype=np.int64)
        n, N = G.n, len(cand)
        self.n, self.N, self.k = n, N, int(k)
        self.obj, self.naive, self.B, self.tol, self.maxit, self.trace = obj, naive, B, tol, maxit, trace
        tau, om, _ = poles(obj, s, G.sigma, G.Lam(k), eps, K=K)
        p = self.p = len(tau)
        self.s = s
        if sketch is None:
            sketch = sketches(G, cand, q, seed, kind)
        Z, F, Gc = sketch
        q = self.q = int(Z.shape[1])
        lib = self.lib = _lib.load()
        self.stream = torch.cuda.current_stream(dev).cuda_stream
        # ---- uploads (outside the timed region, as in the reference) ----
        active_h = np.unique(cand)
        es_h = np.searchsorted(active_h, cand).astype(np.int32)
        nA = self.nA = len(active_h)
        self.act_d, self.pos_d = prepare_active(active_h, n, dev)
        self.tau_d = torch.as_tensor(tau, dtype=torch.float64).to(dev)
        self.om_d = torch.as_tensor(om, dtype=torch.float64).to(dev)
        self.cand_d = torch.as_tensor(cand).to(dev)
        self.es_d = torch.as_tensor(es_h).to(dev).contiguous()
        self.ea_d = self.es_d[:, 0].contiguous()
        self.eb_d = self.es_d[:, 1].contiguous()
        self.RHS = torch.empty((n, 2 * q), dtype=torch.float64, device=dev)
        self.RHS[:, :q] = _f64_on(Z, dev)
        self.RHS[:, q:] = _f64_on(F, dev)
        self.Gd = _f64_on(Gc, dev).contiguous()
        self.live_d = torch.ones(N, dtype=torch.uint8, device=dev)
        self.XY = torch.empty((p, nA, 2 * q), dtype=xdt, device=dev)
        self.h = torch.empty((p, N), dtype=torch.float64, device=dev)
        self.t = torch.empty((p, N), dtype=torch.float64, device=dev)
        Bmax = self.Bmax = max(1, min(B, N))
        self.short_d = torch.empty(Bmax, dtype=torch.int64, device=dev)
        self.sscore_d = torch.empty(Bmax, dtype=torch.float64, device=dev)
        self.topb_tmp = torch.empty(lib.polar_topb_tmp_bytes(N, Bmax), dtype=torch.uint8, device=dev)
        self.Wb = torch.empty((n, Bmax), dtype=torch.float64, device=dev)
        self.ia_d = torch.empty(Bmax, dtype=torch.int32, device=dev)
        self.ib_d = torch.empty(Bmax, dtype=torch.int32, device=dev)
        self.U = torch.empty((p, nA, Bmax), dtype=xdt, device=dev)
        self.gq_d = torch.empty(Bmax, dtype=torch.float64, device=dev)
        self.best_d = torch.zeros(1, dtype=torch.int32, device=dev)
        self.win_d = torch.zeros(6, dtype=torch.int32, device=dev)
        self.mtmp = torch.empty(lib.polar_maintain_tmp_bytes(p, nA, q), dtype=torch.uint8, device=dev)
        self.op = Op(G)
        self.cnt = Counter()
        self.live_h = np.ones(N, bool)
        self.seq, self.marg = [], []
        self.shortlists = []  # per recorded round: (shortlist, its proxy scores, its re-rank scores G_q)
        self.solves = []  # (columns, seed iterations) of every multi-shift solve
        self.ph = _Phase(phases)
        self.wd = int(width) if width else min(2 * q, max_columns(prec))
        if self.wd > max_columns(prec):
            raise ValueError("width above the kernel's column limit")
        self.rnd = 0
        self.banked = False
        self.t0 = None

    def bank(self):
        """The 2q-column solve and the h/t caches (polar_gpu.py:200-206)."""
        if self.t0 is None:
            _sync(self.dev)
            self.t0 = time.perf_counter()
        lib, q, p, nA, N = self.lib, self.q, self.p, self.nA, self.N
        self.ph.mark("bank")
        for lo in range(0, 2 * q, self.wd):
            w = min(self.wd, 2 * q - lo)
            inf = []
            msolve(self.op, self.RHS[:, lo:lo + w], self.tau_d, self.act_d, self.tol, maxit=self.maxit,
                   counter=self.cnt, precision=self.prec, out=self.XY, out_col=lo, active_pos=self.pos_d, info=inf)
            self.solves.extend((w, int(i.iterations)) for i in inf)
        for col, dst in ((0, self.h), (q, self.t)):
            _lib.check(lib.polar_pair_norms(self.XY.data_ptr(), self.x_f32, p, nA, 2 * q, col, q, self.ea_d.data_ptr(),
                                            self.eb_d.data_ptr(), N, dst.data_ptr(), self.stream), "pair_norms")
        self.banked = True

    def screen(self, M, exact=False):
        """Keep live only the M candidates with the largest adjoint gradient of the relaxed
        objective at w = 0, d f_s / d w_e = sum_j om_j ||(A + tau_j)^{-1} b_e||^2 (the
        quantity the proxy's numerator sketches), before any proxy or shortlist; ties go to
        the lower index.  exact=False reads it from the bank's caches (sum_j om_j h_je, one
        pass over p x N); exact=True solves for every candidate's b_e (N / 64 multi-shift
        solves, for pools up to ~10^5).  Runs after bank()."""
        if not self.banked:
            self.bank()
        M = int(M)
        if M >= int(self.live_h.sum()):
            return
        if exact:
            from .adjoint import relaxed_gradient
            g = relaxed_gradient(self.G, self.cand, np.zeros(self.N), self.s, tau=self.tau_d.cpu().numpy(),
                                 om=self.om_d.cpu().numpy(), tol=self.tol,
                                 precision="mixed" if self.prec == _lib.POLAR_MIXED else "fp64")
        else:
            buf = torch.empty(self.N, dtype=torch.float64, device=self.dev)
            _lib.check(self.lib.polar_score_topb(self.h.data_ptr(), self.t.data_ptr(), self.tau_d.data_ptr(),
                                                 self.om_d.data_ptr(), self.G.sigma, self.p, self.N,
                                                 self.live_d.data_ptr(), 2, 1, self.short_d.data_ptr(),
                                                 self.sscore_d.data_ptr(), buf.data_ptr(), self.topb_tmp.data_ptr(),
                                                 self.stream), "screen scores")
            g = buf.cpu().numpy()
        g = np.where(self.live_h, g, -np.inf)
        keep = np.argsort(-g, kind="stable")[:M]
        mask = np.zeros(self.N, bool)
        mask[keep] = True
        self.live_h &= mask
        self.live_d.copy_(torch.as_tensor(self.live_h.astype(np.uint8)))
        self.screened = keep

    def step(self, record=False):
        """One round (polar_gpu.py:215-251): proxy + stable top-B, the B-column shortlist
        solve, the re-rank, then the Sherman–Morrison maintenance of the banks and caches
        and the F / operator update.  Returns the winner's candidate index.  record=True
        keeps the round's shortlist with its proxy and re-rank scores in `shortlists`."""
        if not self.banked:
            self.bank()
        if self.rnd >= self.k:
            raise RuntimeError("all k rounds have run")
        lib, p, nA, q, N, n = self.lib, self.p, self.nA, self.q, self.N, self.n
        st = self.stream
        naive, rnd = self.naive, self.rnd
        if naive and rnd:
            self.bank()
        self.ph.mark("score")
        Br = 1 if naive else min(self.B, int(self.live_h.sum()))
        ob = _OBJ[self.obj]
        _lib.check(lib.polar_score_topb(self.h.data_ptr(), self.t.data_ptr(), self.tau_d.data_ptr(),
                                        self.om_d.data_ptr(), self.G.sigma, p, N, self.live_d.data_ptr(), ob, Br,
                                        self.short_d.data_ptr(), self.sscore_d.data_ptr(), None,
                                        self.topb_tmp.data_ptr(), st), "score_topb")
        if naive:
            _lib.check(lib.polar_select(self.short_d.data_ptr(), None, self.es_d.data_ptr(), self.live_d.data_ptr(),
                                        self.win_d.data_ptr(), st), "select")
            win = self.win_d.cpu().numpy()
            e = int(win[4:6].view(np.int64)[0])
            self.marg.append(float(self.sscore_d[0].item()))
            short = [e]
        else:
            self.ph.mark("shortlist")
            _lib.check(lib.polar_fill_incidence(n, Br, self.cand_d.data_ptr(), self.short_d.data_ptr(),
                                                self.es_d.data_ptr(), self.Wb.data_ptr(), self.Bmax,
                                                self.ia_d.data_ptr(), self.ib_d.data_ptr(), st), "fill_incidence")
            inf = []
            Uv, hh, _ = msolve(self.op, self.Wb[:, :Br], self.tau_d, self.act_d, self.tol, maxit=self.maxit,
                               track=(self.obj != "logdet"), counter=self.cnt, precision=self.prec, out=self.U,
                               out_col=0, active_pos=self.pos_d, info=inf)
            self.solves.extend((Br, int(i.iterations)) for i in inf)
            self.ph.mark("select")
            _lib.check(lib.polar_rerank(self.U.data_ptr(), self.x_f32, p, nA, self.Bmax, self.ia_d.data_ptr(),
                                        self.ib_d.data_ptr(), Br, hh.data_ptr() if hh is not None else None,
                                        self.om_d.data_ptr(), ob, self.gq_d.data_ptr(), self.best_d.data_ptr(), st),
                       "rerank")
            _lib.check(lib.polar_select(self.short_d.data_ptr(), self.best_d.data_ptr(), self.es_d.data_ptr(),
                                        self.live_d.data_ptr(), self.win_d.data_ptr(), st), "select")
            win = self.win_d.cpu().numpy()
            e = int(win[4:6].view(np.int64)[0])
            self.marg.append(float(self.gq_d[int(win[0])].item()))
            short = self.short_d[:Br].cpu().tolist() if (self.trace is not None or record) else None
        if record:
            rr = None if naive else self.gq_d[:Br].cpu().numpy().copy()
            self.shortlists.append((list(short), self.sscore_d[:Br].cpu().numpy().copy(), rr))
        if self.trace is not None:
            self.trace.append(dict(shortlist=[int(x) for x in short], chosen=e))
        self.seq.append(e)
        self.live_h[e] = False
        a, b = int(self.cand[e, 0]), int(self.cand[e, 1])
        if not naive and rnd + 1 < self.k:
            self.ph.mark("maintain")
            XY = self.XY
            _lib.check(lib.polar_maintain(XY.data_ptr(), 2 * q, XY[:, :, q:].data_ptr(), 2 * q, self.x_f32, p, nA, q,
                                          self.U.data_ptr(), self.x_f32, self.Bmax, self.win_d.data_ptr(),
                                          self.Gd.data_ptr(), self.es_d.data_ptr(), N, self.h.data_ptr(),
                                          self.t.data_ptr(), self.mtmp.data_ptr(), st), "maintain")
        _lib.check(lib.polar_rank1_rows(self.RHS[:, q:].data_ptr(), 2 * q, q, self.Gd.data_ptr(),
                                        self.cand_d.data_ptr(), self.win_d[4:].data_ptr(), st), "rank1_rows")
        self.op.add(a, b)
        self.rnd += 1
        return e

    def result(self):
        """polar()'s dict for the rounds run so far."""
        self.ph.mark("end")
        _sync(self.dev)
        seconds = time.perf_counter() - self.t0 if self.t0 is not None else 0.0
        out = dict(sequence=list(self.seq), seconds=seconds, spmv=self.cnt.spmv, rhs=self.cnt.rhs, p=self.p,
                   rounds=len(self.seq), truncated=len(self.seq) < self.k, marginals=list(self.marg),
                   precision="mixed" if self.prec == _lib.POLAR_MIXED else "fp64", solves=list(self.solves))
        if self.ph.enabled:
            out["phases"] = self.ph.summary()
        return out


def polar(G, cand, k, s, q=128, B=16, eps=1e-2, tol=1e-7, obj="frac", sketch=None, naive=False, seed=2026,
          kind="block", trace=None, time_limit=None, *, K=None, precision="fp64", width=None, maxit=100000,
          phases=False, screen=None, screen_exact=False):
    """Greedy POLAR (realworld/polar_gpu.py:180-254).  Returns the reference keys
    (sequence, seconds, spmv, rhs, p, rounds, truncated) plus `marginals`: the re-rank value
    G_q(e*) of each round's winner (naive rounds: the proxy value), and `precision`.
    screen=M: after the bank, only the M candidates with the largest adjoint gradient
    d f_s / d w_e stay in the pool (Greedy.screen); None keeps the reference's path."""
    g = Greedy(G, cand, k, s, q=q, B=B, eps=eps, tol=tol, obj=obj, sketch=sketch, naive=naive, seed=seed, kind=kind,
               trace=trace, K=K, precision=precision, width=width, maxit=maxit, phases=phases)
    g.bank()
    if screen is not None:
        if obj != "frac" or naive:
            raise ValueError("the gradient screen applies to obj='frac' without naive re-banking")
        g.screen(screen, exact=screen_exact)
    for rnd in range(g.k):
        if rnd and time_limit is not None and time.perf_counter() - g.t0 > time_limit:
            break
        g.step()
    return g.result()


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
