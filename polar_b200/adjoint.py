"""Relaxed-weight objective and its adjoint (the differentiation path of the solve-and-score
operator).

For candidate edges e = (a_e, b_e) with relaxed weights w_e in [0, 1] and b_e = e_a - e_b:

    A_0 = L + sigma I,   A_w = A_0 + sum_e w_e b_e b_e^T,
    f_s(w, sigma) = Tr(A_0^{-s}) - Tr(A_w^{-s}),

with A^{-s} ~= sum_j om_j (A + tau_j I)^{-1}, the same positive Stieltjes rule (tau, om)
as the greedy (realworld/polar_gpu.py:18-43; `poles(..., K=K)` for a fixed pole count).

* Gradient in w (the adjoint).  d f_s / d w_e = s b_e^T A_w^{-s-1} b_e, which under the
  rule is  sum_j om_j ||(A_w + tau_j I)^{-1} b_e||^2.  These are the tracked norms h_j of
  ONE multi-shift solve with every candidate's b_e as a right-hand side on the relaxed
  operator.  This is the quantity whose sketch is the greedy's proxy numerator
  (realworld/polar_gpu.py:205, 211), computed exactly.
* Value.  Adding the weighted edges one at a time, each rank-one step is exact by
  Sherman-Morrison (realworld/polar_gpu.py:229-237):
      Tr((M + tau)^{-1}) - Tr((M + w b b^T + tau)^{-1}) = w h / (1 + w t),
  with h = ||u||^2, t = b^T u, u = (M + tau)^{-1} b.  So f_s is a sum of per-edge terms
  from single-column multi-shift solves on the growing operator.
* Gradient in sigma.  d f_s / d sigma = -s f_{s+1}.  From x^{-(s+1)} = x^{-1} x^{-s} and
  partial fractions over the same poles,
      x^{-(s+1)} ~= sum_j (om_j / tau_j) (x^{-1} - (x + tau_j)^{-1}),
  so f_{s+1} is obtained from the same chain with one extra zero shift.

Everything runs through polar_b200.msolve (the CUDA multi-shift CG).  Only obj = 'frac'
(0 < s < 1, all tau_j > 0) is supported.
"""
import math

import numpy as np
import torch

from . import _lib
from .graph import Op
from .quadrature import poles
from .solver import max_columns, msolve, precision_code, prepare_active

__all__ = ["relaxed_rule", "relaxed_gradient", "relaxed_objective", "FracTrace"]


def relaxed_rule(G, s, K=24, eps=1e-2, k=0):
    """(tau, om) for the relaxed objective: the greedy's rule for Lam(k) (all tau_j > 0)."""
    if not 0.0 < s < 1.0:
        raise ValueError("relaxed objective needs 0 < s < 1")
    tau, om, _ = poles("frac", s, G.sigma, G.Lam(k), eps, K=K)
    if np.any(tau <= 0.0):
        raise ValueError("rule has a non-positive pole")
    return np.asarray(tau, np.float64), np.asarray(om, np.float64)


def _check_cand(G, cand, w):
    cand = np.asarray(cand, dtype=np.int64).reshape(-1, 2)
    w = np.asarray(w, dtype=np.float64).reshape(-1)
    if len(w) != len(cand):
        raise ValueError("one weight per candidate")
    if len(cand) and (cand.min() < 0 or cand.max() >= G.n or np.any(cand[:, 0] == cand[:, 1])):
        raise ValueError("candidate endpoints out of range or equal")
    if np.any(w < 0.0):
        raise ValueError("weights must be non-negative")
    return cand, w


def _relaxed_op(G, cand, w):
    op = Op(G)
    for (a, b), we in zip(cand, w):
        if we != 0.0:
            op.add(int(a), int(b), float(we))
    return op


def relaxed_gradient(G, cand, w, s, *, K=24, eps=1e-2, tau=None, om=None, dsigma=0.0, tol=1e-10,
                     precision="fp64", maxit=100000):
    """d f_s / d w_e for every candidate at (w, sigma = G.sigma + dsigma): float64 (m,) on the
    host.  One multi-shift solve per block of candidate columns on the relaxed operator."""
    cand, w = _check_cand(G, cand, w)
    if tau is None:
        tau, om = relaxed_rule(G, s, K=K, eps=eps)
    m = len(cand)
    if m == 0:
        return np.zeros(0)
    dev = G.device
    op = _relaxed_op(G, cand, w)
    ends = np.unique(cand.ravel())
    act_d, pos_d = prepare_active(ends, G.n, dev)
    shifts = torch.as_tensor(np.asarray(tau, np.float64) + dsigma, device=dev)
    om_d = torch.as_tensor(np.asarray(om, np.float64), device=dev)
    grad = np.empty(m)
    width = max_columns(precision_code(precision))
    ca = torch.as_tensor(cand[:, 0], device=dev)
    cb = torch.as_tensor(cand[:, 1], device=dev)
    for lo in range(0, m, width):
        hi = min(m, lo + width)
        r = hi - lo
        W = torch.zeros((G.n, r), dtype=torch.float64, device=dev)
        cols = torch.arange(r, device=dev)
        W[ca[lo:hi], cols] = 1.0
        W[cb[lo:hi], cols] = -1.0
        _, h, _ = msolve(op, W, shifts, act_d, tol, maxit=maxit, track=True, precision=precision,
                         active_pos=pos_d)
        grad[lo:hi] = (om_d[:, None] * h).sum(0).cpu().numpy()
    return grad


def relaxed_objective(G, cand, w, s, *, K=24, eps=1e-2, tau=None, om=None, dsigma=0.0, tol=1e-10,
                      precision="fp64", maxit=100000, with_next=False):
    """f_s(w, sigma = G.sigma + dsigma) by the rank-one chain (one single-column multi-shift
    solve per candidate with w_e > 0, in the given order).  With with_next, also returns
    f_{s+1}, so that d f_s / d sigma = -s f_{s+1}."""
    cand, w = _check_cand(G, cand, w)
    if tau is None:
        tau, om = relaxed_rule(G, s, K=K, eps=eps)
    tau = np.asarray(tau, np.float64)
    om = np.asarray(om, np.float64)
    dev = G.device
    shifts = np.concatenate([[0.0], tau]) + dsigma  # ascending: the zero shift is the seed
    shifts_d = torch.as_tensor(shifts, device=dev)
    phi = np.zeros(len(shifts))  # Tr((A_0 + t)^{-1}) - Tr((A_w + t)^{-1}) per shift t
    op = Op(G)
    for (a, b), we in zip(cand, w):
        if we == 0.0:
            continue
        a, b = int(a), int(b)
        col = torch.zeros((G.n, 1), dtype=torch.float64, device=dev)
        col[a, 0] = 1.0
        col[b, 0] = -1.0
        act = np.array(sorted((a, b)))
        X, h, _ = msolve(op, col, shifts_d, act, tol, maxit=maxit, track=True, precision=precision)
        Xh = X[:, :, 0].double().cpu().numpy()
        ia, ib = (0, 1) if a < b else (1, 0)
        t = Xh[:, ia] - Xh[:, ib]
        hh = h[:, 0].cpu().numpy()
        phi += we * hh / (1.0 + we * t)
        op.add(a, b, float(we))
    f = float(np.dot(om, phi[1:]))
    if not with_next:
        return f
    f_next = float(np.dot(om / tau, phi[0] - phi[1:]))
    return f, f_next


class FracTrace(torch.autograd.Function):
    """f_s(w, sigma) with its adjoint.

    forward(w, sigma, G, cand, s, K, tol, precision): w float64 (m,) tensor, sigma a 0-d
    float64 tensor; returns the 0-d tensor f_s.  backward gives d f/d w (the multi-shift
    adjoint) and d f/d sigma = -s f_{s+1}.  The quadrature rule is fixed by G's own sigma, so
    sigma enters as a shift of every pole."""

    @staticmethod
    def forward(ctx, w, sigma, G, cand, s, K=24, tol=1e-10, precision="fp64"):
        wh = w.detach().double().cpu().numpy()
        ds = float(sigma.detach().cpu()) - G.sigma
        tau, om = relaxed_rule(G, s, K=K)
        f, f_next = relaxed_objective(G, cand, wh, s, tau=tau, om=om, dsigma=ds, tol=tol, precision=precision,
                                      with_next=True)
        ctx.args = (G, np.asarray(cand), wh, s, tau, om, ds, tol, precision, f_next)
        return torch.tensor(f, dtype=torch.float64)

    @staticmethod
    def backward(ctx, gout):
        G, cand, wh, s, tau, om, ds, tol, precision, f_next = ctx.args
        gw = gsig = None
        if ctx.needs_input_grad[0]:
            g = relaxed_gradient(G, cand, wh, s, tau=tau, om=om, dsigma=ds, tol=tol, precision=precision)
            gw = gout * torch.as_tensor(g, dtype=torch.float64)
        if ctx.needs_input_grad[1]:
            gsig = gout * torch.tensor(-s * f_next, dtype=torch.float64)
        return gw, gsig, None, None, None, None, None, None
