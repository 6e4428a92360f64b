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
  on the growing operator.  Edges are added a group of g at a time (Woodbury, see
  relaxed_objective): one g-column solve with every row active per group, so 4,096
  candidates cost 64 solves rather than 4,096.
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

__all__ = ["relaxed_rule", "relaxed_gradient", "relaxed_objective", "relaxed_central_difference", "FracTrace"]


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
                      precision="fp64", maxit=100000, with_next=False, group=None):
    """f_s(w, sigma = G.sigma + dsigma).  With with_next, also returns f_{s+1}, so that
    d f_s / d sigma = -s f_{s+1}.

    The weighted edges join the operator a group at a time (group = the solver's column
    limit by default; group=1 is the plain rank-one chain).  For a group with incidence
    block B and weights W on the operator A built so far, Woodbury gives, per shift t,
        Tr((A + t)^{-1}) - Tr((A + B W B^T + t)^{-1}) = Tr(C^{-1} U^T U),
        U = (A + t)^{-1} B,   C = W^{-1} + B^T U,
    so one multi-shift solve of the group's columns with every row active (U in full) and a
    g x g Gram product per shift replace g sequential single-column solves."""
    cand, w = _check_cand(G, cand, w)
    if group is None:
        group = max_columns(precision_code(precision))
    if group > 1:
        return _objective_grouped(G, cand, w, s, K=K, eps=eps, tau=tau, om=om, dsigma=dsigma, tol=tol,
                                  precision=precision, maxit=maxit, with_next=with_next, group=int(group))
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


def _objective_grouped(G, cand, w, s, *, K, eps, tau, om, dsigma, tol, precision, maxit, with_next, group):
    if tau is None:
        tau, om = relaxed_rule(G, s, K=K, eps=eps)
    tau = np.asarray(tau, np.float64)
    om = np.asarray(om, np.float64)
    dev = G.device
    shifts = np.concatenate([[0.0], tau]) + dsigma  # ascending: the zero shift is the seed
    shifts_d = torch.as_tensor(shifts, device=dev)
    keep = np.flatnonzero(w != 0.0)
    all_rows = np.arange(G.n)
    act_d, pos_d = prepare_active(all_rows, G.n, dev)
    phi = torch.zeros(len(shifts), dtype=torch.float64, device=dev)
    op = Op(G)
    for lo in range(0, len(keep), group):
        idx = keep[lo:lo + group]
        g = len(idx)
        ca = torch.as_tensor(cand[idx, 0], device=dev)
        cb = torch.as_tensor(cand[idx, 1], device=dev)
        cols = torch.arange(g, device=dev)
        Bm = torch.zeros((G.n, g), dtype=torch.float64, device=dev)
        Bm[ca, cols] = 1.0
        Bm[cb, cols] = -1.0
        X, _, _ = msolve(op, Bm, shifts_d, act_d, tol, maxit=maxit, precision=precision, active_pos=pos_d)
        U = X.double()                                   # [shifts, n, g], rows in vertex order
        S = U[:, ca, :] - U[:, cb, :]                    # B^T U: [shifts, g, g]
        S = 0.5 * (S + S.transpose(1, 2))
        Gm = torch.matmul(U.transpose(1, 2), U)          # U^T U
        C = S + torch.diag(torch.as_tensor(1.0 / w[idx], device=dev))[None]
        L = torch.linalg.cholesky(C)
        phi += torch.einsum("jii->j", torch.cholesky_solve(Gm, L))
        del X, U, S, Gm, C, L
        for e in idx:
            op.add(int(cand[e, 0]), int(cand[e, 1]), float(w[e]))
    phi = phi.cpu().numpy()
    f = float(np.dot(om, phi[1:]))
    if not with_next:
        return f
    f_next = float(np.dot(om / tau, phi[0] - phi[1:]))
    return f, f_next


def relaxed_central_difference(G, cand, w, s, i, h=1e-4, *, K=24, eps=1e-2, tau=None, om=None, tol=1e-12,
                               precision="fp64", maxit=100000):
    """(f(w + h e_i) - f(w - h e_i)) / (2h) for one candidate i, from a solve that does not
    share the gradient's: with edge i ordered last, f(w +- h e_i) differ only in its own
    rank-one term, so with u = (A_{w without i} + tau_j)^{-1} b_i (h' = ||u||^2, t' = b_i^T u)
        f(w + d e_i) - f(w - d e_i) = sum_j om_j [(w_i + d) h' / (1 + (w_i + d) t')
                                               - (w_i - d) h' / (1 + (w_i - d) t')]
    exactly under the quadrature rule.  Needs w_i >= h."""
    cand, w = _check_cand(G, cand, w)
    if tau is None:
        tau, om = relaxed_rule(G, s, K=K, eps=eps)
    if w[i] < h:
        raise ValueError("central difference needs w_i >= h")
    w_wo = w.copy()
    w_wo[i] = 0.0
    op = _relaxed_op(G, cand, w_wo)
    a, b = int(cand[i, 0]), int(cand[i, 1])
    col = torch.zeros((G.n, 1), dtype=torch.float64, device=G.device)
    col[a, 0] = 1.0
    col[b, 0] = -1.0
    act = np.array(sorted((a, b)))
    X, hh, _ = msolve(op, col, torch.as_tensor(np.asarray(tau, np.float64), device=G.device), act, tol,
                      maxit=maxit, track=True, precision=precision)
    Xh = X[:, :, 0].double().cpu().numpy()
    ia, ib = (0, 1) if a < b else (1, 0)
    t = Xh[:, ia] - Xh[:, ib]
    hh = hh[:, 0].cpu().numpy()
    up, dn = w[i] + h, w[i] - h
    return float(np.dot(om, up * hh / (1.0 + up * t) - dn * hh / (1.0 + dn * t)) / (2.0 * h))


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
