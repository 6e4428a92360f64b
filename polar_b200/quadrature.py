"""Positive Stieltjes quadrature poles (host side; a few hundred scalars).

x^-s = sin(pi s)/pi * int_0^inf t^-s / (x + t) dt  is discretised as  sum_j om_j / (x + tau_j)
with every om_j > 0, so (M + tau_j I)^-1 solves give M^-s and its derivatives.

Two rules:
* `composite(s, a, z, eps)` — the composite rule of realworld/polar_gpu.py:18-36:
  r = ceil(log(256/eps)/log 4) nodes per panel, a Gauss–Jacobi panel under a, dyadic
  Gauss–Legendre panels on [a, z], and a Gauss–Jacobi tail panel.  Derivative relative
  error <= 256 * 4^-r on [a, z].
* `fixed_rule(s, K, c)` — a K-pole Gauss–Jacobi rule in t = c(1-y)/(1+y), the fixed-count
  rule of synthetic/controls/shortlist_stieltjes_benchmark.py:7-10; with c = sqrt(sigma*Lam)
  the nodes are balanced geometrically across the spectrum [sigma, Lam].
"""
import math

import numpy as np

__all__ = ["composite", "fixed_rule", "poles"]


def _golub_welsch(diag, off):
    """Nodes and first-component-squared weights of the symmetric tridiagonal Jacobi matrix."""
    lam, vec = np.linalg.eigh(np.diag(diag) + np.diag(off, 1) + np.diag(off, -1))
    return lam, vec[0] ** 2


def _jacobi_panel(r, beta):
    """r-point Gauss rule on [0, 1] for the weight x^beta (Jacobi (0, beta) recurrence)."""
    k = np.arange(1, r, dtype=np.float64)
    diag = np.empty(r)
    diag[0] = beta / (beta + 2.0)
    diag[1:] = beta ** 2 / ((2 * k + beta) * (2 * k + beta + 2))
    off = 2.0 / (2 * k + beta) * np.sqrt(k ** 2 * (k + beta) ** 2 / ((2 * k + beta - 1) * (2 * k + beta + 1)))
    y, w0 = _golub_welsch(diag, off)
    return 0.5 * (1.0 + y), w0 / (beta + 1.0)


def composite(s, a, z, eps):
    """Composite rule on [a, z]; returns (tau ascending, omega, a-priori bound 256*4^-r)."""
    r = int(math.ceil(math.log(256.0 / eps) / math.log(4.0)))
    levels = int(math.ceil(math.log2(z / a)))
    c = math.sin(math.pi * s) / math.pi
    nodes, weights = [], []
    x, w = _jacobi_panel(r, -s)                      # (0, a]: weight t^-s
    nodes.append(a * x)
    weights.append(c * a ** (1.0 - s) * w)
    y, wl = np.polynomial.legendre.leggauss(r)       # [a 2^l, a 2^(l+1)]
    for ell in range(levels):
        lo = a * 2.0 ** ell
        t = lo * (3.0 + y) / 2.0
        nodes.append(t)
        weights.append(c * lo / 2.0 * wl * t ** (-s))
    top = a * 2.0 ** levels                          # [top, inf): t = top / x
    x, w = _jacobi_panel(r, s - 1.0)
    nodes.append(top / x)
    weights.append(c * top ** (1.0 - s) * w / x)
    tau = np.concatenate(nodes)
    om = np.concatenate(weights)
    order = np.argsort(tau)
    return tau[order], om[order], 256.0 * 4.0 ** (-r)


def fixed_rule(s, K, c):
    """K poles: tau_j = c (1 - y_j)/(1 + y_j) from the Gauss–Jacobi nodes y_j; ascending."""
    if s == 1:
        return np.zeros(1), np.ones(1)
    i = np.arange(K, dtype=np.float64)
    diag = (1.0 - 2.0 * s) / (4.0 * i ** 2 - 1.0)
    j = np.arange(1, K, dtype=np.float64)
    off = np.sqrt((j - s) * (j + s - 1.0)) / (2.0 * j - 1.0)
    if K > 1:
        off[0] *= math.sqrt(2.0)
    y, w0 = _golub_welsch(diag, off)
    tau = c * (1.0 - y) / (1.0 + y)
    om = c ** (1.0 - s) * 2.0 * w0 / (1.0 + y)
    return np.ascontiguousarray(tau[::-1]), np.ascontiguousarray(om[::-1])


def poles(obj, s, sigma, Lam, eps, K=None):
    """Poles for an objective (realworld/polar_gpu.py:39-43).  'er' and 'logdet' use a single
    pole at 0.  With K, the fixed K-pole rule with scale sqrt(sigma*Lam) (bound: nan)."""
    if obj in ("er", "logdet"):
        return np.zeros(1), np.ones(1), 0.0
    if obj != "frac":
        raise ValueError(f"unknown objective {obj!r}")
    if K is not None:
        tau, om = fixed_rule(s, int(K), math.sqrt(sigma * Lam))
        return tau, om, float("nan")
    return composite(s, sigma, Lam, eps)
