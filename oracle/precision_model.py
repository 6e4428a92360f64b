"""CPU model of the mixed-precision multi-shift CG: which vectors may be rounded to FP32.

Test infrastructure (like the rest of oracle/): a NumPy restatement of the seed CG and the
shifted recurrences of realworld/polar_gpu.py:88-133 (msolve, with the norm tracker of
:115-117) in which chosen vectors are rounded to FP32 each iteration, as the device
kernels store them.  It measures, for a shortlist-style solve (incidence right-hand sides
e_a - e_b), the seed iteration count and the relative error of the re-rank marginal
G = sum_j om_j h_j / (1 + b^T u_j) (polar_gpu.py:231-235) against the all-FP64 run.

Knobs (each True = stored in FP32):
  r    the residual                       d    the direction recurrence
  dm   the SpMM's copy of the direction   v    the SpMM output
  xp   the shifted iterates X, P (rounded once per M-step deferred update)
The device's mixed scheme is r = d = False, dm = v = xp = True.
ru = m adds reliable updates: the seed iterate x is kept on all rows in FP64 (x += alpha d
with the direction the SpMM read), and every m iterations the recurred residual is replaced
by the true residual W - (M + tau_0) x accumulated in FP64 (then stored as the r knob says).
"""
import numpy as np
import scipy.sparse as sp

__all__ = ["shortlist_solve", "laplacian"]


def _f32(x):
    return x.astype(np.float32).astype(np.float64)


def laplacian(n, edges):
    """Off-diagonal part of L (as the reference's CSR M0 without the diagonal) and degrees."""
    e = np.asarray(edges, dtype=np.int64)
    A = sp.coo_matrix((-np.ones(2 * len(e)), (np.r_[e[:, 0], e[:, 1]], np.r_[e[:, 1], e[:, 0]])),
                      shape=(n, n)).tocsr()
    deg = np.bincount(e[:, 0], minlength=n) + np.bincount(e[:, 1], minlength=n)
    return A, deg.astype(np.float64)


def shortlist_solve(A, deg, sigma, tau, om, pairs, tol=1e-7, M=16, r=False, d=False, dm=False, v=False, xp=False,
                    maxit=100000, ru=None, matmul=None):
    """Multi-shift CG for (L + sigma + tau_j) U = W, W[:, c] = e_a - e_b for pairs[c].
    matmul: callable x -> A @ x (default SciPy's product; a threaded one for large graphs).

    Returns (iterations of the seed system, G per column)."""
    n = A.shape[0]
    R = len(pairs)
    cols = np.arange(R)
    W = np.zeros((n, R))
    W[pairs[:, 0], cols] = 1.0
    W[pairs[:, 1], cols] = -1.0
    diag = deg + sigma + tau[0]
    shift = (tau - tau[0])[:, None]
    p = len(tau)
    ident = lambda x: x
    rR, rD, rDm, rV, rX = (_f32 if k else ident for k in (r, d, dm, v, xp))
    mul = matmul if matmul is not None else (lambda x: A @ x)
    xs = np.zeros((n, R)) if ru else None
    res = W.copy()
    dirn = W.copy()
    rr = (res * res).sum(0)
    stop = tol * np.sqrt(rr)
    act = rr > 0
    rows = np.stack([pairs[:, 0], pairs[:, 1]])
    X = np.zeros((p, 2, R))
    P = np.broadcast_to(W[rows, cols][None], (p, 2, R)).copy()
    z = np.ones((p, R))
    zp = np.ones((p, R))
    live = np.broadcast_to(act[None], (p, R)).copy()
    h = np.zeros((p, R))
    ip = np.zeros((p, R))
    pn = np.broadcast_to(rr[None], (p, R)).copy()
    ap = np.ones(R)
    bp = np.zeros(R)
    it = 0
    while act.any():
        if it >= maxit:
            raise RuntimeError("multi-shift CG iteration cap")
        dg = rDm(dirn)
        vv = rV(diag[:, None] * dg + mul(dg))
        dv = (dg * vv).sum(0)
        a = np.where(act, rr / np.where(act, dv, 1.0), 0.0)
        rn = rR(res - a * vv)
        if ru:
            xs += a * dg
            if (it + 1) % ru == 0:  # reliable update: the true residual, accumulated in FP64
                rn = rR(np.where(act, W - (diag[:, None] * xs + mul(xs)), rn))
        rrn = (rn * rn).sum(0)
        be = np.where(act, rrn / np.where(act, rr, 1.0), 0.0)
        c = np.where(act, a * bp / ap, 0.0)
        zn = z / (1 + a * shift + c * (1 - z / zp))
        fac = zn / z
        m = live & act[None]
        aj = np.where(m, a * fac, 0.0)
        bj = be * fac * fac
        X = X + aj[:, None, :] * P
        r_act = _f32(rn[rows, cols]) if xp else rn[rows, cols]  # the history holds r in FP32
        P = np.where(m[:, None, :], zn[:, None, :] * r_act[None] + bj[:, None, :] * P, P)
        if (it + 1) % M == 0:
            X = rX(X)
            P = rX(P)
        h += 2 * aj * ip + aj * aj * pn
        ip = np.where(m, bj * (ip + aj * pn), ip)
        pn = np.where(m, zn * zn * rrn + bj * bj * pn, pn)
        zp = np.where(m, z, zp)
        z = np.where(m, zn, z)
        nr = np.sqrt(rrn)
        live &= ~(m & (np.abs(zn) * nr <= stop))
        done = act & (nr <= stop)
        dirn = rD(np.where(act, rn + be * dirn, dirn))
        res = np.where(act, rn, res)
        rr = np.where(act, rrn, rr)
        ap = np.where(act, a, ap)
        bp = np.where(act, be, bp)
        act &= ~done
        it += 1
    X = rX(X)
    bu = X[:, 0, :] - X[:, 1, :]
    return it, (om[:, None] * h / (1 + bu)).sum(0)
