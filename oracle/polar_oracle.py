"""CPU oracle for the POLAR solve-and-score path.  TEST INFRASTRUCTURE ONLY.

A plain NumPy/SciPy FP64 restatement of the reference algorithm in
realworld/polar_gpu.py (chenty2333/POLAR).  Only tests, the smoke check and the
CPU-baseline leg of the benchmark may import this module; the product path
(polar_b200) never calls it.

Parity pin: tests/golden/make_golden.py runs the unmodified reference polar_gpu.py
under a NumPy stand-in for CuPy and stores its outputs; tests/test_oracle_golden.py
checks every function below against those vectors.
"""
import math
import time

import numpy as np
import scipy.sparse as sp

__all__ = ["composite", "fixed_rule", "poles", "Graph", "Op", "msolve", "sketches", "candidates",
           "polar", "true_marginals", "degree_greedy", "random_set", "chunk_width"]


# ---------------------------------------------------------------------------------------
# Quadrature
def _gauss_jacobi_unit(r, beta):
    """Nodes/weights on [0,1] of the r-point Gauss rule for weight x^beta (Golub–Welsch).
    Follows polar_gpu.py:23-28."""
    k = np.arange(1, r, dtype=np.float64)
    diag = np.empty(r)
    diag[0] = beta / (beta + 2.0)
    diag[1:] = beta * beta / ((2 * k + beta) * (2 * k + beta + 2))
    off = 2.0 / (2 * k + beta) * np.sqrt(k * k * (k + beta) ** 2 / ((2 * k + beta - 1) * (2 * k + beta + 1)))
    J = np.diag(diag) + np.diag(off, 1) + np.diag(off, -1)
    x, Q = np.linalg.eigh(J)
    return (1.0 + x) / 2.0, Q[0] ** 2 / (beta + 1.0)


def composite(s, a, z, eps):
    """Composite positive Stieltjes rule on [a, z] (polar_gpu.py:18-36).

    r = ceil(log(256/eps)/log 4) nodes per panel; one Gauss–Jacobi panel below a, K
    dyadic Gauss–Legendre panels [a 2^l, a 2^(l+1)], and one Gauss–Jacobi panel for the
    tail above a 2^K.  Returns (tau ascending, omega, 256*4^-r)."""
    r = int(math.ceil(math.log(256.0 / eps) / math.log(4.0)))
    K = int(math.ceil(math.log2(z / a)))
    cs = math.sin(math.pi * s) / math.pi
    x_lo, w_lo = _gauss_jacobi_unit(r, -s)
    x_hi, w_hi = _gauss_jacobi_unit(r, s - 1.0)
    x_mid, w_mid = np.polynomial.legendre.leggauss(r)
    taus = [a * x_lo]
    oms = [cs * a ** (1.0 - s) * w_lo]
    for ell in range(K):
        L = a * 2.0 ** ell
        t = L * (3.0 + x_mid) / 2.0
        taus.append(t)
        oms.append(cs * L / 2.0 * w_mid * t ** (-s))
    C = a * 2.0 ** K
    taus.append(C / x_hi)
    oms.append(cs * C ** (1.0 - s) * w_hi / x_hi)
    tau = np.concatenate(taus)
    om = np.concatenate(oms)
    order = np.argsort(tau)
    return tau[order], om[order], 256.0 * 4.0 ** (-r)


def fixed_rule(s, K, c):
    """K-pole Gauss–Jacobi Stieltjes rule with scale c, the fixed-count rule of
    synthetic/controls/shortlist_stieltjes_benchmark.py:7-10:
    x^-s ~= sum_j omega_j / (x + tau_j), tau_j = c (1-y_j)/(1+y_j)."""
    if s == 1:
        return np.zeros(1), np.ones(1)
    i = np.arange(K, dtype=np.float64)
    diag = (1.0 - 2.0 * s) / (4.0 * i * i - 1.0)
    j = np.arange(1, K, dtype=np.float64)
    off = np.sqrt((j - s) * (j + s - 1.0)) / (2.0 * j - 1.0)
    if K > 1:
        off[0] *= math.sqrt(2.0)
    y, V = np.linalg.eigh(np.diag(diag) + np.diag(off, 1) + np.diag(off, -1))
    tau = c * ((1.0 - y) / (1.0 + y))[::-1]
    om = c ** (1.0 - s) * (2.0 * V[0] ** 2 / (1.0 + y))[::-1]
    return np.ascontiguousarray(tau), np.ascontiguousarray(om)


def poles(obj, s, sigma, Lam, eps, K=None):
    """Pole set for an objective (polar_gpu.py:39-43).  'er'/'logdet' use one pole at 0.
    With K given, the fixed K-pole rule with scale sqrt(sigma*Lam) replaces the composite
    rule (bound reported as nan: the fixed rule has no a-priori certificate here)."""
    if obj in ("er", "logdet"):
        return np.zeros(1), np.ones(1), 0.0
    if K is not None:
        tau, om = fixed_rule(s, int(K), math.sqrt(sigma * Lam))
        return tau, om, float("nan")
    return composite(s, sigma, Lam, eps)


# ---------------------------------------------------------------------------------------
# Operator
class Graph:
    """M0 = diag(deg + sigma) - A as a sorted FP64 CSR (polar_gpu.py:47-60)."""

    def __init__(self, n, edges, sigma, weights=None):
        self.n = int(n)
        self.sigma = float(sigma)
        u = edges[:, 0]
        v = edges[:, 1]
        w = np.ones(len(u)) if weights is None else np.asarray(weights, np.float64)
        deg = np.bincount(u, w, self.n) + np.bincount(v, w, self.n)
        A = sp.coo_matrix((np.r_[w, w], (np.r_[u, v], np.r_[v, u])), shape=(self.n, self.n)).tocsr()
        M = (sp.diags(deg + self.sigma) - A).tocsr()
        M.sort_indices()
        self.M0 = M
        self.dmax = float(deg.max()) if len(deg) else 0.0
        self.m = len(u)
        self.edges = edges
        self.weights = w

    def Lam(self, k):
        return self.sigma + 2.0 * self.dmax + 4.0 * k


class Op:
    """y = (M0 + sum_S b b^T + shift I) x (polar_gpu.py:63-80)."""

    def __init__(self, G, threads=1):
        self.M0 = G.M0
        self.A = []
        self.B = []
        # threads > 1: the product with M0 in row blocks on a thread pool (the sparse
        # product releases the interpreter lock); each row is computed as with one thread
        self.pool, self.rows = None, []
        if threads > 1:
            from concurrent.futures import ThreadPoolExecutor
            n = self.M0.shape[0]
            cuts = [(i * n) // (4 * threads) for i in range(4 * threads + 1)]
            self.rows = [(lo, hi, self.M0[lo:hi]) for lo, hi in zip(cuts[:-1], cuts[1:]) if hi > lo]
            self.pool = ThreadPoolExecutor(threads)

    def add(self, a, b):
        self.A.append(int(a))
        self.B.append(int(b))

    def _m0(self, x):
        if self.pool is None:
            return self.M0 @ x
        y = np.empty((self.M0.shape[0],) + x.shape[1:], dtype=np.result_type(self.M0.dtype, x.dtype))

        def blk(r):
            y[r[0]:r[1]] = r[2] @ x

        list(self.pool.map(blk, self.rows))
        return y

    def __call__(self, x, shift):
        y = self._m0(x)
        if shift:
            y = y + shift * x
        if self.A:
            ia = np.asarray(self.A)
            ib = np.asarray(self.B)
            diff = x[ia] - x[ib]
            np.add.at(y, ia, diff)
            np.add.at(y, ib, -diff)
        return y


class Counter:
    def __init__(self):
        self.spmv = 0
        self.rhs = 0


def msolve(op, W, tau, active, tol, maxit=100000, track=False, counter=None, on_iteration=None, threads=1):
    """Multi-shift CG for (M + tau_j I) U = W over all poles and columns
    (polar_gpu.py:88-133).

    Column c runs its own seed CG on the smallest pole tau[0]; pole j follows through
    the zeta recurrence, its iterate X and direction P are kept on the `active` rows
    only, and it freezes once |zeta| * ||r|| <= tol * ||w||.  With `track`, the three
    scalars (h, ip, pn) give ||U_j[:, c]||^2 without full vectors.  threads > 1 spreads
    the shifted updates of X and P (elementwise, the bulk of the work) over a thread pool
    by (pole, row block); every element is computed as with one thread.  Returns
    (X[p, nA, R], h[p, R] or None, iterations[R])."""
    W = np.asarray(W, np.float64)
    n, R = W.shape
    tau = np.asarray(tau, np.float64)
    p = len(tau)
    theta = (tau - tau[0])[:, None]
    active = np.asarray(active)
    r = W.copy()
    d = r.copy()
    rr = np.sum(r * r, axis=0)
    stop = tol * np.sqrt(rr)
    act = rr > 0
    X = np.zeros((p, len(active), R))
    P = np.repeat(W[active][None], p, axis=0)
    z = np.ones((p, R))
    zp = np.ones((p, R))
    live = np.repeat(act[None], p, axis=0)
    if track:
        h = np.zeros((p, R))
        ip = np.zeros((p, R))
        pn = np.repeat(rr[None], p, axis=0)
    ap = np.ones(R)
    bp = np.zeros(R)
    iters = np.zeros(R, dtype=np.int64)
    safe = lambda x: np.where(act, x, 1.0)
    pool, blocks = None, []
    if threads > 1:
        from concurrent.futures import ThreadPoolExecutor
        nA = len(active)
        per = max(1, (p * nA) // (4 * threads))
        blocks = [(j, lo, min(nA, lo + per)) for j in range(p) for lo in range(0, nA, per)]
        pool = ThreadPoolExecutor(threads)
    for it in range(maxit):
        v = op(d, float(tau[0]))
        dv = np.sum(d * v, axis=0)
        a = np.where(act, rr / safe(dv), 0.0)
        rn = r - a * v
        rrn = np.sum(rn * rn, axis=0)
        be = np.where(act, rrn / safe(rr), 0.0)
        chi = np.where(act, a * bp / ap, 0.0)
        zn = z / (1.0 + a * theta + chi * (1.0 - z / zp))
        fac = zn / z
        m = live & act[None]
        aj = np.where(m, a * fac, 0.0)
        bj = be * fac * fac
        if pool is None:
            X += aj[:, None, :] * P
            P = np.where(m[:, None, :], zn[:, None, :] * rn[active][None] + bj[:, None, :] * P, P)
        else:
            ra = rn[active]

            def upd(blk, aj=aj, bj=bj, zn=zn, m=m, ra=ra):
                j, lo, hi = blk
                Xs, Ps = X[j, lo:hi], P[j, lo:hi]
                Xs += aj[j] * Ps
                Ps[...] = np.where(m[j], zn[j] * ra[lo:hi] + bj[j] * Ps, Ps)

            list(pool.map(upd, blocks))
        if track:
            h += 2.0 * aj * ip + aj * aj * pn
            ip = np.where(m, bj * (ip + aj * pn), ip)
            pn = np.where(m, zn * zn * rrn + bj * bj * pn, pn)
        zp = np.where(m, z, zp)
        z = np.where(m, zn, z)
        nr = np.sqrt(rrn)
        live &= ~(m & (np.abs(zn) * nr <= stop))
        iters += act
        done = act & (nr <= stop)
        d = np.where(act, rn + be * d, d)
        r = np.where(act, rn, r)
        rr = np.where(act, rrn, rr)
        ap = np.where(act, a, ap)
        bp = np.where(act, be, bp)
        act &= ~done
        if on_iteration is not None:
            on_iteration(it)  # the benchmark's CPU baseline times single iterations
        if it % 8 == 7 and not act.any():
            break
    else:
        if pool is not None:
            pool.shutdown()
        raise RuntimeError("multi-shift CG iteration cap")
    if pool is not None:
        pool.shutdown()
    if counter is not None:
        counter.spmv += int(iters.sum())
        counter.rhs += R
    return X, (h if track else None), iters


# ---------------------------------------------------------------------------------------
# Sketches (inputs).  Same generation order as polar_gpu.py:137-165.
def _block_rows(rows, q, rng, center=False):
    nb = -(-rows // q)
    G = rng.normal(size=(nb, q, q))
    Q, Rm = np.linalg.qr(G)
    Q = Q * np.sign(np.diagonal(Rm, axis1=1, axis2=2))[:, None, :]
    out = np.transpose(Q, (0, 2, 1)).reshape(nb * q, q)[:rows]
    if center:
        out = out - out.mean(0)
    return out


def sketches(G, cand, q, seed, kind="block", chunk=4_000_000):
    rng = np.random.default_rng(seed)
    n = G.n
    if kind == "gauss":
        Z = rng.normal(size=(n, q)) / np.sqrt(q)
    else:
        Z = _block_rows(n, q, rng, center=True)
    F = np.zeros((n, q))
    u, v = G.edges[:, 0], G.edges[:, 1]
    sw = np.sqrt(G.weights)
    for lo in range(0, G.m, chunk):
        hi = min(G.m, lo + chunk)
        U = rng.normal(size=(hi - lo, q)) / np.sqrt(q) if kind == "gauss" else _block_rows(hi - lo, q, rng)
        U *= sw[lo:hi, None]
        ne = hi - lo
        C = sp.coo_matrix((np.r_[np.ones(ne), -np.ones(ne)],
                           (np.r_[u[lo:hi], v[lo:hi]], np.r_[np.arange(ne), np.arange(ne)])),
                          shape=(n, ne)).tocsr()
        F += C @ U
    Gc = rng.normal(size=(len(cand), q)) / np.sqrt(q) if kind == "gauss" else _block_rows(len(cand), q, rng)
    return Z, F, Gc


def chunk_width(n, p, nA, budget=10e9):
    """Bank column width heuristic of polar_gpu.py:169-173."""
    per_col = 8.0 * (10 * n + 4 * p * nA)
    cap = 16 if n > 3e6 else 64
    return int(max(8, min(cap, budget // per_col)))


# ---------------------------------------------------------------------------------------
def polar(G, cand, k, s, q=128, B=16, eps=1e-2, tol=1e-7, obj="frac", sketch=None, naive=False,
          seed=2026, kind="block", trace=None, time_limit=None, K=None, width=None):
    """Greedy POLAR with the cache backend (polar_gpu.py:180-254).

    Returns the reference keys plus `marginals`: the re-rank value
    G_q(e*) = sum_j om_j hh_j / (1 + b^T u_j) of each round's winner (for B=1 it is
    computed from the champion solve with tracking, without changing the selection;
    naive rounds report the proxy value)."""
    n, N = G.n, len(cand)
    sigma = G.sigma
    tau, om, _ = poles(obj, s, sigma, G.Lam(k), eps, K=K)
    p = len(tau)
    if sketch is None:
        sketch = sketches(G, cand, q, seed, kind)
    Z, F, Gc = sketch
    q = Z.shape[1]
    F = np.array(F, dtype=np.float64, copy=True)
    active = np.unique(cand)
    es = np.searchsorted(active, cand)
    ea, eb = es[:, 0], es[:, 1]
    ocol = om[:, None]
    op = Op(G)
    cnt = Counter()
    live = np.ones(N, bool)
    seq, marg = [], []
    t0 = time.perf_counter()
    wd = chunk_width(n, p, len(active)) if width is None else int(width)

    def bank():
        RHS = np.concatenate([Z, F], axis=1)
        parts = [msolve(op, RHS[:, lo:lo + wd], tau, active, tol, counter=cnt)[0]
                 for lo in range(0, 2 * q, wd)]
        XY = np.concatenate(parts, axis=2)
        X, Y = XY[:, :, :q].copy(), XY[:, :, q:].copy()
        h = np.sum((X[:, ea] - X[:, eb]) ** 2, axis=-1)
        t = np.sum((Y[:, ea] - Y[:, eb]) ** 2, axis=-1)
        return X, Y, h, t

    def proxy(h, t):
        return proxy_scores(h, t, om, tau, sigma, obj)

    X, Y, h, t = bank()
    for rnd in range(k):
        if rnd and time_limit is not None and time.perf_counter() - t0 > time_limit:
            break
        if naive and rnd:
            X, Y, h, t = bank()
        sc = proxy(h, t)
        sc[~live] = -np.inf
        Br = 1 if naive else min(B, int(live.sum()))
        short = np.argsort(-sc, kind="stable")[:Br]
        if naive:
            e = int(short[0])
            marg.append(float(sc[e]))
        else:
            Wb = np.zeros((n, Br))
            cols = np.arange(Br)
            Wb[cand[short, 0], cols] = 1.0
            Wb[cand[short, 1], cols] = -1.0
            U, hh, _ = msolve(op, Wb, tau, active, tol, track=obj != "logdet", counter=cnt)
            bu = U[:, es[short, 0], cols] - U[:, es[short, 1], cols]
            if obj == "logdet":
                gq = np.log1p(bu[0])
            else:
                gq = np.sum(ocol * hh / (1.0 + bu), axis=0)
            j = 0 if Br == 1 else int(np.argmax(gq))
            e = int(short[j])
            u = U[:, :, j]
            marg.append(float(gq[j]))
        if trace is not None:
            trace.append(dict(shortlist=[int(x) for x in short], chosen=e))
        seq.append(e)
        live[e] = False
        aa, bb = es[e]
        a, b = cand[e]
        if not naive and rnd + 1 < k:
            h, t = maintain(X, Y, h, t, u, Gc[e], aa, bb, ea, eb)
        F[a] += Gc[e]
        F[b] -= Gc[e]
        op.add(a, b)
    return dict(sequence=seq, marginals=marg, seconds=time.perf_counter() - t0, spmv=cnt.spmv,
                rhs=cnt.rhs, p=p, rounds=len(seq), truncated=len(seq) < k)


def proxy_scores(h, t, om, tau, sigma, obj="frac"):
    """Proxy G^_e of every candidate from the caches (polar_gpu.py:208-211)."""
    if obj == "logdet":
        return np.log1p(t[0] + sigma * h[0])
    return np.sum(om[:, None] * h / (1.0 + t + (sigma + tau[:, None]) * h), axis=0)


def maintain(X, Y, h, t, u, g_e, aa, bb, ea, eb):
    """Sherman–Morrison maintenance after the winner e = (aa, bb) joins the graph
    (polar_gpu.py:242-249): X, Y updated in place; returns the new caches (h, t)."""
    xi = X[:, aa] - X[:, bb]
    eta = g_e[None] - (Y[:, aa] - Y[:, bb])
    D = 1.0 + u[:, aa] - u[:, bb]
    cc = (u[:, ea] - u[:, eb]) / D[:, None]
    wX = np.einsum("pnq,pq->pn", X, xi)
    wY = np.einsum("pnq,pq->pn", Y, eta)
    h = np.maximum(0.0, h - 2 * cc * (wX[:, ea] - wX[:, eb]) + cc * cc * np.sum(xi * xi, 1)[:, None])
    t = np.maximum(0.0, t + 2 * cc * (wY[:, ea] - wY[:, eb]) + cc * cc * np.sum(eta * eta, 1)[:, None])
    X -= u[:, :, None] * xi[:, None, :] / D[:, None, None]
    Y += u[:, :, None] * eta[:, None, :] / D[:, None, None]
    return h, t


def candidates(n, edges, N, seed):
    """Uniform non-edge pool, one pair per draw (realworld/graphs.py:61-69): the rule the
    batched polar_b200.synth.candidates must reproduce."""
    keys = np.sort(np.asarray(edges, np.int64)[:, 0] * n + np.asarray(edges, np.int64)[:, 1])
    rng = np.random.default_rng(seed)
    chosen = set()
    while len(chosen) < N:
        u, v = sorted(map(int, rng.integers(n, size=2)))
        i = np.searchsorted(keys, u * n + v)
        if u != v and not (i < len(keys) and keys[i] == u * n + v):
            chosen.add((u, v))
    c = np.asarray(sorted(chosen), dtype=np.int64)
    return np.ascontiguousarray(c[rng.permutation(N)])


def degree_greedy(G, cand, k):
    """Degree-sum baseline (polar_gpu.py:258-265)."""
    deg = np.bincount(G.edges[:, 0], G.weights, G.n) + np.bincount(G.edges[:, 1], G.weights, G.n)
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
    """Random baseline (polar_gpu.py:268-269)."""
    return np.random.default_rng(seed).choice(len(cand), k, replace=False).tolist()


def true_marginals(G, cand, seq, s, obj="frac", eps=1e-9, tol=1e-10, kmax=None, K=None):
    """Certified marginals along a sequence (polar_gpu.py:273-291)."""
    kmax = kmax or len(seq)
    tau, om, qerr = poles(obj, s, G.sigma, G.Lam(kmax), eps, K=K)
    op = Op(G)
    cnt = Counter()
    out = []
    for e in seq:
        a, b = int(cand[e, 0]), int(cand[e, 1])
        w = np.zeros((G.n, 1))
        w[a, 0] = 1.0
        w[b, 0] = -1.0
        U, hh, _ = msolve(op, w, tau, np.asarray([a, b]), tol, track=obj != "logdet", counter=cnt)
        bu = U[:, 0, 0] - U[:, 1, 0]
        if obj == "logdet":
            g = float(np.log1p(bu[0]))
        else:
            g = float(np.sum(om * hh[:, 0] / (1.0 + bu)))
        out.append(g)
        op.add(a, b)
    rho = tol * float(np.max((G.Lam(kmax) + tau) / (G.sigma + tau)))
    return np.array(out), dict(quadrature_bound=qerr, residual_rho=rho, p=len(tau), spmv=cnt.spmv)


# ---------------------------------------------------------------------------------------
# Relaxed-weight objective (the differentiation path).  No counterpart in the reference:
# its oracle is the dense FP64 eigendecomposition, plus the same positive Stieltjes rule
# evaluated densely so that the device path can be checked with the rule's error removed.
def relaxed_dense(n, edges, sigma, cand, w, s, tau=None, om=None):
    """Exact f_s(w, sigma) = Tr(A_0^{-s}) - Tr(A_w^{-s}), d f/d w_e = s b_e^T A_w^{-s-1} b_e
    and d f/d sigma = -s (Tr(A_0^{-s-1}) - Tr(A_w^{-s-1})) from eigendecompositions, with
    A_0 = L + sigma I, A_w = A_0 + sum_e w_e b_e b_e^T.  With (tau, om), also the rule's
    values: f_q = sum_j om_j phi(tau_j), g_q = sum_j om_j ||(A_w + tau_j)^{-1} b_e||^2 and
    ds_q = -s sum_j (om_j / tau_j)(phi(0) - phi(tau_j)), where
    phi(t) = Tr((A_0 + t)^{-1}) - Tr((A_w + t)^{-1})."""
    edges = np.asarray(edges, np.int64).reshape(-1, 2)
    cand = np.asarray(cand, np.int64).reshape(-1, 2)
    w = np.asarray(w, np.float64)
    A0 = np.zeros((n, n))
    for a, b in edges:
        A0[a, a] += 1.0
        A0[b, b] += 1.0
        A0[a, b] -= 1.0
        A0[b, a] -= 1.0
    A0 += sigma * np.eye(n)
    Aw = A0.copy()
    for (a, b), we in zip(cand, w):
        Aw[a, a] += we
        Aw[b, b] += we
        Aw[a, b] -= we
        Aw[b, a] -= we
    l0 = np.linalg.eigvalsh(A0)
    lw, V = np.linalg.eigh(Aw)
    D = V[cand[:, 0]] - V[cand[:, 1]]  # (m, n): b_e^T v_i
    out = dict(f=float(np.sum(l0 ** -s) - np.sum(lw ** -s)),
               grad=s * (D ** 2) @ (lw ** (-s - 1)),
               dsigma=float(-s * (np.sum(l0 ** (-s - 1)) - np.sum(lw ** (-s - 1)))))
    if tau is not None:
        tau = np.asarray(tau, np.float64)
        om = np.asarray(om, np.float64)
        phi = lambda t: np.sum(1.0 / (l0 + t)) - np.sum(1.0 / (lw + t))
        out["f_q"] = float(sum(o * phi(t) for t, o in zip(tau, om)))
        out["grad_q"] = np.array([sum(o * np.sum((d / (lw + t)) ** 2) for t, o in zip(tau, om)) for d in D])
        out["dsigma_q"] = float(-s * sum((o / t) * (phi(0.0) - phi(t)) for t, o in zip(tau, om)))
    return out


# ---------------------------------------------------------------------------------------
# Dense eigendecomposition oracles (realworld/exact.py), the small-graph certificate.
def _dense_add(M, a, b):
    M[a, a] += 1
    M[b, b] += 1
    M[a, b] -= 1
    M[b, a] -= 1


def frac_value(lam, s, obj):
    """Objective of an eigenvalue set (exact.py:12-17)."""
    if obj == "frac":
        return float(np.sum(lam ** (-s)))
    if obj == "er":
        return float(np.sum(1.0 / lam))
    return float(-np.sum(np.log(lam)))


def twin_gain(M, pairs, s):
    """Closed-form marginal for candidates joining non-adjacent twins (exact.py:20-28):
    x^-s - (x + 2)^-s with x = M_uu; nan for other pairs."""
    a = pairs[:, 0]
    b = pairs[:, 1]
    r = np.arange(len(pairs))
    D = M[a] - M[b]
    D[r, a] = 0
    D[r, b] = 0
    twin = (np.abs(D).max(1) == 0) & (M[a, b] == 0) & (M[a, a] == M[b, b])
    x = M[a, a]
    g = -x ** (-s) * np.expm1(-s * np.log1p(2 / x))
    return np.where(twin, g, np.nan)


def exact_greedy(M0, cand, k, s, obj="frac"):
    """True-marginal greedy with eps = 1e-9 interval screening (exact.py:31-62)."""
    M = np.array(M0, dtype=np.float64, copy=True)
    live = np.ones(len(cand), bool)
    seq, contenders = [], []
    ea, eb = cand[:, 0], cand[:, 1]
    for _ in range(k):
        lam, V = np.linalg.eigh(M)
        Wc = (V[ea] - V[eb]) ** 2
        if obj == "er":
            sc = (Wc @ lam ** -2) / (1 + Wc @ (1 / lam))
            sc[~live] = -np.inf
            e = int(np.argmax(sc))
        elif obj == "logdet":
            sc = np.log1p(Wc @ (1 / lam))
            sc[~live] = -np.inf
            e = int(np.argmax(sc))
        else:
            tau, om, eps = composite(s, float(lam[0]) * 0.999, float(lam[-1]) + 2.001, 1e-9)
            eps = max(eps, 1e-9)
            D = 1 / (lam[:, None] + tau[None])
            sc = ((Wc @ (D * D)) / (1 + Wc @ D)) @ om
            sc[~live] = -np.inf
            best_lo = float(np.max(sc)) / (1 + eps)
            ids = np.flatnonzero((sc / (1 - eps) >= best_lo) & live)
            if len(ids) == 1:
                e = int(ids[0])
                contenders.append((1, 0))
            else:
                vals = np.empty(len(ids))
                tw = twin_gain(M, cand[ids], s)
                solved = 0
                old = float(np.sum(lam ** -s))
                for i, c in enumerate(ids):
                    if np.isfinite(tw[i]):
                        vals[i] = tw[i]
                        continue
                    A = M.copy()
                    _dense_add(A, int(cand[c, 0]), int(cand[c, 1]))
                    solved += 1
                    vals[i] = old - float(np.sum(np.linalg.eigvalsh(A) ** -s))
                e = int(ids[int(np.argmax(vals))])
                contenders.append((len(ids), solved))
        seq.append(e)
        live[e] = False
        _dense_add(M, int(cand[e, 0]), int(cand[e, 1]))
    return dict(sequence=seq, contenders=contenders)


def eval_prefix_multi(M0, cand, seq, targets):
    """Exact prefix gains for several (obj, s) targets (exact.py:65-82)."""
    M = np.array(M0, dtype=np.float64, copy=True)
    lam = np.linalg.eigvalsh(M)
    base = [frac_value(lam, s, o) for o, s in targets]
    out = [[] for _ in targets]
    for e in seq:
        _dense_add(M, int(cand[e, 0]), int(cand[e, 1]))
        lam = np.linalg.eigvalsh(M)
        for i, (o, s) in enumerate(targets):
            out[i].append(base[i] - frac_value(lam, s, o))
    return [np.array(v) for v in out]


def brute_force(M0, cand, k, s, obj="frac"):
    """Best budget-k set by enumeration (exact.py:85-108); first maximum in
    itertools.combinations order."""
    import itertools
    M = np.asarray(M0, dtype=np.float64)
    base = frac_value(np.linalg.eigvalsh(M), s, obj)
    best, arg = -np.inf, None
    for C in itertools.combinations(range(len(cand)), k):
        A = M.copy()
        for j in C:
            _dense_add(A, int(cand[j, 0]), int(cand[j, 1]))
        g = base - frac_value(np.linalg.eigvalsh(A), s, obj)
        if g > best:
            best, arg = g, list(C)
    return best, arg
