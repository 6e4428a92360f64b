"""Seeded synthetic inputs: Chung–Lu graphs and uniform non-edge candidate pools.

The reference runs on SNAP graphs (realworld/graphs.py:11-19); those files are not
available here, so seeded Chung–Lu graphs with the same vertex/edge counts stand in
for them. Host-side NumPy: this is input generation, not part of the timed path.
"""
import numpy as np

__all__ = ["chung_lu", "candidates", "CONFIGS", "make_config", "batch_specs"]


def _chung_lu_weights(n, mean_deg, gamma, dmax):
    """Expected degrees w_i = C (i + i0)^(-1/(gamma-1)), sum w = n * mean_deg, w_0 = dmax.

    i0 is found by bisection so that the largest expected degree equals `dmax`
    (default: the structural cutoff sqrt(sum w), which keeps w_i w_j / sum w <= 1)."""
    total = float(n) * float(mean_deg)
    if dmax is None:
        dmax = np.sqrt(total)
    alpha = 1.0 / (gamma - 1.0)
    i = np.arange(n, dtype=np.float64)

    def top(i0):
        base = (i + i0) ** (-alpha)
        return total * base[0] / base.sum()

    lo, hi = 1e-6, float(n)
    if top(lo) < dmax:
        i0 = lo
    else:
        for _ in range(200):
            mid = np.sqrt(lo * hi)
            if mid == lo or mid == hi:
                break  # fixed point: every further step leaves (lo, hi) unchanged
            if top(mid) > dmax:
                lo = mid
            else:
                hi = mid
        i0 = hi
    w = (i + i0) ** (-alpha)
    return w * (total / w.sum())


def _sorted_unique(x):
    """np.unique for int64 keys by one sort (NumPy's hashing path is slower at 10^7)."""
    x = np.sort(x)
    if len(x) < 2:
        return x
    return x[np.r_[True, x[1:] != x[:-1]]]


def chung_lu(n, mean_deg, gamma, seed, dmax=None, m=None, min_degree=0):
    """Undirected simple Chung–Lu graph on vertices 0..n-1 (hubs at low ids).

    Endpoints are drawn independently with probability proportional to the expected
    degree; the result is made undirected, stripped of self-loops and deduplicated with
    the same preprocessing rule as realworld/graphs.py:52-53 (sort each pair, drop u==v,
    unique).  Sampling repeats until exactly `m` distinct edges exist (default
    round(n*mean_deg/2)); a final seeded subset trims any overshoot.
    With min_degree=1, every vertex left isolated gets one edge to a partner drawn in
    proportion to expected degree (the SNAP graphs these stand in for contain only
    endpoint vertices, realworld/graphs.py:51); the edge count then grows by the number of
    such vertices.  Returns int64[m', 2] with u < v, rows sorted lexicographically."""
    rng = np.random.default_rng(seed)
    w = _chung_lu_weights(n, mean_deg, gamma, dmax)
    target = int(round(n * mean_deg / 2)) if m is None else int(m)
    cdf = np.cumsum(w)
    cdf /= cdf[-1]
    keys = np.empty(0, dtype=np.int64)
    while len(keys) < target:
        need = target - len(keys)
        draw = int(need * 1.15) + 64
        u = np.searchsorted(cdf, rng.random(draw), side="right").clip(0, n - 1)
        v = np.searchsorted(cdf, rng.random(draw), side="right").clip(0, n - 1)
        a = np.minimum(u, v).astype(np.int64)
        b = np.maximum(u, v).astype(np.int64)
        keep = a != b
        keys = _sorted_unique(np.concatenate([keys, a[keep] * n + b[keep]]))
    if len(keys) > target:
        keys = keys[np.sort(rng.choice(len(keys), target, replace=False))]
    if min_degree >= 1:
        deg = np.bincount(np.r_[keys // n, keys % n], minlength=n)
        iso = np.flatnonzero(deg == 0)
        if len(iso):
            part = np.searchsorted(cdf, rng.random(len(iso)), side="right").clip(0, n - 1)
            clash = part == iso
            while clash.any():
                part[clash] = np.searchsorted(cdf, rng.random(int(clash.sum())), side="right").clip(0, n - 1)
                clash = part == iso
            a = np.minimum(iso, part).astype(np.int64)
            b = np.maximum(iso, part).astype(np.int64)
            keys = _sorted_unique(np.concatenate([keys, a * n + b]))
    return np.stack([keys // n, keys % n], axis=1).astype(np.int64)


def candidates(n, edges, N, seed):
    """Uniform random non-edge pool, the rule of realworld/graphs.py:61-69, in batches.

    The rule draws one pair per `rng.integers(n, size=2)` call, orders it (u <= v),
    rejects u == v and pairs that are edges (keys u*n + v of the edge list as given),
    collects distinct pairs until N exist, sorts them and shuffles with
    `rng.permutation(N)`.  NumPy's bounded-integer stream does not depend on how the
    draws are split into calls (the bit generator carries its spare 32-bit half across
    calls), so here the pairs come in large batches: each batch is filtered with sorted
    key lookups, the first occurrence of each new key is kept in draw order, and the
    pool closes at the pair that makes it N long.  The generator is then rewound and
    advanced by exactly the pairs the rule consumed, so the final permutation draws
    from the same state.  Same seed, same pool, same order as the rule; about 1 s at
    N = 10^6 instead of minutes."""
    n = int(n)
    N = int(N)
    e = np.asarray(edges, dtype=np.int64).reshape(-1, 2)
    keys = np.sort(e[:, 0] * n + e[:, 1])
    rng = np.random.default_rng(seed)
    if N <= 0:
        return np.zeros((0, 2), np.int64)
    if N > n * (n - 1) // 2 - len(_sorted_unique(keys)):
        raise ValueError("more candidates requested than non-edges exist")
    start = rng.bit_generator.state
    pool = np.empty(0, np.int64)          # accepted keys, sorted
    consumed = 0
    while True:
        need = N - len(pool)
        batch = max(4096, int(need * 1.25) + 1024)
        xy = rng.integers(n, size=2 * batch).reshape(batch, 2)
        u = np.minimum(xy[:, 0], xy[:, 1])
        v = np.maximum(xy[:, 0], xy[:, 1])
        key = u * n + v
        ok = u != v
        if len(keys):
            i = np.searchsorted(keys, key).clip(0, len(keys) - 1)
            ok &= keys[i] != key
        if len(pool):
            j = np.searchsorted(pool, key).clip(0, len(pool) - 1)
            ok &= pool[j] != key
        pos = np.flatnonzero(ok)
        ukey, first = np.unique(key[pos], return_index=True)
        order = np.sort(pos[first])       # draw positions of the new distinct keys
        if len(order) >= need:
            last = int(order[need - 1])
            consumed += last + 1
            pool = _sorted_unique(np.concatenate([pool, key[order[:need]]]))
            break
        consumed += batch
        pool = _sorted_unique(np.concatenate([pool, ukey]))
    rng.bit_generator.state = start
    rng.integers(n, size=2 * consumed)    # the rule's draws, to reach its final state
    c = np.stack([pool // n, pool % n], axis=1)
    return np.ascontiguousarray(c[rng.permutation(N)])


# Workload shapes.  Each entry: graph (n, mean degree, exponent, seed, dmax), pool size N,
# pole count K, sketch width q, shortlist B, rounds k, sigma, s, CG tolerance.
CONFIGS = {
    "plain-n2000": dict(n=2000, mean_deg=6.0, gamma=2.5, seed=0, dmax=None, min_degree=1, N=20000,
                        K=16, q=32, B=1, k=10, sigma=1e-2, s=0.5, tol=1e-8),
    "precision-n317k": dict(n=317080, mean_deg=2 * 1049866 / 317080, gamma=2.4, seed=1, dmax=None, min_degree=1,
                            N=200000, K=24, q=64, B=16, k=50, sigma=1e-2, s=0.5, tol=1e-7),
    "diff-n1.13M": dict(n=1134890, mean_deg=2 * 2987624 / 1134890, gamma=2.2, seed=3, dmax=None, min_degree=1,
                        N=4096, K=24, q=64, B=16, k=0, sigma=1e-2, s=0.5, tol=1e-7),
    "full-n4M": dict(n=3997962, mean_deg=2 * 34681189 / 3997962, gamma=2.1, seed=4, dmax=15000, min_degree=1,
                     N=1000000, K=32, q=64, B=16, k=100, sigma=1e-2, s=0.5, tol=1e-6),
    # many graphs solved together: per-graph shapes from batch_specs; each graph's bank
    # solve (2q right-hand sides) over the endpoints of up to N candidates
    "batch48": dict(graphs=48, N=20000, K=16, q=32, k=10, tol=1e-7),
}


def batch_specs(count=48, seed=3):
    """Per-graph shapes of the many-graphs workload: n log-uniform in [5k, 400k], mean
    degree uniform in [4, 20], exponent uniform in [2.2, 2.8], sigma from {1e-3, 1e-2,
    1e-1} and s from {0.3, 0.5, 0.7}, each drawn per graph from one seeded stream."""
    rng = np.random.default_rng(seed)
    out = []
    for g in range(count):
        n = int(round(np.exp(rng.uniform(np.log(5e3), np.log(4e5)))))
        out.append(dict(n=n, mean_deg=float(rng.uniform(4.0, 20.0)), gamma=float(rng.uniform(2.2, 2.8)),
                        seed=1000 + g, sigma=float(rng.choice([1e-3, 1e-2, 1e-1])),
                        s=float(rng.choice([0.3, 0.5, 0.7]))))
    return out


def make_config(name, n=None, N=None, cand_seed=None, cache=None):
    """Build (edges, n, cand, config) for a named workload, optionally shrunk to `n`
    vertices (mean degree and exponent kept) and `N` candidates.

    cache: a directory (default $POLAR_DATA when set) holding one .npz per (workload, n, N,
    candidate seed), written on first use and read afterwards, as realworld/graphs.py:46-50
    caches each prepared graph; the generation takes about a minute at 4M vertices."""
    import os
    c = dict(CONFIGS[name])
    n = c["n"] if n is None else int(n)
    N = c["N"] if N is None else int(N)
    seed = c["seed"] + 7919 if cand_seed is None else int(cand_seed)
    cache = cache if cache is not None else os.environ.get("POLAR_DATA")
    path = None
    if cache:
        os.makedirs(cache, exist_ok=True)
        path = os.path.join(cache, f"{name}_n{n}_N{N}_s{seed}.npz")
        if os.path.exists(path):
            z = np.load(path)
            return z["edges"].astype(np.int64), n, z["cand"].astype(np.int64), c
    dmax = c["dmax"] if n == c["n"] else None
    edges = chung_lu(n, c["mean_deg"], c["gamma"], c["seed"], dmax=dmax, min_degree=c.get("min_degree", 0))
    cand = candidates(n, edges, N, seed)
    if path:
        tmp = path + ".tmp.npz"
        np.savez(tmp, edges=edges.astype(np.int32), cand=cand.astype(np.int32))
        os.replace(tmp, path)
    return edges, n, cand, c
