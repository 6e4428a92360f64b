"""Dense FP64 eigendecomposition oracles on the device: realworld/exact.py.

The small-graph certificate for the greedy: the true-marginal greedy with the eps = 1e-9
interval screen of Theorem 1 (exact.py:31-62), exact prefix gains (:65-82), brute force
over budget-k sets (:85-108) and the twin closed form (:20-28).  Same rules and tie
order as the reference; the dense work runs in FP64 on the GPU through
torch.linalg.eigh / eigvalsh (cuSOLVER, a library call, as the reference's
cupy.linalg is).  Where the reference loops one eigenvalue solve at a time (each
screened contender, each prefix, each batch of combinations) the solves here are
stacked into one batched call sized to a memory budget.

    exact_greedy(M0, cand, k, s, obj='frac') -> dict(sequence, seconds, contenders)
    eval_prefix(M0, cand, seq, s, obj='frac') -> np.ndarray
    eval_prefix_multi(M0, cand, seq, targets) -> list[np.ndarray]
    brute_force(M0, cand, k, s, obj='frac', batch=4096) -> (best, arg)
    twin_gain(M, pairs, s) -> np.ndarray

M0 is the dense (or SciPy sparse, or `Graph.M0`) matrix L + sigma I, n up to a few
thousand; cand int64[N, 2].
"""
import itertools
import time

import numpy as np
import torch

from .quadrature import composite

__all__ = ["exact_greedy", "eval_prefix", "eval_prefix_multi", "brute_force", "twin_gain", "frac_value"]

BATCH_BYTES = 2 << 30  # device bytes of stacked matrices per batched eigenvalue call


def _device(device):
    if device is not None:
        return torch.device(device)
    if not torch.cuda.is_available():
        raise RuntimeError("polar_b200.exact needs a CUDA device")
    return torch.device("cuda", torch.cuda.current_device())


def _dense(M0, dev):
    if hasattr(M0, "get"):  # Graph.M0 (host CSR behind .get(), as the reference's cupyx matrix)
        M0 = M0.get()
    if hasattr(M0, "toarray"):
        M0 = M0.toarray()
    if isinstance(M0, torch.Tensor):
        return M0.to(device=dev, dtype=torch.float64).clone()
    return torch.as_tensor(np.asarray(M0, dtype=np.float64)).to(dev)


def _add(M, a, b):
    """M += b_e b_e^T for the edge (a, b) (exact.py:8-9)."""
    M[a, a] += 1
    M[b, b] += 1
    M[a, b] -= 1
    M[b, a] -= 1


def _add_batch(A, rows, a, b):
    """A[rows] += b_e b_e^T, one edge per stacked matrix."""
    A[rows, a, a] += 1
    A[rows, b, b] += 1
    A[rows, a, b] -= 1
    A[rows, b, a] -= 1


def frac_value(lam, s, obj):
    """Objective of eigenvalue sets along the last axis (exact.py:12-17)."""
    if obj == "frac":
        return torch.sum(lam ** (-s), dim=-1)
    if obj == "er":
        return torch.sum(1.0 / lam, dim=-1)
    return -torch.sum(torch.log(lam), dim=-1)


def _per_batch(n, budget=BATCH_BYTES):
    return max(1, int(budget // (8 * n * n)))


def twin_gain(M, pairs, s):
    """x^-s - (x + 2)^-s, x = M_uu, for candidates joining non-adjacent twins of the current
    unweighted graph (identical neighbour sets: adding uv moves one eigenvalue by 2);
    nan for other pairs (exact.py:20-28)."""
    M = M if isinstance(M, torch.Tensor) else _dense(M, _device(None))
    dev = M.device
    pairs = np.asarray(pairs, dtype=np.int64).reshape(-1, 2)
    if len(pairs) == 0:
        return np.zeros(0)
    a = torch.as_tensor(pairs[:, 0], device=dev)
    b = torch.as_tensor(pairs[:, 1], device=dev)
    r = torch.arange(len(pairs), device=dev)
    D = M[a] - M[b]
    D[r, a] = 0
    D[r, b] = 0
    twin = (D.abs().amax(1) == 0) & (M[a, b] == 0) & (M[a, a] == M[b, b])
    x = M[a, a]
    g = -x ** (-s) * torch.expm1(-s * torch.log1p(2 / x))
    return torch.where(twin, g, torch.full_like(g, float("nan"))).cpu().numpy()


def exact_greedy(M0, cand, k, s, obj="frac", *, device=None):
    """True-marginal greedy (exact.py:31-62).  'frac' scores every live candidate with the
    eps = 1e-9 composite rule over the current spectrum, keeps those whose score interval
    [sc / (1 + eps), sc / (1 - eps)] reaches the best lower end, and resolves them exactly:
    twins by the closed form, the rest by the spectrum of M + b_e b_e^T (all contenders in
    one batched eigvalsh).  'er' / 'logdet' take the closed-form argmax.  First maximum
    wins ties, as the reference's argmax."""
    dev = _device(device)
    M = _dense(M0, dev)
    n = M.shape[0]
    cand = np.asarray(cand, dtype=np.int64)
    live = np.ones(len(cand), bool)
    seq, contenders = [], []
    ea = torch.as_tensor(cand[:, 0], device=dev)
    eb = torch.as_tensor(cand[:, 1], device=dev)
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    for _ in range(k):
        lam, V = torch.linalg.eigh(M)
        Wc = (V[ea] - V[eb]) ** 2
        dead = torch.as_tensor(~live, device=dev)
        if obj == "er":
            sc = (Wc @ lam ** -2) / (1 + Wc @ (1 / lam))
            sc[dead] = -torch.inf
            e = int(torch.argmax(sc))
        elif obj == "logdet":
            sc = torch.log1p(Wc @ (1 / lam))
            sc[dead] = -torch.inf
            e = int(torch.argmax(sc))
        else:
            tau, om, eps = composite(s, float(lam[0]) * 0.999, float(lam[-1]) + 2.001, 1e-9)
            eps = max(eps, 1e-9)
            D = 1 / (lam[:, None] + torch.as_tensor(tau, device=dev)[None])
            sc = ((Wc @ (D * D)) / (1 + Wc @ D)) @ torch.as_tensor(om, device=dev)
            sc[dead] = -torch.inf
            best_lo = float(torch.max(sc)) / (1 + eps)
            ids = np.flatnonzero((sc / (1 - eps) >= best_lo).cpu().numpy() & live)
            if len(ids) == 1:
                e = int(ids[0])
                contenders.append((1, 0))
            else:
                vals = np.empty(len(ids))
                tw = twin_gain(M, cand[ids], s)
                old = float(torch.sum(lam ** -s))
                todo = [i for i in range(len(ids)) if not np.isfinite(tw[i])]
                vals[np.isfinite(tw)] = tw[np.isfinite(tw)]
                step = _per_batch(n)
                for lo in range(0, len(todo), step):
                    part = todo[lo:lo + step]
                    A = M.expand(len(part), n, n).clone()
                    r = torch.arange(len(part), device=dev)
                    c = cand[ids[part]]
                    _add_batch(A, r, torch.as_tensor(c[:, 0], device=dev), torch.as_tensor(c[:, 1], device=dev))
                    lamc = torch.linalg.eigvalsh(A)
                    vals[part] = old - frac_value(lamc, s, "frac").cpu().numpy()
                    del A, lamc
                e = int(ids[int(np.argmax(vals))])
                contenders.append((len(ids), len(todo)))
        seq.append(e)
        live[e] = False
        _add(M, int(cand[e, 0]), int(cand[e, 1]))
    torch.cuda.synchronize(dev)
    return dict(sequence=seq, seconds=time.perf_counter() - t0, contenders=contenders)


def _prefix_spectra(M, cand, seq):
    """Spectra of M plus every prefix of `seq` (index 0: M itself), in batched calls."""
    n = M.shape[0]
    dev = M.device
    k = len(seq)
    out = [torch.linalg.eigvalsh(M)[None]]
    step = _per_batch(n)
    A0 = M.clone()
    for lo in range(0, k, step):
        hi = min(k, lo + step)
        A = A0.expand(hi - lo, n, n).clone()
        # prefix j holds the edges seq[:j + 1]: edge i goes into every prefix j >= i
        for i in range(lo, hi):
            a, b = int(cand[seq[i], 0]), int(cand[seq[i], 1])
            rows = torch.arange(i - lo, hi - lo, device=dev)
            _add_batch(A, rows, a, b)
            _add(A0, a, b)
        out.append(torch.linalg.eigvalsh(A))
        del A
    return torch.cat(out, 0)


def eval_prefix_multi(M0, cand, seq, targets, *, device=None):
    """Exact gains f(S_r) - f(S_0) for every prefix r, for several (obj, s) targets, from
    one spectrum per prefix (exact.py:74-82)."""
    dev = _device(device)
    M = _dense(M0, dev)
    cand = np.asarray(cand, dtype=np.int64)
    lam = _prefix_spectra(M, cand, [int(e) for e in seq])
    out = []
    for o, s in targets:
        f = frac_value(lam, s, o)
        out.append((f[0] - f[1:]).cpu().numpy())
    return out


def eval_prefix(M0, cand, seq, s, obj="frac", *, device=None):
    """Exact gains for every prefix (exact.py:65-71)."""
    return eval_prefix_multi(M0, cand, seq, [(obj, s)], device=device)[0]


def brute_force(M0, cand, k, s, obj="frac", batch=4096, *, device=None):
    """Optimal budget-k set by exhaustive enumeration in itertools.combinations order, with
    batched eigenvalue solves (exact.py:85-108).  Returns (best gain, index list)."""
    dev = _device(device)
    M = _dense(M0, dev)
    n = M.shape[0]
    cand = np.asarray(cand, dtype=np.int64)
    base = float(frac_value(torch.linalg.eigvalsh(M), s, obj))
    best, arg = -np.inf, None
    combos = itertools.combinations(range(len(cand)), k)
    step = max(1, min(int(batch), _per_batch(n)))
    while True:
        chunk = list(itertools.islice(combos, step))
        if not chunk:
            break
        C = np.asarray(chunk)
        A = M.expand(len(C), n, n).clone()
        r = torch.arange(len(C), device=dev)
        for j in range(k):
            _add_batch(A, r, torch.as_tensor(cand[C[:, j], 0], device=dev),
                       torch.as_tensor(cand[C[:, j], 1], device=dev))
        g = base - frac_value(torch.linalg.eigvalsh(A), s, obj)
        i = int(torch.argmax(g))
        v = float(g[i])
        if v > best:
            best, arg = v, C[i].tolist()
        del A
    return best, arg
