"""Batched multi-shift solves: many graphs of different size, sigma and pole set in one
call (polar_msolve_batch; concurrent streams of the kernel-per-phase driver, or one
cooperative launch of the persistent driver), checked per graph against the oracle's msolve
(realworld/polar_gpu.py:88-133 restated in NumPy) and against the single-graph solver.
Needs a B200."""
import numpy as np
import pytest

from oracle import polar_oracle as O
from polar_b200.synth import chung_lu

pytestmark = pytest.mark.gpu

# (n, mean degree, exponent, seed, sigma, s): uneven sizes, one graph per CTA share
SPECS = [(300, 5.0, 2.5, 11, 1e-2, 0.5), (1200, 8.0, 2.2, 12, 1e-1, 0.3), (700, 4.0, 2.8, 13, 1e-3, 0.7),
         (2500, 6.0, 2.2, 14, 1e-2, 0.5), (150, 12.0, 2.4, 15, 1e-1, 0.3)]


def _rel(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300)


def _problems(pg, specs, R=5, K=8, weighted=False):
    rng = np.random.default_rng(2026)
    out = []
    for n, md, gam, seed, sigma, s in specs:
        E = chung_lu(n, md, gam, seed, min_degree=1)
        w = rng.uniform(0.5, 2.0, size=len(E)) if weighted else None
        G = pg.Graph(n, E, sigma, weights=w)
        tau, om, _ = pg.poles("frac", s, sigma, G.Lam(5), 1e-2, K=K)
        W = rng.normal(size=(n, R))
        active = np.unique(rng.choice(n, size=max(2, n // 4), replace=False))
        out.append(dict(n=n, E=E, w=w, sigma=sigma, G=G, op=pg.Op(G), tau=tau, W=W, active=active))
    return out


def _solve(pb, tol, prec="fp64", **kw):
    from polar_b200.batch import msolve_batch
    return msolve_batch([q["op"] for q in pb], [q["W"] for q in pb], [q["tau"] for q in pb],
                        [q["active"] for q in pb], tol, track=True, precision=prec, **kw)


@pytest.mark.parametrize("weighted", [False, True])
@pytest.mark.parametrize("driver", ["graph", "persistent"])
def test_batch_fp64_matches_oracle_per_graph(weighted, driver):
    import polar_b200 as pg
    from polar_b200.solver import set_solver_mode
    specs = SPECS if not weighted else SPECS[:3]
    pb = _problems(pg, specs, weighted=weighted)
    set_solver_mode(driver)
    try:
        res = _solve(pb, 1e-10)
    finally:
        set_solver_mode("graph")
    for q, (X, h, it) in zip(pb, res):
        og = O.Graph(q["n"], q["E"], q["sigma"], weights=q["w"])
        Xo, ho, ito = O.msolve(O.Op(og), q["W"], q["tau"], q["active"], 1e-10, track=True)
        assert _rel(X.cpu().numpy(), Xo) < 1e-8
        assert _rel(h.cpu().numpy(), ho) < 1e-8
        assert np.max(np.abs(it - ito)) <= max(3, 0.02 * ito.max())


def test_batch_matches_single_solves():
    """Each problem of a batch gives the solve the single-graph solver gives (FP64: 1e-9).
    Mixed precision against FP64: 1e-4 for the iterates and the tracked norms (two of the
    graphs have sigma = 1e-3)."""
    import polar_b200 as pg
    pb = _problems(pg, SPECS)
    res = _solve(pb, 1e-10)
    mix = _solve(pb, 1e-8, "mixed")
    for q, (X, h, it), (Xm, hm, itm) in zip(pb, res, mix):
        Xs, hs, its = pg.msolve(q["op"], q["W"], q["tau"], q["active"], 1e-10, track=True)
        assert _rel(X.cpu().numpy(), Xs.cpu().numpy()) < 1e-9
        assert _rel(h.cpu().numpy(), hs.cpu().numpy()) < 1e-9
        assert np.max(np.abs(it - its)) <= 3
        assert Xm.element_size() == 4
        assert _rel(Xm.cpu().numpy(), Xs.cpu().numpy()) < 1e-4
        assert _rel(hm.cpu().numpy(), hs.cpu().numpy()) < 1e-4


def test_batch_errors_and_recovery():
    import polar_b200 as pg
    from polar_b200 import _lib
    pb = _problems(pg, SPECS[:3])
    # one problem capped: its status is the iteration cap
    with pytest.raises(RuntimeError, match="iteration cap"):
        _solve(pb, 1e-12, maxit=[100000, 4, 100000])
    # a non-finite right-hand side
    bad = [dict(q) for q in pb]
    bad[2]["W"] = bad[2]["W"].copy()
    bad[2]["W"][5, 1] = np.nan
    with pytest.raises(_lib.PolarError) as ei:
        _solve(bad, 1e-10)
    assert ei.value.status == _lib.POLAR_ERR_NONFINITE
    # widths that pad differently are rejected before launch
    wide = [dict(q) for q in pb]
    wide[1]["W"] = np.random.default_rng(0).normal(size=(wide[1]["n"], 20))
    with pytest.raises(_lib.PolarError) as ei:
        _solve(wide, 1e-10)
    assert ei.value.status == _lib.POLAR_ERR_BAD_ARG
    # persistent driver: barrier waits that run out end every multi-CTA problem with
    # TIMEOUT, and the context stays usable
    from polar_b200.solver import set_solver_mode
    lib = _lib.load()
    set_solver_mode("persistent")
    lib.polar_set_barrier_timeout_ns(1)
    try:
        with pytest.raises(_lib.PolarError) as ei:
            _solve(_problems(pg, SPECS[3:4]), 1e-10)
        assert ei.value.status == _lib.POLAR_ERR_TIMEOUT
    finally:
        lib.polar_set_barrier_timeout_ns(4_000_000_000)
        set_solver_mode("graph")
    res = _solve(pb, 1e-10)
    assert all(np.isfinite(X.cpu().numpy()).all() for X, _, _ in res)
