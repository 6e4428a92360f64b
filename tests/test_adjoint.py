"""Relaxed-weight objective f_s(w, sigma) and its adjoint (polar_b200.adjoint) against the
dense FP64 eigendecomposition (oracle.relaxed_dense) and central finite differences."""
import numpy as np
import pytest

from oracle import polar_oracle as O
from polar_b200.quadrature import poles
from polar_b200.synth import chung_lu

N, SIGMA, S, K = 400, 1e-2, 0.5, 24


def _problem(m=10, seed=0):
    E = chung_lu(N, 6.0, 2.5, 3, min_degree=1)
    have = set(map(tuple, np.sort(E, axis=1)))
    rng = np.random.default_rng(seed)
    cand = []
    while len(cand) < m:
        a, b = sorted(rng.integers(0, N, 2))
        if a != b and (a, b) not in have and (a, b) not in cand:
            cand.append((a, b))
    return E, np.array(cand), rng.uniform(0.0, 1.0, m)


def _rule(E, m):
    deg = np.bincount(E.ravel(), minlength=N)
    tau, om, _ = poles("frac", S, SIGMA, SIGMA + 2.0 * deg.max() + 4.0 * int(np.ceil(m)), 1e-2, K=K)
    return tau, om


def test_rule_against_eigendecomposition():
    """The 24-pole rule: d f/d w to 1e-6; f and -s f_{s+1} (the sigma derivative) to 1e-3."""
    E, cand, w = _problem()
    tau, om = _rule(E, w.sum())
    d = O.relaxed_dense(N, E, SIGMA, cand, w, S, tau, om)
    assert np.max(np.abs(d["grad_q"] - d["grad"]) / np.abs(d["grad"])) < 1e-6
    assert abs(d["f_q"] - d["f"]) / abs(d["f"]) < 1e-3
    assert abs(d["dsigma_q"] - d["dsigma"]) / abs(d["dsigma"]) < 1e-3
    # the exact derivatives themselves, by central differences of the exact f (h = 1e-3:
    # eigenvalue rounding limits smaller steps; truncation error ~1e-7)
    h = 1e-3
    for i in (0, 3):
        wp, wm = w.copy(), w.copy()
        wp[i] += h
        wm[i] -= h
        fd = (O.relaxed_dense(N, E, SIGMA, cand, wp, S)["f"] - O.relaxed_dense(N, E, SIGMA, cand, wm, S)["f"]) / (2 * h)
        assert fd == pytest.approx(d["grad"][i], rel=1e-5)
    hs = 1e-4 * SIGMA
    fd = (O.relaxed_dense(N, E, SIGMA + hs, cand, w, S)["f"] - O.relaxed_dense(N, E, SIGMA - hs, cand, w, S)["f"]) / (2 * hs)
    assert fd == pytest.approx(d["dsigma"], rel=1e-5)


@pytest.mark.gpu
def test_relaxed_gradient_and_objective_on_device():
    import polar_b200 as pg
    from polar_b200.adjoint import relaxed_gradient, relaxed_objective
    E, cand, w = _problem()
    tau, om = _rule(E, w.sum())
    d = O.relaxed_dense(N, E, SIGMA, cand, w, S, tau, om)
    G = pg.Graph(N, E, SIGMA)
    g = relaxed_gradient(G, cand, w, S, tau=tau, om=om, tol=1e-11)
    assert np.max(np.abs(g - d["grad_q"]) / np.abs(d["grad_q"])) < 1e-8
    assert np.max(np.abs(g - d["grad"]) / np.abs(d["grad"])) < 1e-5
    f, fn = relaxed_objective(G, cand, w, S, tau=tau, om=om, tol=1e-11, with_next=True)
    assert f == pytest.approx(d["f_q"], rel=1e-8)
    assert -S * fn == pytest.approx(d["dsigma_q"], rel=1e-7)
    # mixed precision: FP32 vectors, FP64 scalars
    gm = relaxed_gradient(G, cand, w, S, tau=tau, om=om, tol=1e-7, precision="mixed")
    assert np.max(np.abs(gm - g) / np.abs(g)) < 1e-5


@pytest.mark.gpu
def test_adjoint_matches_central_differences():
    """The device gradient is the adjoint of the device forward: central differences of
    relaxed_objective (h = 1e-4) agree to 1e-5."""
    import polar_b200 as pg
    from polar_b200.adjoint import relaxed_gradient, relaxed_objective
    E, cand, w = _problem(m=6, seed=1)
    tau, om = _rule(E, w.sum())
    G = pg.Graph(N, E, SIGMA)
    g = relaxed_gradient(G, cand, w, S, tau=tau, om=om, tol=1e-12)
    h = 1e-4
    for i in range(len(w)):
        wp, wm = w.copy(), w.copy()
        wp[i] += h
        wm[i] -= h
        fd = (relaxed_objective(G, cand, wp, S, tau=tau, om=om, tol=1e-12)
              - relaxed_objective(G, cand, wm, S, tau=tau, om=om, tol=1e-12)) / (2 * h)
        assert fd == pytest.approx(g[i], rel=1e-5)


@pytest.mark.gpu
def test_frac_trace_autograd():
    import torch
    import polar_b200 as pg
    from polar_b200.adjoint import FracTrace, relaxed_gradient, relaxed_rule
    E, cand, w = _problem(m=8, seed=2)
    G = pg.Graph(N, E, SIGMA)
    wt = torch.tensor(w, dtype=torch.float64, requires_grad=True)
    sig = torch.tensor(SIGMA * 1.5, dtype=torch.float64, requires_grad=True)
    f = FracTrace.apply(wt, sig, G, cand, S, K, 1e-11)
    f.backward()
    tau, om = relaxed_rule(G, S, K=K)
    # sigma enters as a shift of every pole: relative to L + 1.5 sigma the poles are tau
    d = O.relaxed_dense(N, E, SIGMA * 1.5, cand, w, S, tau, om)
    assert float(f.detach()) == pytest.approx(d["f_q"], rel=1e-8)
    assert np.allclose(wt.grad.numpy(), d["grad_q"], rtol=1e-8)
    assert float(sig.grad) == pytest.approx(d["dsigma_q"], rel=1e-7)
    assert abs(float(sig.grad) - d["dsigma"]) / abs(d["dsigma"]) < 2e-3
    g = relaxed_gradient(G, cand, w, S, tau=tau, om=om, dsigma=0.5 * SIGMA, tol=1e-11)
    assert np.allclose(wt.grad.numpy(), g, rtol=1e-12)


@pytest.mark.gpu
def test_grouped_objective_matches_chain_and_dense():
    """Woodbury groups (4 edges per solve, and the default column-limit group) give the
    rank-one chain's f and f_{s+1}; both match the dense rule."""
    import polar_b200 as pg
    from polar_b200.adjoint import relaxed_objective
    E, cand, w = _problem(m=10, seed=4)
    w[3] = 0.0  # a zero weight is skipped by every form
    tau, om = _rule(E, w.sum())
    d = O.relaxed_dense(N, E, SIGMA, cand, w, S, tau, om)
    G = pg.Graph(N, E, SIGMA)
    chain = relaxed_objective(G, cand, w, S, tau=tau, om=om, tol=1e-12, with_next=True, group=1)
    for grp in (4, None):
        f, fn = relaxed_objective(G, cand, w, S, tau=tau, om=om, tol=1e-12, with_next=True, group=grp)
        assert f == pytest.approx(chain[0], rel=1e-9)
        assert fn == pytest.approx(chain[1], rel=1e-9)
    assert chain[0] == pytest.approx(d["f_q"], rel=1e-8)


@pytest.mark.gpu
def test_central_difference_matches_gradient():
    """relaxed_central_difference (a solve on the operator without edge i) against the
    gradient (one solve on the full relaxed operator) and the dense rule, h = 1e-4."""
    import polar_b200 as pg
    from polar_b200.adjoint import relaxed_central_difference, relaxed_gradient
    E, cand, w = _problem(m=12, seed=5)
    w = np.maximum(w, 1e-3)
    tau, om = _rule(E, w.sum())
    d = O.relaxed_dense(N, E, SIGMA, cand, w, S, tau, om)
    G = pg.Graph(N, E, SIGMA)
    g = relaxed_gradient(G, cand, w, S, tau=tau, om=om, tol=1e-12)
    for i in (0, 5, 11):
        fd = relaxed_central_difference(G, cand, w, S, i, 1e-4, tau=tau, om=om, tol=1e-12)
        assert fd == pytest.approx(g[i], rel=1e-5)
        assert fd == pytest.approx(d["grad_q"][i], rel=1e-5)


@pytest.mark.gpu
def test_gradient_screen():
    """polar(..., screen=M): the live pool after the bank is the top M by the sketched
    adjoint sum_j om_j h_je (stable order), the exact screen ranks by the dense FP64
    gradient of the rule, and a screen that holds every edge the unscreened run ever
    shortlisted leaves the sequence alone (a smaller screen may change a shortlist, and the
    exact re-rank may then pick another edge)."""
    import torch
    import polar_b200 as pg
    from polar_b200.synth import candidates
    E = chung_lu(N, 6.0, 2.5, 3, min_degree=1)
    cand = candidates(N, E, 3000, 17)
    G = pg.Graph(N, E, SIGMA)
    sk = pg.sketches(G, cand, 16, 2026)
    kw = dict(q=16, B=4, tol=1e-9, sketch=sk, K=12)
    trace = []
    ref = pg.polar(G, cand, 5, S, trace=trace, **kw)
    g = pg.Greedy(G, cand, 5, S, **kw)
    g.bank()
    score = (g.om_d[:, None] * g.h).sum(0).cpu().numpy()
    g.screen(400)
    want = np.sort(np.argsort(-score, kind="stable")[:400])
    np.testing.assert_array_equal(np.flatnonzero(g.live_h), want)
    assert np.array_equal(g.live_d.cpu().numpy().astype(bool), g.live_h)
    rank = np.empty(len(cand), int)
    rank[np.argsort(-score, kind="stable")] = np.arange(len(cand))
    M = int(max(rank[t["shortlist"]].max() for t in trace)) + 1
    res = pg.polar(G, cand, 5, S, screen=M, **kw)
    assert res["sequence"] == ref["sequence"]
    # exact screen: d f/d w_e at w = 0 for every candidate, against the dense rule
    sub = cand[:300]
    ge = pg.Greedy(G, sub, 3, S, q=16, B=4, tol=1e-11, sketch=pg.sketches(G, sub, 16, 2026), K=12)
    ge.bank()
    ge.screen(50, exact=True)
    tau, om = ge.tau_d.cpu().numpy(), ge.om_d.cpu().numpy()
    d = O.relaxed_dense(N, E, SIGMA, sub, np.zeros(len(sub)), S, tau, om)
    np.testing.assert_array_equal(np.flatnonzero(ge.live_h), np.sort(np.argsort(-d["grad_q"], kind="stable")[:50]))
