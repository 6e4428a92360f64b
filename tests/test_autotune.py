"""The SpMM layout autotuner: it times the solver's layouts (lanes per row, sliced-ELL or CSR
rows, heavy-row threshold), records the fastest on the graph, and the solver's results with
the recorded layout equal the automatic layout's up to summation order.  Needs a B200."""
import numpy as np
import pytest

from polar_b200.synth import chung_lu

pytestmark = pytest.mark.gpu


def _rel(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300)


@pytest.mark.parametrize("prec,R", [("fp64", 16), ("mixed", 16), ("mixed", 64)])
def test_autotune_records_layout_and_keeps_results(prec, R):
    import polar_b200 as pg
    from polar_b200 import autotune
    n = 4000
    E = chung_lu(n, 8.0, 2.1, 21, min_degree=1)  # hubs: some rows are split into chunks
    G = pg.Graph(n, E, 1e-2)
    op = pg.Op(G)
    rng = np.random.default_rng(5)
    W = rng.normal(size=(n, R))
    tau, _, _ = pg.poles("frac", 0.5, 1e-2, G.Lam(5), 1e-2, K=8)
    active = np.unique(rng.choice(n, size=700, replace=False))
    X0, h0, it0 = pg.msolve(op, W, tau, active, 1e-9, track=True, precision=prec)
    res = autotune.tune_msolve(op, R, prec, iters=32, reps=1)
    assert len(res["table"]) >= 8
    assert res["best"] in [t[:3] for t in res["table"]]
    assert all(t[3] > 0 for t in res["table"])
    assert autotune.tuned(G, prec, R) == res["best"]
    X1, h1, it1 = pg.msolve(op, W, tau, active, 1e-9, track=True, precision=prec)
    # mixed precision: different layouts round differently (the bounds of the mixed solver
    # against the reference: 1e-4 for the iterates, 1e-5 for the tracked norms)
    lim, hlim = (1e-9, 1e-9) if prec == "fp64" else (1e-4, 1e-5)
    assert _rel(X1.cpu().numpy(), X0.cpu().numpy()) < lim
    assert _rel(h1.cpu().numpy(), h0.cpu().numpy()) < hlim
    # FP32 rounding differs between layouts; near the tolerance a column's residual can sit on
    # a plateau, so mixed-precision iteration counts may move by some 15 %
    assert np.max(np.abs(it1 - it0)) <= (3 if prec == "fp64" else max(3, 0.15 * it0.max()))
    # every timed layout gives the same solve
    for lb, sell, thresh, _ in res["table"][:: max(1, len(res["table"]) // 6)]:
        autotune.record(G, prec, R, (lb, sell, thresh))
        X2, h2, _ = pg.msolve(op, W, tau, active, 1e-9, track=True, precision=prec)
        assert _rel(X2.cpu().numpy(), X0.cpu().numpy()) < lim, (lb, sell, thresh)
        assert _rel(h2.cpu().numpy(), h0.cpu().numpy()) < hlim, (lb, sell, thresh)
    autotune.clear(G)
    assert autotune.tuned(G, prec, R) is None
