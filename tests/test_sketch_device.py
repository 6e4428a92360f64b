"""Sketches built on the device (sketches(..., device=True): host draws, device QR,
centring and F += C_0^T U) against the host construction, which the golden vectors pin to
the reference (realworld/polar_gpu.py:137-165).  Needs a B200."""
import json
from pathlib import Path

import numpy as np
import pytest

from polar_b200.synth import candidates, chung_lu

pytestmark = pytest.mark.gpu
GOLD = Path(__file__).resolve().parent / "golden"


def _close(dev_arr, host_arr, rel=1e-12):
    d = dev_arr.cpu().numpy()
    assert d.shape == host_arr.shape and d.dtype == np.float64
    np.testing.assert_allclose(d, host_arr, rtol=0, atol=rel * max(1.0, float(np.max(np.abs(host_arr)))))


@pytest.mark.parametrize("kind", ["block", "gauss", "rademacher"])
def test_device_sketches_match_host(kind):
    import polar_b200 as pg
    z = np.load(GOLD / "reference_vectors.npz")
    G = pg.Graph(500, z["g2_edges"], 1e-2)
    cand = z["g2_cand"]
    host = pg.sketches(G, cand, 16, 2026, kind=kind)
    dev = pg.sketches(G, cand, 16, 2026, kind=kind, device=True)
    for d, h in zip(dev, host):
        _close(d, h)


def test_device_sketches_chunked_weighted():
    """Several edge chunks (the reference's 4M-edge chunks, here 300 edges), weighted
    edges (U scaled by sqrt(w)), q = 32 with a ragged last block."""
    import polar_b200 as pg
    n = 1500
    E = chung_lu(n, 5.0, 2.3, 9, min_degree=1)
    w = np.random.default_rng(4).uniform(0.5, 2.0, size=len(E))
    G = pg.Graph(n, E, 1e-2, weights=w)
    cand = candidates(n, E, 333, 5)
    host = pg.sketches(G, cand, 32, 11, chunk=300)
    dev = pg.sketches(G, cand, 32, 11, chunk=300, device=True)
    for d, h in zip(dev, host):
        _close(d, h)
    Zd = dev[0].cpu().numpy()
    assert np.max(np.abs(Zd.mean(0))) < 1e-14


def test_greedy_with_device_sketches_matches_reference():
    """The FP64 greedy fed device sketches selects the reference's sequence."""
    import polar_b200 as pg
    z = np.load(GOLD / "reference_vectors.npz")
    meta = json.loads((GOLD / "reference_vectors.json").read_text())
    cfg = meta["runs"]["frac_B4_K12"]
    G = pg.Graph(500, z["g2_edges"], 1e-2)
    cand = z["g2_cand"]
    sk = pg.sketches(G, cand, 16, 2026, device=True)
    res = pg.polar(G, cand, cfg["k"], cfg["s"], q=16, B=cfg["B"], tol=1e-8, obj=cfg["obj"], sketch=sk, K=cfg["K"])
    assert res["sequence"] == list(z["run_frac_B4_K12_sequence"])
