"""Dense FP64 eigendecomposition oracles on the device (polar_b200.exact, realworld/exact.py)
against the reference's own outputs (tests/golden/make_golden.py --part exact) and the host
oracle.  Sequences, contender counts and brute-force sets exactly; gains to 1e-10
relative.  Needs a B200."""
import json
from pathlib import Path

import numpy as np
import pytest

from oracle import polar_oracle as O
from polar_b200.synth import candidates, chung_lu

pytestmark = pytest.mark.gpu
GOLD = Path(__file__).resolve().parent / "golden"


def _case(key):
    z = np.load(GOLD / "reference_exact.npz")
    meta = json.loads((GOLD / "reference_exact.json").read_text())
    n = meta["exact_cases"][key][0]
    M0 = O.Graph(n, z[f"ex_{key}_edges"], 1e-2).M0.toarray()
    return z, meta, M0, z[f"ex_{key}_cand"]


@pytest.mark.parametrize("key", ["a", "b"])
def test_exact_device_matches_reference(key):
    from polar_b200 import exact as X
    z, meta, M0, cand = _case(key)
    for obj, s in (("frac", 0.5), ("frac", 0.25), ("er", 1.0), ("logdet", 0.5)):
        tag = f"{obj}{int(round(s * 100)):03d}"
        r = X.exact_greedy(M0, cand, 4, s, obj=obj)
        assert r["sequence"] == [int(x) for x in z[f"ex_{key}_{tag}_sequence"]]
        if obj == "frac":
            np.testing.assert_array_equal(np.array(r["contenders"]), z[f"ex_{key}_{tag}_contenders"])
        np.testing.assert_allclose(X.eval_prefix(M0, cand, r["sequence"], s, obj=obj), z[f"ex_{key}_{tag}_prefix"],
                                   rtol=1e-10)
    seq = [int(x) for x in z[f"ex_{key}_frac050_sequence"]]
    multi = X.eval_prefix_multi(M0, cand, seq, [tuple(t) for t in meta[f"ex_{key}_targets"]])
    np.testing.assert_allclose(np.array(multi), z[f"ex_{key}_multi"], rtol=1e-10)
    np.testing.assert_allclose(X.twin_gain(M0, cand, 0.5), z[f"ex_{key}_twin"], rtol=1e-12)
    best, arg = X.brute_force(M0, cand[:24], 2, 0.5)
    assert arg == [int(x) for x in z[f"ex_{key}_brute_arg"]]
    assert best == pytest.approx(float(z[f"ex_{key}_brute_best"]), rel=1e-10)


def test_exact_device_matches_oracle_larger():
    """A 600-vertex graph with many pendant twins, 8 rounds, against the host oracle; the
    device greedy's prefix gains against a Graph's M0 (the drivers' G.M0.get() input)."""
    import polar_b200 as pg
    from polar_b200 import exact as X
    n = 600
    E = chung_lu(n, 3.0, 2.2, 77, min_degree=1)
    cand = candidates(n, E, 2000, 78)
    G = pg.Graph(n, E, 1e-2)
    M0 = G.M0.get().toarray()
    r = X.exact_greedy(G.M0, cand, 8, 0.5)
    ro = O.exact_greedy(M0, cand, 8, 0.5)
    assert r["sequence"] == ro["sequence"]
    assert r["contenders"] == ro["contenders"]
    np.testing.assert_allclose(X.eval_prefix(G.M0, cand, r["sequence"], 0.5),
                               O.eval_prefix_multi(M0, cand, r["sequence"], [("frac", 0.5)])[0], rtol=1e-10)
    best, arg = X.brute_force(M0, cand[:30], 2, 0.5, batch=100)  # several batches
    bo, ao = O.brute_force(M0, cand[:30], 2, 0.5)
    assert arg == ao
    assert best == pytest.approx(bo, rel=1e-10)
