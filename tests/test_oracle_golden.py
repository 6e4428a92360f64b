"""Pin the CPU oracle to golden vectors produced by the unmodified reference
(tests/golden/make_golden.py).  CPU only."""
import json
from pathlib import Path

import numpy as np
import pytest

from oracle import polar_oracle as O
from polar_b200.synth import chung_lu, candidates

GOLD = Path(__file__).resolve().parent / "golden"


@pytest.fixture(scope="module")
def gold():
    z = np.load(GOLD / "reference_vectors.npz")
    meta = json.loads((GOLD / "reference_vectors.json").read_text())
    return z, meta


def test_composite_matches_reference(gold):
    z, meta = gold
    for i, (s, a, zz, eps) in enumerate(meta["composite_cases"]):
        tau, om, bnd = O.composite(s, a, zz, eps)
        np.testing.assert_allclose(tau, z[f"composite{i}_tau"], rtol=1e-13)
        np.testing.assert_allclose(om, z[f"composite{i}_om"], rtol=1e-12)
        assert bnd == float(z[f"composite{i}_bound"])


def test_generators_reproduce_reference_inputs(gold):
    z, _ = gold
    E1 = chung_lu(300, 6.0, 2.5, 11)
    np.testing.assert_array_equal(E1, z["g1_edges"])
    # candidate pool rule (realworld/graphs.py:61-69): identical stream and pool
    np.testing.assert_array_equal(candidates(300, E1, 400, 5), z["g1_cand"])
    G = O.Graph(300, E1, 1e-2)
    np.testing.assert_array_equal(G.M0.indptr, z["g1_indptr"])
    np.testing.assert_array_equal(G.M0.indices, z["g1_indices"])
    np.testing.assert_array_equal(G.M0.data, z["g1_data"])
    Gw = O.Graph(300, E1, 0.1, weights=z["g1w_weights"])
    np.testing.assert_allclose(Gw.M0.data, z["g1w_data"], rtol=1e-15)
    cand = z["g1_cand"]
    for kind in ("block", "gauss"):
        Z, F, Gc = O.sketches(G, cand, 8, 2026, kind=kind)
        np.testing.assert_allclose(Z, z[f"g1_sk_{kind}_Z"], rtol=0, atol=1e-14)
        np.testing.assert_allclose(F, z[f"g1_sk_{kind}_F"], rtol=0, atol=1e-14)
        np.testing.assert_allclose(Gc, z[f"g1_sk_{kind}_Gc"], rtol=0, atol=1e-14)
    assert O.degree_greedy(G, cand, 7) == list(z["g1_degree_greedy"])
    assert O.random_set(cand, 7, 1003) == list(z["g1_random_set"])


def test_msolve_matches_reference(gold):
    z, meta = gold
    G = O.Graph(300, z["g1_edges"], 1e-2)
    op = O.Op(G)
    for a, b in meta["ms_added"]:
        op.add(a, b)
    X, h, it = O.msolve(op, z["ms_W"], z["ms_tau"], z["ms_active"], 1e-10, track=True)
    scale = np.abs(z["ms_X"]).max()
    assert np.abs(X - z["ms_X"]).max() <= 1e-9 * scale
    np.testing.assert_allclose(h, z["ms_h"], rtol=1e-8, atol=1e-12 * np.abs(z["ms_h"]).max())
    assert np.abs(it.astype(int) - z["ms_iters"].astype(int)).max() <= 1
    assert it[3] == 0 and np.all(X[:, :, 3] == 0)


@pytest.mark.parametrize("name", ["frac_B4_K12", "frac_B1_K12", "frac_s025_B3_K10", "er_B4",
                                  "logdet_B4", "naive_K12", "frac_B2_eps"])
def test_greedy_sequences_match_reference(gold, name):
    z, meta = gold
    cfg = meta["runs"][name]
    G = O.Graph(500, z["g2_edges"], 1e-2)
    cand = z["g2_cand"]
    sk = O.sketches(G, cand, 16, 2026)
    trace = []
    res = O.polar(G, cand, cfg["k"], cfg["s"], q=16, B=cfg["B"], eps=cfg.get("eps", 1e-2), tol=1e-8,
                  obj=cfg["obj"], sketch=sk, naive=cfg.get("naive", False), trace=trace, K=cfg["K"])
    assert res["sequence"] == list(z[f"run_{name}_sequence"])
    np.testing.assert_array_equal(np.array([t["shortlist"] for t in trace]), z[f"run_{name}_shortlists"])
    assert res["p"] == int(z[f"run_{name}_p"])
    assert abs(res["spmv"] - int(z[f"run_{name}_spmv"])) <= 2 * cfg["k"] + 2
    key = f"run_{name}_rerank_max"
    if key in z.files:
        np.testing.assert_allclose(res["marginals"], z[key], rtol=1e-9)


def test_plain_workload_matches_reference(gold):
    z, _ = gold
    E = chung_lu(2000, 6.0, 2.5, 0, min_degree=1)
    assert int(E.sum()) == int(z["plain_edges_checksum"])
    cand = candidates(2000, E, 20000, 7919)
    np.testing.assert_array_equal(cand[:64], z["plain_cand_head"])
    G = O.Graph(2000, E, 1e-2)
    sk = O.sketches(G, cand, 32, 2026)
    res = O.polar(G, cand, 10, 0.5, q=32, B=1, tol=1e-8, sketch=sk, K=16)
    assert res["sequence"] == list(z["plain_sequence"])


def test_true_marginals_match_reference(gold):
    z, meta = gold
    G = O.Graph(500, z["g2_edges"], 1e-2)
    cand = z["g2_cand"]
    for obj in ("frac", "er", "logdet"):
        g, cert = O.true_marginals(G, cand, meta["tm_seq"], 0.5, obj=obj, eps=1e-4, tol=1e-10)
        np.testing.assert_allclose(g, z[f"tm_{obj}"], rtol=1e-9)
        assert cert["residual_rho"] == pytest.approx(float(z[f"tm_{obj}_rho"]))


# ---------------------------------------------------------------------------------------
# dense eigendecomposition oracles (realworld/exact.py) against the reference's outputs
def _exact_case(key):
    import json
    z = np.load(GOLD / "reference_exact.npz")
    meta = json.loads((GOLD / "reference_exact.json").read_text())
    n = meta["exact_cases"][key][0]
    E = z[f"ex_{key}_edges"]
    M0 = O.Graph(n, E, 1e-2).M0.toarray()
    return z, meta, M0, z[f"ex_{key}_cand"]


@pytest.mark.parametrize("key", ["a", "b"])
def test_exact_oracles_match_reference(key):
    z, meta, M0, cand = _exact_case(key)
    for obj, s in (("frac", 0.5), ("frac", 0.25), ("er", 1.0), ("logdet", 0.5)):
        tag = f"{obj}{int(round(s * 100)):03d}"
        r = O.exact_greedy(M0, cand, 4, s, obj=obj)
        assert r["sequence"] == [int(x) for x in z[f"ex_{key}_{tag}_sequence"]]
        if obj == "frac":
            np.testing.assert_array_equal(np.array(r["contenders"]), z[f"ex_{key}_{tag}_contenders"])
        pre = O.eval_prefix_multi(M0, cand, r["sequence"], [(obj, s)])[0]
        np.testing.assert_allclose(pre, z[f"ex_{key}_{tag}_prefix"], rtol=1e-10)
    seq = [int(x) for x in z[f"ex_{key}_frac050_sequence"]]
    multi = O.eval_prefix_multi(M0, cand, seq, [tuple(t) for t in meta[f"ex_{key}_targets"]])
    np.testing.assert_allclose(np.array(multi), z[f"ex_{key}_multi"], rtol=1e-10)
    np.testing.assert_allclose(O.twin_gain(M0, cand, 0.5), z[f"ex_{key}_twin"], rtol=1e-12)
    best, arg = O.brute_force(M0, cand[:24], 2, 0.5)
    assert arg == [int(x) for x in z[f"ex_{key}_brute_arg"]]
    assert best == pytest.approx(float(z[f"ex_{key}_brute_best"]), rel=1e-10)


# ---------------------------------------------------------------------------------------
# inputs of the workload-shaped golden cases (the greedy runs themselves are -m gpu tests)
@pytest.mark.parametrize("name", ["s025", "s050", "s075", "plain_rad"])
def test_mid_golden_inputs(name):
    import json
    from polar_b200.sketch import sketches
    p = GOLD / f"reference_mid_{name}.npz"
    if not p.exists():
        pytest.skip("golden case not generated")
    z = np.load(p)
    c = json.loads((GOLD / f"reference_mid_{name}.json").read_text())[name]
    pre = f"mid_{name}_"
    if name == "plain_rad":
        n, E = 2000, chung_lu(2000, 6.0, 2.5, 0, min_degree=1)
        cand = candidates(n, E, 20000, 7919)
    else:
        n = 20000
        E = chung_lu(n, 2 * 1049866 / 317080, 2.4, 1, min_degree=1)
        cand = candidates(n, E, 20000, 1 + 7919)
    assert (n, len(cand)) == (c["n"], c["N"])
    assert int(E.sum()) == int(z[pre + "edges_sum"]) and len(E) == int(z[pre + "m"])
    np.testing.assert_array_equal(cand[:64], z[pre + "cand_head"])
    assert int(cand.sum()) == int(z[pre + "cand_sum"])
    sk = sketches(O.Graph(n, E, 1e-2), cand, c["q"], 2026, kind=c["kind"])
    np.testing.assert_allclose([float(np.sum(a)) for a in sk], z[pre + "sketch_sums"], rtol=1e-9, atol=1e-9)
    assert z[pre + "shortlists"].shape == (c["k"], c["B"])
    assert len(z[pre + "sequence"]) == c["k"]
