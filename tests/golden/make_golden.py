"""Generate golden vectors by running the UNMODIFIED reference on CPU.

The reference realworld/polar_gpu.py (and realworld/graphs.py for the candidate rule)
is imported from a checkout of chenty2333/POLAR with a NumPy stand-in for CuPy
(tests/golden/_standin) ahead of it on sys.path.  Its outputs are saved to
tests/golden/reference_*.npz; the tests compare the oracle (and, on a GPU, the CUDA path)
against them.  The checkout path comes from $POLAR_REFERENCE (required).  Parts:

    POLAR_REFERENCE=<checkout> python tests/golden/make_golden.py [--part base|mid|exact]

base   small graphs: quadrature, CSR, candidates, sketches, msolve, 7 greedy runs, the
       n = 2000 plain workload, certified marginals -> reference_vectors.npz/.json
mid    the workload shapes at a size the CPU finishes in minutes: Chung-Lu exponent 2.4,
       n = 20,000, 20,000 candidates, K = 24, q = 64, B = 16, 10 rounds, tol 1e-7 for
       s = 0.25, 0.5, 0.75; and the n = 2000 plain workload with a Rademacher sketch
       -> reference_mid.npz/.json
exact  the dense eigendecomposition oracles of realworld/exact.py (exact greedy with
       interval screening, prefix gains, brute force, twin closed form) on small graphs
       -> reference_exact.npz/.json
"""
import argparse
import json
import os
import sys
import time
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REPO = HERE.parent.parent
if "POLAR_REFERENCE" not in os.environ:
    sys.exit("set POLAR_REFERENCE to a checkout of chenty2333/POLAR")
REF = Path(os.environ["POLAR_REFERENCE"]) / "realworld"
sys.path.insert(0, str(HERE / "_standin"))
sys.path.insert(1, str(REF))
sys.path.insert(2, str(REPO))

import cupy  # noqa: E402  (the stand-in)
import polar_gpu as ref  # noqa: E402
import graphs as ref_graphs  # noqa: E402

from polar_b200.synth import chung_lu  # noqa: E402
from oracle.polar_oracle import fixed_rule  # noqa: E402

out = {}
meta = {}


def put(key, val):
    out[key] = np.asarray(val)


def fixed_poles(K):
    """Patch for ref.poles: the fixed K-pole rule with scale sqrt(sigma * Lam)."""
    def _poles(obj, s, sigma, Lam, eps):
        if obj in ("er", "logdet"):
            return np.zeros(1), np.ones(1), 0.0
        tau, om = fixed_rule(s, K, np.sqrt(sigma * Lam))
        return tau, om, float("nan")
    return _poles


def part_base():
    """Small-graph vectors -> reference_vectors.npz/.json."""
    t_start = time.time()
    # 1. quadrature ------------------------------------------------------------------------
    comp_cases = [(0.5, 1e-2, 300.0, 1e-2), (0.25, 1.0, 50.0, 1e-3), (0.75, 1e-3, 1e4, 1e-1)]
    for i, (s, a, z, eps) in enumerate(comp_cases):
        tau, om, bnd = ref.composite(s, a, z, eps)
        put(f"composite{i}_tau", tau)
        put(f"composite{i}_om", om)
        put(f"composite{i}_bound", bnd)
    meta["composite_cases"] = comp_cases

    # 2. graph + candidates + sketches -----------------------------------------------------
    n1 = 300
    E1 = chung_lu(n1, 6.0, 2.5, 11)
    put("g1_edges", E1)
    G1 = ref.Graph(n1, E1, 1e-2)
    put("g1_indptr", G1.M0.indptr)
    put("g1_indices", G1.M0.indices)
    put("g1_data", G1.M0.data)
    cand1 = ref_graphs.candidates(n1, E1, 400, 5)
    put("g1_cand", cand1)
    for kind in ("block", "gauss"):
        Z, F, Gc = ref.sketches(G1, cand1, 8, 2026, kind=kind)
        put(f"g1_sk_{kind}_Z", Z)
        put(f"g1_sk_{kind}_F", F)
        put(f"g1_sk_{kind}_Gc", Gc)
    put("g1_degree_greedy", ref.degree_greedy(G1, cand1, 7))
    put("g1_random_set", ref.random_set(cand1, 7, 1003))
    wts = np.random.default_rng(3).uniform(0.5, 2.0, size=len(E1))
    Gw = ref.Graph(n1, E1, 0.1, weights=wts)
    put("g1w_weights", wts)
    put("g1w_data", Gw.M0.data)
    put("g1w_indices", Gw.M0.indices)
    put("g1w_indptr", Gw.M0.indptr)

    # 3. msolve ------------------------------------------------------------------------------
    rng = np.random.default_rng(21)
    W = rng.normal(size=(n1, 6))
    W[:, 3] = 0.0                                  # a zero column returns immediately
    active = np.unique(cand1)[:90]
    tau, om, _ = ref.composite(0.5, 1e-2, G1.Lam(5), 1e-1)
    put("ms_W", W)
    put("ms_active", active)
    put("ms_tau", tau)
    op = ref.Op(G1)
    op.add(int(cand1[0, 0]), int(cand1[0, 1]))
    op.add(int(cand1[1, 0]), int(cand1[1, 1]))
    X, h, it = ref.msolve(op, W, tau, active, 1e-10, track=True)
    put("ms_X", X)
    put("ms_h", h)
    put("ms_iters", it)
    meta["ms_added"] = [[int(cand1[0, 0]), int(cand1[0, 1])], [int(cand1[1, 0]), int(cand1[1, 1])]]

    # 4. greedy runs -------------------------------------------------------------------------
    n2 = 500
    E2 = chung_lu(n2, 6.0, 2.5, 12)
    cand2 = ref_graphs.candidates(n2, E2, 3000, 6)
    put("g2_edges", E2)
    put("g2_cand", cand2)
    G2 = ref.Graph(n2, E2, 1e-2)
    sk2 = ref.sketches(G2, cand2, 16, 2026)
    runs = {
        "frac_B4_K12": dict(obj="frac", B=4, K=12, k=6, s=0.5),
        "frac_B1_K12": dict(obj="frac", B=1, K=12, k=6, s=0.5),
        "frac_s025_B3_K10": dict(obj="frac", B=3, K=10, k=5, s=0.25),
        "er_B4": dict(obj="er", B=4, K=None, k=5, s=1.0),
        "logdet_B4": dict(obj="logdet", B=4, K=None, k=5, s=0.5),
        "naive_K12": dict(obj="frac", B=4, K=12, k=4, s=0.5, naive=True),
        "frac_B2_eps": dict(obj="frac", B=2, K=None, k=4, s=0.5, eps=1e-1),
    }
    orig_poles = ref.poles
    for name, cfg in runs.items():
        ref.poles = fixed_poles(cfg["K"]) if cfg["K"] else orig_poles
        cupy.ARGMAX_LOG.clear()
        trace = []
        res = ref.polar(G2, cand2, cfg["k"], cfg["s"], q=16, B=cfg["B"], eps=cfg.get("eps", 1e-2),
                        tol=1e-8, obj=cfg["obj"], sketch=sk2, naive=cfg.get("naive", False), trace=trace)
        put(f"run_{name}_sequence", res["sequence"])
        put(f"run_{name}_spmv", res["spmv"])
        put(f"run_{name}_p", res["p"])
        put(f"run_{name}_shortlists", np.array([t["shortlist"] for t in trace]))
        if cfg["B"] > 1 and not cfg.get("naive"):
            scores = [np.asarray(a, dtype=np.float64) for a in cupy.ARGMAX_LOG]
            if cfg["obj"] == "logdet":
                scores = [np.asarray(a) for a in scores]
            put(f"run_{name}_rerank_max", [float(np.max(a)) for a in scores])
        print(name, res["sequence"], res["spmv"], f"{time.time() - t_start:.1f}s", flush=True)
    ref.poles = orig_poles
    meta["runs"] = runs

    # 5. plain workload at n=2000 (K=16, q=32, B=1, k=10, tol 1e-8, sigma 1e-2, s 0.5) ----------
    n3 = 2000
    E3 = chung_lu(n3, 6.0, 2.5, 0, min_degree=1)
    cand3 = ref_graphs.candidates(n3, E3, 20000, 0 + 7919)
    G3 = ref.Graph(n3, E3, 1e-2)
    sk3 = ref.sketches(G3, cand3, 32, 2026)
    ref.poles = fixed_poles(16)
    trace = []
    res = ref.polar(G3, cand3, 10, 0.5, q=32, B=1, tol=1e-8, sketch=sk3, trace=trace)
    ref.poles = orig_poles
    put("plain_edges_checksum", int(E3.sum()))
    put("plain_cand_head", cand3[:64])
    put("plain_sequence", res["sequence"])
    put("plain_spmv", res["spmv"])
    put("plain_shortlists", np.array([t["shortlist"] for t in trace]))
    print("plain", res["sequence"], res["spmv"], f"{time.time() - t_start:.1f}s", flush=True)

    # 6. certified marginals -----------------------------------------------------------------
    seq = list(out["run_frac_B4_K12_sequence"][:4])
    for obj in ("frac", "er", "logdet"):
        g, cert = ref.true_marginals(G2, cand2, seq, 0.5, obj=obj, eps=1e-4, tol=1e-10)
        put(f"tm_{obj}", g)
        put(f"tm_{obj}_rho", cert["residual_rho"])
    meta["tm_seq"] = [int(x) for x in seq]

    np.savez_compressed(HERE / "reference_vectors.npz", **out)
    (HERE / "reference_vectors.json").write_text(json.dumps(meta, indent=1))
    print("wrote", HERE / "reference_vectors.npz", f"{time.time() - t_start:.1f}s")


# ---- mid-size workload shapes -------------------------------------------------------------
MID_N = 20000
MID_CASES = {
    # name: (s, graph, pool, K, q, B, k, tol, sketch kind)
    "s025": dict(s=0.25, K=24, q=64, B=16, k=10, tol=1e-7, kind="block"),
    "s050": dict(s=0.50, K=24, q=64, B=16, k=10, tol=1e-7, kind="block"),
    "s075": dict(s=0.75, K=24, q=64, B=16, k=10, tol=1e-7, kind="block"),
    "plain_rad": dict(s=0.50, K=16, q=32, B=1, k=10, tol=1e-8, kind="rademacher"),
}


def mid_inputs(name):
    """(n, edges, cand) of a mid case: the precision workload's Chung-Lu shape (exponent 2.4,
    mean degree 6.62, min degree 1, graph seed 1, pool seed 1 + 7919) at n = 20,000 with
    20,000 candidates; the plain case is the n = 2000 workload (exponent 2.5, mean degree 6,
    seed 0, pool seed 7919)."""
    if name == "plain_rad":
        n = 2000
        E = chung_lu(n, 6.0, 2.5, 0, min_degree=1)
        return n, E, ref_graphs.candidates(n, E, 20000, 7919)
    n = MID_N
    E = chung_lu(n, 2 * 1049866 / 317080, 2.4, 1, min_degree=1)
    return n, E, ref_graphs.candidates(n, E, 20000, 1 + 7919)


def part_mid(name):
    """One mid case -> reference_mid_<name>.npz/.json: sequence, shortlists, SpMV count,
    pole count, the re-rank scores G_q of every shortlisted edge per round (B > 1) and the
    proxy scores of the shortlist per round."""
    from polar_b200.sketch import sketches as host_sketches
    t_start = time.time()
    c = MID_CASES[name]
    n, E, cand = mid_inputs(name)
    G = ref.Graph(n, E, 1e-2)
    # the block and gauss kinds follow the reference's own stream; the Rademacher kind is
    # drawn in the same order by polar_b200.sketch (the reference takes sketches as input)
    sk = ref.sketches(G, cand, c["q"], 2026, kind=c["kind"]) if c["kind"] != "rademacher" else \
        host_sketches(G, cand, c["q"], 2026, kind="rademacher")
    ref.poles = fixed_poles(c["K"])
    cupy.ARGMAX_LOG.clear()
    cupy.ARGSORT_LOG.clear()
    trace = []
    res = ref.polar(G, cand, c["k"], c["s"], q=c["q"], B=c["B"], tol=c["tol"], sketch=sk, trace=trace)
    pre = f"mid_{name}_"
    put(pre + "edges_sum", int(E.sum()))
    put(pre + "m", len(E))
    put(pre + "cand_head", cand[:64])
    put(pre + "cand_sum", int(cand.sum()))
    put(pre + "sketch_sums", [float(np.sum(a)) for a in sk])
    put(pre + "sequence", res["sequence"])
    put(pre + "spmv", res["spmv"])
    put(pre + "p", res["p"])
    short = np.array([t["shortlist"] for t in trace])
    put(pre + "shortlists", short)
    proxy = []
    for rnd, a in enumerate(cupy.ARGSORT_LOG):
        proxy.append(-np.asarray(a)[short[rnd]])
    put(pre + "proxy", np.array(proxy))
    if c["B"] > 1:
        put(pre + "rerank", np.array([np.asarray(a, np.float64) for a in cupy.ARGMAX_LOG]))
    meta[name] = dict(c, n=n, N=len(cand), sigma=1e-2, seconds=time.time() - t_start)
    np.savez_compressed(HERE / f"reference_mid_{name}.npz", **out)
    (HERE / f"reference_mid_{name}.json").write_text(json.dumps(meta, indent=1))
    print(name, res["sequence"], res["spmv"], f"{time.time() - t_start:.1f}s", flush=True)


# ---- dense eigendecomposition oracles (realworld/exact.py) ---------------------------------
def part_exact():
    """realworld/exact.py on small graphs -> reference_exact.npz/.json."""
    import exact as ref_exact
    t_start = time.time()
    cases = {"a": (120, 4.0, 2.5, 31, 160, 41), "b": (200, 6.0, 2.3, 32, 300, 42)}
    for key, (n, deg, gam, gseed, N, cseed) in cases.items():
        E = chung_lu(n, deg, gam, gseed, min_degree=1)
        cand = ref_graphs.candidates(n, E, N, cseed)
        M0 = ref.Graph(n, E, 1e-2).M0.toarray()
        put(f"ex_{key}_edges", E)
        put(f"ex_{key}_cand", cand)
        for obj, s in (("frac", 0.5), ("frac", 0.25), ("er", 1.0), ("logdet", 0.5)):
            tag = f"{obj}{int(round(s * 100)):03d}"
            r = ref_exact.exact_greedy(M0, cand, 4, s, obj=obj)
            put(f"ex_{key}_{tag}_sequence", r["sequence"])
            if obj == "frac":
                put(f"ex_{key}_{tag}_contenders", np.array(r["contenders"]))
            put(f"ex_{key}_{tag}_prefix", ref_exact.eval_prefix(M0, cand, r["sequence"], s, obj=obj))
        seq = [int(x) for x in out[f"ex_{key}_frac050_sequence"]]
        targets = [("frac", 0.25), ("frac", 0.5), ("er", 1.0), ("logdet", 0.5)]
        multi = ref_exact.eval_prefix_multi(M0, cand, seq, targets)
        put(f"ex_{key}_multi", np.array(multi))
        meta[f"ex_{key}_targets"] = targets
        put(f"ex_{key}_twin", ref_exact.twin_gain(M0, cand, 0.5))
        sub = cand[:24]
        best, arg = ref_exact.brute_force(M0, sub, 2, 0.5, obj="frac")
        put(f"ex_{key}_brute_best", best)
        put(f"ex_{key}_brute_arg", arg)
        print(key, out[f"ex_{key}_frac050_sequence"], arg, f"{time.time() - t_start:.1f}s", flush=True)
    meta["exact_cases"] = cases
    np.savez_compressed(HERE / "reference_exact.npz", **out)
    (HERE / "reference_exact.json").write_text(json.dumps(meta, indent=1))
    print("wrote", HERE / "reference_exact.npz", f"{time.time() - t_start:.1f}s")


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--part", default="base", choices=["base", "mid", "exact"])
    ap.add_argument("--case", default=None, help="mid case name (default: all, one after another)")
    a = ap.parse_args()
    if a.part == "base":
        part_base()
    elif a.part == "exact":
        part_exact()
    else:
        for name in ([a.case] if a.case else list(MID_CASES)):
            out.clear()
            meta.clear()
            part_mid(name)
