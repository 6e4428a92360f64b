"""Host-side logic and the C-ABI library surface.  CPU only."""
import re
from pathlib import Path

import numpy as np
import pytest

import polar_b200 as pg
from oracle import polar_oracle as O
from polar_b200 import _lib
from polar_b200.synth import chung_lu

ROOT = Path(__file__).resolve().parent.parent
GOLD = ROOT / "tests" / "golden"


def test_library_exports_every_declared_symbol():
    header = (ROOT / "include" / "polar.h").read_text()
    declared = set(re.findall(r"^\s*(?:[\w\*\s]+?)\b(polar_\w+)\s*\(", header, re.M))
    assert len(declared) >= 18
    lib = _lib.load()
    for name in declared:
        assert hasattr(lib, name), name
    assert set(_lib.SIGNATURES) == declared
    assert lib.polar_version() >= 1


def test_quadrature_matches_oracle_and_reference():
    z = np.load(GOLD / "reference_vectors.npz")
    import json
    meta = json.loads((GOLD / "reference_vectors.json").read_text())
    for i, (s, a, zz, eps) in enumerate(meta["composite_cases"]):
        tau, om, b = pg.composite(s, a, zz, eps)
        np.testing.assert_allclose(tau, z[f"composite{i}_tau"], rtol=1e-13)
        np.testing.assert_allclose(om, z[f"composite{i}_om"], rtol=1e-12)
    for s in (0.25, 0.5, 0.75):
        for K in (8, 16, 24, 32):
            t1, o1 = pg.fixed_rule(s, K, 3.0)
            t2, o2 = O.fixed_rule(s, K, 3.0)
            np.testing.assert_allclose(t1, t2, rtol=1e-13)
            np.testing.assert_allclose(o1, o2, rtol=1e-13)
            assert np.all(np.diff(t1) > 0) and np.all(o1 > 0)


@pytest.mark.parametrize("s", [0.25, 0.5, 0.75])
def test_fixed_rule_reproduces_power(s):
    # sum_j om_j / (x + tau_j) ~= x^-s on [sigma, Lam]; the error falls with K.
    sigma, Lam = 1e-2, 300.0
    x = np.geomspace(sigma, Lam, 200)
    errs = []
    for K in (8, 16, 32):
        tau, om = pg.fixed_rule(s, K, np.sqrt(sigma * Lam))
        approx = (om[None, :] / (x[:, None] + tau[None, :])).sum(1)
        errs.append(np.max(np.abs(approx / x ** (-s) - 1)))
    assert errs[0] > errs[1] > errs[2]
    assert errs[2] < 2e-4  # K=32 on a 3e4 spectral range


def test_composite_rule_known_answer():
    # Quadrature KAT of synthetic/controls/verify_stieltjes.py:43-52: on a dense n=50
    # graph the composite-rule marginals match eigenvalue marginals within 256*4^-r.
    rng = np.random.default_rng(7)
    n, sigma, s = 50, 0.5, 0.5
    A = np.triu(rng.random((n, n)) < 0.08, 1)
    A = (A + A.T).astype(float)
    i = np.arange(n)
    A[i, (i + 1) % n] = A[(i + 1) % n, i] = 1.0
    M = np.diag(A.sum(1)) - A + sigma * np.eye(n)
    lam = np.linalg.eigvalsh(M)
    pairs = np.argwhere(np.triu(A == 0, 1))[:200]
    E = np.zeros((n, len(pairs)))
    E[pairs[:, 0], np.arange(len(pairs))] = 1
    E[pairs[:, 1], np.arange(len(pairs))] = -1
    exact = np.array([np.sum(lam ** -s) - np.sum(np.linalg.eigvalsh(M + np.outer(b, b)) ** -s) for b in E.T])
    for eps in (1e-1, 1e-2, 1e-4):
        tau, om, bound = pg.composite(s, sigma, lam[-1] + 2, eps)
        approx = np.zeros(len(pairs))
        for tj, wj in zip(tau, om):
            X = np.linalg.solve(M + tj * np.eye(n), E)
            approx += wj * np.sum(X * X, 0) / (1 + np.sum(E * X, 0))
        assert np.max(np.abs(approx - exact) / exact) <= bound


def test_sketches_match_reference():
    z = np.load(GOLD / "reference_vectors.npz")
    G = O.Graph(300, z["g1_edges"], 1e-2)
    cand = z["g1_cand"]
    for kind in ("block", "gauss"):
        Z, F, Gc = pg.sketches(G, cand, 8, 2026, kind=kind)
        np.testing.assert_allclose(Z, z[f"g1_sk_{kind}_Z"], rtol=0, atol=1e-14)
        np.testing.assert_allclose(F, z[f"g1_sk_{kind}_F"], rtol=0, atol=1e-14)
        np.testing.assert_allclose(Gc, z[f"g1_sk_{kind}_Gc"], rtol=0, atol=1e-14)
    Z, F, Gc = pg.sketches(G, cand, 16, 5, kind="rademacher")
    assert np.allclose(np.abs(Gc), 0.25) and np.allclose(Z.mean(0), 0)
    assert np.allclose(np.linalg.norm(Gc, axis=1), 1.0)


def test_chung_lu_shape():
    E = chung_lu(5000, 8.0, 2.2, 3, dmax=400)
    assert len(E) == 20000
    assert np.all(E[:, 0] < E[:, 1])
    assert len(np.unique(E[:, 0] * 5000 + E[:, 1])) == len(E)
    deg = np.bincount(E.ravel(), minlength=5000)
    assert 150 < deg.max() <= 800


def test_graph_host_structures_and_heavy_split():
    import torch
    E = chung_lu(3000, 6.0, 2.2, 5)
    G = pg.Graph(3000, E, 1e-2, heavy_thresh=16, device="cpu")
    M = O.Graph(3000, E, 1e-2).M0
    assert (G.M0.get() != M).nnz == 0
    degs = np.diff(G._indptr_h)
    heavy = np.flatnonzero(degs > 16)
    assert G.nheavy == len(heavy) > 0
    lo = G.chunk_lo.numpy()
    hi = G.chunk_hi.numpy()
    row = G.chunk_row.numpy()
    off = G.hchunk_off.numpy()
    for h, r in enumerate(heavy):
        segs = list(zip(lo[off[h]:off[h + 1]], hi[off[h]:off[h + 1]]))
        assert segs[0][0] == G._indptr_h[r] and segs[-1][1] == G._indptr_h[r + 1]
        assert all(b0 == a1 for (_, a1), (b0, _) in zip(segs[:-1], segs[1:]))
        assert all(0 < b - a <= G.CHUNK for a, b in segs)
        assert len(segs) == -(-(G._indptr_h[r + 1] - G._indptr_h[r]) // G.CHUNK)
        assert np.all(row[off[h]:off[h + 1]] == h)
    s = G.struct()
    assert s.nheavy == G.nheavy and s.nchunks == G.nchunks and s.d_wts is None
    assert G.Lam(3) == pytest.approx(1e-2 + 2 * G.dmax + 12)


def test_status_mapping():
    with pytest.raises(RuntimeError, match="iteration cap"):
        _lib.check(_lib.POLAR_ERR_ITER_CAP)
    with pytest.raises(_lib.PolarError):
        _lib.check(_lib.POLAR_ERR_BAD_ARG, "x")


def test_batch_problem_struct_matches_header(tmp_path):
    """ctypes' polar_msolve_problem has the C layout: size and every field offset, as gcc
    lays out the struct declared in include/polar.h."""
    import ctypes
    import shutil
    import subprocess
    if shutil.which("gcc") is None:
        pytest.skip("gcc not available")
    names = [f[0] for f in _lib.MsolveProblem._fields_]
    src = tmp_path / "layout.c"
    body = "".join(f'  printf("{nm} %zu\\n", offsetof(polar_msolve_problem, {nm}));\n' for nm in names)
    src.write_text('#include <stdio.h>\n#include <stddef.h>\n#include "polar.h"\nint main(void) {\n'
                   '  printf("size %zu\\n", sizeof(polar_msolve_problem));\n' + body + "  return 0;\n}\n")
    exe = tmp_path / "layout"
    subprocess.check_call(["gcc", "-I", str(ROOT / "include"), str(src), "-o", str(exe)])
    got = dict(line.split() for line in subprocess.check_output([str(exe)], text=True).splitlines())
    assert int(got["size"]) == ctypes.sizeof(_lib.MsolveProblem)
    for nm in names:
        assert int(got[nm]) == getattr(_lib.MsolveProblem, nm).offset, nm


def test_autotune_lane_resolution_matches_library():
    """The tuner's model of how lane bytes resolve to lanes per row agrees with the
    library's sliced-ELL height (32 / lanes) for every width and precision (host-only
    calls, no device needed)."""
    from polar_b200 import autotune
    lib = _lib.load()
    try:
        for prec in (_lib.POLAR_FP64, _lib.POLAR_MIXED):
            maxc = 128 if prec == _lib.POLAR_MIXED else 64
            for R in (1, 3, 8, 16, 33, 64, maxc):
                if R > maxc:
                    continue
                ld = autotune._ld(prec, R)
                for lb in (16, 32, 64):
                    lib.polar_set_spmm_lane_bytes(lb)
                    lanes = autotune._lanes(prec, ld, lb)
                    assert lib.polar_sell_rows(prec, R) == 32 // lanes, (prec, R, lb)
                    assert lib.polar_heavy_threshold(prec, R) == max(16, 8 * lanes), (prec, R, lb)
    finally:
        lib.polar_set_spmm_lane_bytes(0)


def test_batch_rejects_bad_arguments_before_launch():
    """polar_msolve_batch checks its arguments on the host: no problems, too many, an
    unknown precision and a missing pointer are BAD_ARG without touching a device."""
    import ctypes
    lib = _lib.load()
    assert lib.polar_msolve_batch(None, 1, _lib.POLAR_FP64, None) == _lib.POLAR_ERR_BAD_ARG
    probs = (_lib.MsolveProblem * 65)()
    assert lib.polar_msolve_batch(probs, 0, _lib.POLAR_FP64, None) == _lib.POLAR_ERR_BAD_ARG
    assert lib.polar_msolve_batch(probs, 65, _lib.POLAR_FP64, None) == _lib.POLAR_ERR_BAD_ARG
    assert lib.polar_msolve_batch(probs, 1, 7, None) == _lib.POLAR_ERR_BAD_ARG
    g = _lib.PolarGraph()
    g.n = 10
    probs[0].g = ctypes.pointer(g)
    probs[0].R = 4
    assert lib.polar_msolve_batch(probs, 1, _lib.POLAR_FP64, None) == _lib.POLAR_ERR_BAD_ARG
    assert b"null pointer" in lib.polar_last_error()


def test_batch_specs_follow_the_workload_rules():
    """The 48-graph workload: n log-uniform in [5k, 400k], mean degree in [4, 20],
    exponent in [2.2, 2.8], sigma and s from their three values; seeded."""
    from polar_b200.synth import batch_specs
    sp = batch_specs()
    assert len(sp) == 48 and sp == batch_specs()
    assert all(5000 <= x["n"] <= 400000 for x in sp)
    assert all(4.0 <= x["mean_deg"] <= 20.0 and 2.2 <= x["gamma"] <= 2.8 for x in sp)
    assert {x["sigma"] for x in sp} == {1e-3, 1e-2, 1e-1}
    assert {x["s"] for x in sp} == {0.3, 0.5, 0.7}
    assert len({x["seed"] for x in sp}) == 48


def test_batch_cta_split(tmp_path):
    """The persistent batch driver's CTA split (csrc/batch_split.h, host C++): every
    problem gets at least one CTA and at most its cap, the total never exceeds the grid,
    spare CTAs go out in proportion to cost, and a grid larger than the caps allow is
    left partly unused."""
    import shutil
    import subprocess
    if shutil.which("g++") is None:
        pytest.skip("g++ not available")
    src = tmp_path / "split.cc"
    src.write_text(r'''
#include <cstdio>
#include "batch_split.h"
int main() {
  using polar::split_ctas;
  std::vector<int> c;
  split_ctas({1, 1, 1, 1}, {100, 100, 100, 100}, 8, c);
  printf("%d %d %d %d\n", c[0], c[1], c[2], c[3]);
  split_ctas({1, 3}, {100, 100}, 10, c);
  printf("%d %d\n", c[0], c[1]);
  split_ctas({1, 1000}, {100, 3}, 50, c);
  printf("%d %d\n", c[0], c[1]);
  split_ctas({5, 1, 1}, {2, 2, 2}, 148, c);
  printf("%d %d %d\n", c[0], c[1], c[2]);
  split_ctas({1, 2, 3, 4, 5}, {1000, 1000, 1000, 1000, 1000}, 148, c);
  int s = 0;
  for (int x : c) s += x;
  printf("%d %d %d %d %d %d\n", c[0], c[1], c[2], c[3], c[4], s);
  return 0;
}
''')
    exe = tmp_path / "split"
    subprocess.check_call(["g++", "-std=c++17", "-I", str(ROOT / "polar_b200" / "csrc"), str(src), "-o", str(exe)])
    out = [list(map(int, ln.split())) for ln in subprocess.check_output([str(exe)], text=True).splitlines()]
    assert out[0] == [2, 2, 2, 2]                 # equal costs share evenly
    assert out[1] == [3, 7]                       # 8 spare CTAs split 1:3 (2 and 6), one more by remainder
    assert out[2] == [47, 3]                      # the costly problem is capped, the rest goes on
    assert out[3] == [2, 2, 2]                    # caps bound the total below the grid
    c = out[4]
    assert c[5] == 148 and all(x >= 1 for x in c[:5])
    assert c[:5] == sorted(c[:5])                 # more cost, no fewer CTAs


def test_candidates_batched_identity_and_cache(tmp_path):
    """The batched pool equals the reference rule's one-pair-per-draw pool (the oracle's
    restatement of realworld/graphs.py:61-69) at N = 10^5, and make_config's .npz cache
    returns the generated workload unchanged."""
    from oracle import polar_oracle as O
    from polar_b200.synth import candidates, chung_lu, make_config
    n = 317080
    E = chung_lu(n, 6.6, 2.4, 1, min_degree=1)
    np.testing.assert_array_equal(candidates(n, E, 100_000, 8), O.candidates(n, E, 100_000, 8))
    E1, n1, c1, _ = make_config("precision-n317k", n=4000, N=3000, cache=str(tmp_path))
    E2, n2, c2, _ = make_config("precision-n317k", n=4000, N=3000, cache=str(tmp_path))
    assert len(list(tmp_path.iterdir())) == 1
    np.testing.assert_array_equal(E1, E2)
    np.testing.assert_array_equal(c1, c2)


def test_device_ingestion_matches_host_csr_and_slices():
    """The torch ingestion (run here on CPU tensors; on the GPU for Graph on a CUDA device)
    builds the scipy CSR and the sliced ELL of the host path exactly."""
    import scipy.sparse as sp
    import torch
    from polar_b200.graph import csr_from_edges, sell_slices, sell_slices_torch
    from polar_b200.synth import chung_lu
    n = 5000
    E = chung_lu(n, 8.0, 2.2, 5, min_degree=1)
    u, v = E[:, 0], E[:, 1]
    A = sp.csr_matrix((np.ones(2 * len(u)), (np.r_[u, v], np.r_[v, u])), shape=(n, n))
    A.sum_duplicates()
    A.sort_indices()
    ip, ind, cnt = csr_from_edges(n, torch.as_tensor(u), torch.as_tensor(v))
    assert np.array_equal(ip.numpy(), A.indptr) and np.array_equal(ind.numpy(), A.indices)
    assert int(cnt.max()) == 1
    deg = np.diff(A.indptr)
    for thresh, S in ((32, 8), (512, 4), (10 ** 6, 16)):
        ref = sell_slices(A.indptr.astype(np.int32), A.indices.astype(np.int32), deg <= thresh, S, window=512)
        got = sell_slices_torch(ip, ind, torch.as_tensor(deg <= thresh), S, window=512)
        for r, g in zip(ref, got):
            assert np.array_equal(r, g.numpy())
    # a repeated edge shows as a merged count of 2
    _, _, cnt = csr_from_edges(4, torch.tensor([0, 1, 0]), torch.tensor([1, 2, 1]))
    assert sorted(cnt.tolist()) == [1, 1, 2, 2]


def test_oracle_threads_give_identical_solves():
    """The oracle's threaded sparse product and shifted updates (the bench's CPU legs use all
    host threads) compute every element as the one-thread path does."""
    from oracle import polar_oracle as O
    from polar_b200.quadrature import poles
    from polar_b200.synth import candidates, chung_lu
    n = 3000
    E = chung_lu(n, 6.0, 2.4, 2, min_degree=1)
    cand = candidates(n, E, 2000, 5)
    G = O.Graph(n, E, 1e-2)
    tau, _, _ = poles("frac", 0.5, 1e-2, G.Lam(5), 1e-2, K=12)
    act = np.unique(cand)
    W = np.zeros((n, 6))
    W[cand[:6, 0], np.arange(6)] = 1.0
    W[cand[:6, 1], np.arange(6)] = -1.0
    one = O.msolve(O.Op(G), W, tau, act, 1e-8, track=True)
    many = O.msolve(O.Op(G, threads=4), W, tau, act, 1e-8, track=True, threads=4)
    for a, b in zip(one, many):
        assert np.array_equal(a, b)
