"""Checks at the workloads' full sizes, where no CPU run of the reference finishes: properties
that hold whatever the size, computed by code independent of the kernels under test.

* Proxy score and stable top-B over 10^6 candidates and 32 poles (the full-scale pool),
  against NumPy's FP64 formula and a stable argsort, with planted exact ties
  (realworld/polar_gpu.py:208-211, 219-221).
* The SpMM on the 4.0M-vertex, 69.5M-nonzero graph against torch's sparse CSR product in
  FP64 (realworld/spmm.py:4-25, polar_gpu.py:71-80).
* A full-scale multi-shift solve with every row active: the true residual
  ||W - (M + tau_j I) X_j|| of every pole, recomputed with torch's CSR product, is within
  the CG tolerance rule of polar_gpu.py:114-116 (a pole stops when |zeta_j| ||r|| <= tol ||w||),
  and the tracked norms h_j (polar_gpu.py:115-117) equal ||X_j||^2; mixed precision tracks
  the same norms within 1e-5.
* The 317k-vertex precision workload's greedy for a few rounds: mixed precision selects the
  FP64 sequence with every marginal within 1e-6 relative.
Needs a B200 (about two minutes, most of it generating the 4.0M-vertex graph on the host).
"""
import numpy as np
import pytest

from polar_b200.synth import CONFIGS, chung_lu, make_config

pytestmark = pytest.mark.gpu


def _rel(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300)


@pytest.fixture(scope="module")
def full_graph():
    import polar_b200 as pg
    c = CONFIGS["full-n4M"]
    E = chung_lu(c["n"], c["mean_deg"], c["gamma"], c["seed"], dmax=c["dmax"], min_degree=1)
    G = pg.Graph(c["n"], E, c["sigma"])
    return G, c


def _torch_laplacian(G):
    """Adjacency of G as a torch FP64 CSR tensor on the device and the degrees."""
    import torch
    crow = G.indptr.to(torch.int64)
    col = G.indices.to(torch.int64)
    adj = torch.sparse_csr_tensor(crow, col, torch.ones(col.numel(), dtype=torch.float64, device=col.device),
                                  size=(G.n, G.n))
    deg = (crow[1:] - crow[:-1]).to(torch.float64)
    return adj, deg


# ---------------------------------------------------------------------------------------
def test_score_topb_full_pool():
    """N = 10^6 candidates, p = 32 poles: every score (score_all keeps the scores of dead
    candidates too) to 1e-14 relative of the NumPy formula, the shortlist equal to a stable
    argsort of the live scores (ties to the lower index), for B = 16 and B = 1, with dead
    candidates, a dead one above all others, and planted exact ties at the top."""
    import torch

    from polar_b200 import _lib
    from polar_b200.quadrature import fixed_rule
    lib = _lib.load()
    dev = torch.device("cuda", 0)
    p, N, sigma = 32, 1_000_000, 1e-2
    tau, om = fixed_rule(0.5, p, np.sqrt(sigma * 3e4))
    rng = np.random.default_rng(5)
    h = rng.gamma(2.0, 1e-3, size=(p, N))
    t = rng.gamma(2.0, 1e-2, size=(p, N))
    hot = [400_001, 17, 999_999]             # one tie group at the top: equal (h, t) columns
    h[:, hot] = 10.0
    t[:, hot] = 0.0
    h[:, 123_456] = 20.0                     # better than the tie group but dead
    t[:, 123_456] = 0.0
    live = np.ones(N, np.uint8)
    live[123_456] = 0
    live[rng.choice(N, 5000, replace=False)] = 0
    live[hot] = 1
    sc_ref = np.sum(om[:, None] * h / (1.0 + t + (sigma + tau)[:, None] * h), axis=0)
    hd, td = (torch.as_tensor(x).to(dev) for x in (h, t))
    taud, omd = (torch.as_tensor(x).to(dev) for x in (tau, om))
    lived = torch.as_tensor(live).to(dev)
    for B in (16, 1):
        idx = torch.empty(B, dtype=torch.int64, device=dev)
        sco = torch.empty(B, dtype=torch.float64, device=dev)
        allsc = torch.empty(N, dtype=torch.float64, device=dev)
        tmp = torch.empty(max(lib.polar_topb_tmp_bytes(N, B), 256), dtype=torch.uint8, device=dev)
        st = torch.cuda.current_stream(dev).cuda_stream
        _lib.check(lib.polar_score_topb(hd.data_ptr(), td.data_ptr(), taud.data_ptr(), omd.data_ptr(), sigma, p,
                                        N, lived.data_ptr(), 0, B, idx.data_ptr(), sco.data_ptr(),
                                        allsc.data_ptr(), tmp.data_ptr(), st), "score_topb")
        s_gpu = allsc.cpu().numpy()              # every candidate's score, dead ones included
        assert _rel(s_gpu, sc_ref) < 1e-14
        masked = np.where(live > 0, s_gpu, -np.inf)
        order = np.argsort(-masked, kind="stable")[:B]
        got = idx.cpu().numpy()
        assert np.array_equal(got, order), (got, order)
        assert np.array_equal(sco.cpu().numpy(), masked[order])
        assert list(got[:min(B, 3)]) == sorted(hot)[:min(B, 3)]   # the tie group, lowest index first


# ---------------------------------------------------------------------------------------
@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_spmm_full_graph_matches_torch_csr(full_graph, prec):
    """Op apply on the full-scale graph at the shortlist width R = 16 (heavy-row chunks and
    sliced-ELL slices both in play) with three added edges, against torch's FP64 CSR product
    of the same operator: 1e-13 relative in FP64; 2e-6 for FP32 inputs and outputs (the row
    sums are FP64, so the bound is FP32 output rounding)."""
    import torch

    import polar_b200 as pg
    G, c = full_graph
    op = pg.Op(G)
    added = [(0, G.n - 1), (5, 3_000_000), (0, 1)]
    for a, b in added:
        op.add(a, b)
    dt = torch.float64 if prec == "fp64" else torch.float32
    gen = torch.Generator(device="cuda").manual_seed(16)
    X = torch.randn((G.n, 16), dtype=torch.float64, device="cuda", generator=gen).to(dt)
    shift = 0.37
    Y = op(X, shift).double()
    adj, deg = _torch_laplacian(G)
    X64 = X.double()
    ref = (deg + G.sigma + shift)[:, None] * X64 - adj @ X64
    for a, b in added:
        dlt = X64[a] - X64[b]
        ref[a] += dlt
        ref[b] -= dlt
    err = ((Y - ref).abs().max() / ref.abs().max()).item()
    print(f"full-scale SpMM {prec}: max error / max |Y| {err:.3e}")
    assert err < (1e-13 if prec == "fp64" else 2e-6), err


@pytest.fixture(scope="module")
def full_solves(full_graph):
    """One multi-shift solve of the full-scale pole set (K = 32, tol 1e-6) for two incidence
    columns, every row active, in FP64 and in mixed precision."""
    import torch

    import polar_b200 as pg
    from polar_b200.quadrature import poles
    G, c = full_graph
    tau, om, _ = poles("frac", c["s"], G.sigma, G.Lam(c["k"]), 1e-2, K=c["K"])
    pairs = [(0, G.n - 1), (1000, 2_000_000)]
    W = torch.zeros((G.n, len(pairs)), dtype=torch.float64, device="cuda")
    for j, (a, b) in enumerate(pairs):
        W[a, j] = 1.0
        W[b, j] = -1.0
    active = np.arange(G.n)
    out = {}
    for prec in ("fp64", "mixed"):
        X, h, it = pg.msolve(pg.Op(G), W, tau, active, c["tol"], track=True, precision=prec)
        out[prec] = (X, h, it)
    return G, c, tau, W, out


def test_full_scale_solve_true_residuals(full_solves):
    """FP64: for every pole j and column, ||W - (M + tau_j I) X_j|| / ||W|| <= 1.5 tol, the
    stopping rule (|zeta_j| ||r|| <= tol ||w||) plus FP64 drift of the recurred residual;
    the residual is recomputed with torch's CSR product, not this library's SpMM.  The
    tracked norms h_j, a recurrence that rests on CG's orthogonality relations, equal
    ||X_j||^2 over all rows to 1e-5."""
    import torch
    G, c, tau, W, out = full_solves
    X, h, it = out["fp64"]
    p, n, R = X.shape
    adj, deg = _torch_laplacian(G)
    taud = torch.as_tensor(tau, device="cuda")
    AX = (adj @ X.permute(1, 0, 2).reshape(n, p * R)).reshape(n, p, R).permute(1, 0, 2)
    Rj = W[None] - ((deg + G.sigma)[None, :, None] + taud[:, None, None]) * X + AX
    rel = (Rj.norm(dim=1) / W.norm(dim=0)[None]).cpu().numpy()
    hx = (X * X).sum(dim=1).cpu().numpy()
    herr = float(np.max(np.abs(h.cpu().numpy() - hx) / hx))
    print(f"full-scale FP64 solve: iterations {list(it)}, max true residual / ||w|| {rel.max():.3e}, "
          f"tracked vs direct ||X_j||^2 {herr:.3e}")
    assert rel.max() <= 1.5 * c["tol"], rel.max()
    assert herr < 1e-5, herr
    assert np.all(it > 100)


def test_full_scale_solve_mixed_norms(full_solves):
    """Mixed precision against FP64 at full scale: the tracked norms h_j (the quantities the
    proxy and re-rank scores are built from) within 1e-5 relative for every pole and column,
    and at most 25 % more seed iterations."""
    G, c, tau, W, out = full_solves
    X64, h64, it64 = out["fp64"]
    Xm, hm, itm = out["mixed"]
    assert Xm.element_size() == 4
    h64, hm = h64.cpu().numpy(), hm.cpu().numpy()
    err = float(np.max(np.abs(hm - h64) / np.abs(h64)))
    print(f"full-scale mixed solve: iterations {list(itm)} (FP64 {list(it64)}), max rel. diff. of h {err:.3e}")
    assert err < 1e-5, err
    assert np.all(itm <= 1.25 * it64 + 10)


# ---------------------------------------------------------------------------------------
def test_precision_workload_mixed_matches_fp64():
    """The 317,080-vertex precision workload (200,000 candidates, K = 24, q = 64, B = 16,
    tol 1e-7), four rounds: mixed precision selects the FP64 sequence, with every round's
    marginal within 1e-6 relative of FP64's and the same shortlist in every round, but for
    at most one edge swapped at a near-tie of the proxy in the B-th place."""
    import polar_b200 as pg
    E, n, cand, c = make_config("precision-n317k")
    G = pg.Graph(n, E, c["sigma"])
    sk = pg.sketches(G, cand, c["q"], 2026, device=True)
    res = {}
    for prec in ("fp64", "mixed"):
        trace = []
        res[prec] = pg.polar(G, cand, 4, c["s"], q=c["q"], B=c["B"], tol=c["tol"], sketch=sk, K=c["K"],
                             precision=prec, trace=trace)
        res[prec]["trace"] = trace
    f, m = res["fp64"], res["mixed"]
    assert m["sequence"] == f["sequence"]
    mf, mm = np.asarray(f["marginals"]), np.asarray(m["marginals"])
    err = float(np.max(np.abs(mm - mf) / np.abs(mf)))
    print(f"precision workload, 4 rounds: sequence {m['sequence']}, max rel. marginal error {err:.3e}")
    assert err < 1e-6, err
    for tf, tm in zip(f["trace"], m["trace"]):       # one swap allowed at a near-tie in B-th place
        assert len(set(tf["shortlist"]) ^ set(tm["shortlist"])) <= 2
