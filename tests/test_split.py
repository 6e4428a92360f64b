"""Column split of the greedy over several ranks (polar_b200.split): the exchange protocol
with two gloo ranks on CPU, each rank holding half of the sketch columns and solving half
of every shortlist through a dense FP64 shard defined here (exact solves, the same
formulas as realworld/polar_gpu.py:200-249 on its columns).  Checked: the same sequence
as one rank holding every column, the same caches h, t (all-reduced partial sums) and
re-rank scores, and the sequence of the oracle's greedy on the same inputs.  The device
shard (DeviceShard, libpolar kernels) is checked on one GPU against Greedy."""
import os
import socket
import sys
from pathlib import Path

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT))

from polar_b200.split import ColumnSplit, Comm, owner_of, share  # noqa: E402

N_V, N_C, Q, KP, B, K_ROUNDS, S, SIGMA = 80, 150, 8, 8, 4, 5, 0.5, 1e-2


def _inputs():
    import polar_b200 as pg
    from polar_b200.synth import candidates, chung_lu
    E = chung_lu(N_V, 5.0, 2.5, 3, min_degree=1)
    cand = candidates(N_V, E, N_C, 11)
    G = pg.Graph(N_V, E, SIGMA, device="cpu")
    sk = pg.sketches(G, cand, Q, 2026)
    tau, om, _ = pg.poles("frac", S, SIGMA, G.Lam(K_ROUNDS), 1e-2, K=KP)
    return E, cand, sk, np.asarray(tau), np.asarray(om)


class DenseShard:
    """One rank's columns [c0, c1) of a greedy run with exact dense FP64 solves."""

    naive = False

    def __init__(self, E, cand, sk, tau, om, c0, c1):
        n = N_V
        A = np.zeros((n, n))
        for a, b in E:
            A[a, a] += 1
            A[b, b] += 1
            A[a, b] -= 1
            A[b, a] -= 1
        self.M = A + SIGMA * np.eye(n)
        self.cand = np.asarray(cand)
        self.tau, self.om = tau, om
        Z, F, Gc = sk
        self.Z, self.F, self.Gc = Z[:, c0:c1].copy(), F[:, c0:c1].copy(), Gc[:, c0:c1].copy()
        self.active = np.unique(self.cand)
        es = np.searchsorted(self.active, self.cand)
        self.ea, self.eb = es[:, 0], es[:, 1]
        self.k, self.B = K_ROUNDS, B
        self.live = np.ones(len(cand), bool)
        self.U = np.zeros((len(tau), len(self.active), B))
        self.seq, self.marg = [], []

    def _solve(self, W):
        n = self.M.shape[0]
        return np.stack([np.linalg.solve(self.M + t * np.eye(n), W) for t in self.tau])

    def bank(self):
        self.X = self._solve(self.Z)[:, self.active]
        self.Y = self._solve(self.F)[:, self.active]
        self.h = torch.as_tensor(((self.X[:, self.ea] - self.X[:, self.eb]) ** 2).sum(-1))
        self.t = torch.as_tensor(((self.Y[:, self.ea] - self.Y[:, self.eb]) ** 2).sum(-1))

    def caches(self):
        return self.h, self.t

    def live_count(self):
        return int(self.live.sum())

    def shortlist(self, Br):
        h, t = self.h.numpy(), self.t.numpy()
        td = self.tau[:, None]
        sc = (self.om[:, None] * h / (1 + t + (SIGMA + td) * h)).sum(0)
        sc[~self.live] = -np.inf
        self.short = np.argsort(-sc, kind="stable")[:Br]

    def solve_rerank(self, b0, b1):
        cols = self.short[b0:b1]
        if len(cols) == 0:
            return torch.empty(0, dtype=torch.float64)
        W = np.zeros((N_V, len(cols)))
        W[self.cand[cols, 0], np.arange(len(cols))] = 1.0
        W[self.cand[cols, 1], np.arange(len(cols))] = -1.0
        Ufull = self._solve(W)
        hh = (Ufull ** 2).sum(1)
        Ua = Ufull[:, self.active]
        self.U[:, :, b0:b1] = Ua
        r = np.arange(len(cols))
        bu = Ua[:, self.ea[cols], r] - Ua[:, self.eb[cols], r]
        return torch.as_tensor((self.om[:, None] * hh / (1 + bu)).sum(0))

    def winner_column(self, j):
        return torch.as_tensor(np.ascontiguousarray(self.U[:, :, j]))

    def empty_column(self):
        return torch.empty(self.U.shape[:2], dtype=torch.float64)

    def take_winner(self, j, u, owned, score):
        if not owned:
            self.U[:, :, j] = u.numpy()
        self.j = j
        e = int(self.short[j])
        self.seq.append(e)
        self.marg.append(score)
        self.live[e] = False
        return e

    def maintain_delta(self):
        e = self.seq[-1]
        aa, bb = self.ea[e], self.eb[e]
        u = self.U[:, :, self.j]
        xi = self.X[:, aa] - self.X[:, bb]
        eta = self.Gc[e][None] - (self.Y[:, aa] - self.Y[:, bb])
        D = 1 + u[:, aa] - u[:, bb]
        cc = (u[:, self.ea] - u[:, self.eb]) / D[:, None]
        wX = np.einsum("pnq,pq->pn", self.X, xi)
        wY = np.einsum("pnq,pq->pn", self.Y, eta)
        dh = -2 * cc * (wX[:, self.ea] - wX[:, self.eb]) + cc * cc * (xi * xi).sum(1)[:, None]
        dt = 2 * cc * (wY[:, self.ea] - wY[:, self.eb]) + cc * cc * (eta * eta).sum(1)[:, None]
        self.X -= u[:, :, None] * xi[:, None, :] / D[:, None, None]
        self.Y += u[:, :, None] * eta[:, None, :] / D[:, None, None]
        return torch.as_tensor(dh), torch.as_tensor(dt)

    def apply_cache(self, dh, dt):
        self.h = torch.clamp(self.h + dh, min=0.0)
        self.t = torch.clamp(self.t + dt, min=0.0)

    def finish(self, e):
        a, b = self.cand[e]
        self.F[a] += self.Gc[e]
        self.F[b] -= self.Gc[e]
        for x, y in ((a, a), (b, b)):
            self.M[x, y] += 1
        self.M[a, b] -= 1
        self.M[b, a] -= 1


def _run(comm):
    E, cand, sk, tau, om = _inputs()
    c0, c1 = share(Q, comm.world, comm.rank)
    shard = DenseShard(E, cand, sk, tau, om, c0, c1)
    run = ColumnSplit(shard, comm)
    run.bank()
    h0 = shard.h.clone()
    for _ in range(K_ROUNDS):
        run.step()
    return shard.seq, shard.marg, h0.numpy(), shard.h.numpy(), shard.t.numpy()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        out[rank] = _run(Comm())
    finally:
        dist.destroy_process_group()


def test_shares_cover_the_range():
    for total in (1, 3, 16, 17, 64):
        for world in (1, 2, 3, 8):
            parts = [share(total, world, r) for r in range(world)]
            assert parts[0][0] == 0 and parts[-1][1] == total
            assert all(parts[r][1] == parts[r + 1][0] for r in range(world - 1))
            assert max(h - l for l, h in parts) - min(h - l for l, h in parts) <= 1
            for j in range(total):
                lo, hi = parts[owner_of(j, total, world)]
                assert lo <= j < hi


def test_column_split_two_ranks_gloo():
    one = _run(Comm())
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    mp.spawn(_rank_main, args=(2, _free_port(), out), nprocs=2, join=True)
    for r in range(2):
        seq, marg, h0, h, t = out[r]
        assert seq == one[0]
        np.testing.assert_allclose(marg, one[1], rtol=1e-12)
        np.testing.assert_allclose(h0, one[2], rtol=1e-12, atol=1e-15)
        np.testing.assert_allclose(h, one[3], rtol=1e-10, atol=1e-14)
        np.testing.assert_allclose(t, one[4], rtol=1e-10, atol=1e-14)
    # the oracle's greedy (CG solves, polar_gpu.py:180-254) on the same inputs
    from oracle import polar_oracle as O
    E, cand, sk, _, _ = _inputs()
    ref = O.polar(O.Graph(N_V, E, SIGMA), cand, K_ROUNDS, S, q=Q, B=B, tol=1e-12, sketch=sk, K=KP)
    assert ref["sequence"] == one[0]
    np.testing.assert_allclose(ref["marginals"], one[1], rtol=1e-8)


@pytest.mark.gpu
@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_device_shard_matches_greedy(prec):
    import polar_b200 as pg
    from polar_b200.split import polar_split
    from polar_b200.synth import candidates, chung_lu
    n = 2000
    E = chung_lu(n, 6.0, 2.5, 0, min_degree=1)
    cand = candidates(n, E, 3000, 11)
    G = pg.Graph(n, E, 1e-2)
    sk = pg.sketches(G, cand, 32, 2026)
    ref = pg.polar(G, cand, 4, 0.5, q=32, B=6, tol=1e-8, sketch=sk, K=16, precision=prec)
    res = polar_split(G, cand, 4, 0.5, q=32, B=6, tol=1e-8, sketch=sk, K=16, precision=prec)
    assert res["sequence"] == ref["sequence"]
    np.testing.assert_allclose(res["marginals"], ref["marginals"], rtol=1e-9 if prec == "fp64" else 1e-6)
