"""Greedy POLAR with its right-hand sides split over the ranks of a process group, one GPU
per rank (realworld/polar_gpu.py:180-254 is the one-GPU form; the reference has no
multi-GPU path).

The bank's q sketch columns (with them the X / Y bank columns and the F / Gc columns) and
each round's B shortlist columns are independent right-hand sides, so rank r solves a
contiguous share of each.  The exchanges, taken in the same order on every rank:
  * after the bank: all-reduce (sum) of the partial caches h, t (p x N each), since
    h_je = sum_c (X_j[a,c] - X_j[b,c])^2 is a sum over sketch columns;
  * every round: all-gather of the shortlist's re-rank scores, broadcast of the winner's
    solve column u (p x nA) from the rank that solved it, and all-reduce (sum) of the
    per-rank cache changes dh, dt (p x N each) before they are clamped in,
    h = max(0, h + dh), t = max(0, t + dt) (polar_gpu.py:246-247).
Proxy scores, the stable top-B and the winner choice then run identically on every rank.
The operator's added edges and the F columns are updated locally by every rank.

The exchange protocol (ColumnSplit) is separate from the per-rank compute (a shard
object): DeviceShard runs the libpolar kernels on this rank's GPU; the protocol only sees
tensors, so its host logic runs the same with gloo on CPU.
"""
import numpy as np
import torch

from . import _lib
from .greedy import Greedy, _OBJ
from .sketch import sketches
from .solver import msolve

__all__ = ["share", "Comm", "ColumnSplit", "DeviceShard", "polar_split"]


def share(total, world, rank):
    """Contiguous, balanced share [lo, hi) of `total` items for `rank` of `world`."""
    return (rank * total) // world, ((rank + 1) * total) // world


def owner_of(j, total, world):
    """The rank whose share(total, world, rank) holds item j."""
    for r in range(world):
        lo, hi = share(total, world, r)
        if lo <= j < hi:
            return r
    raise ValueError("item outside the range")


class Comm:
    """Collectives of one process group (torch.distributed), or none for one rank."""

    def __init__(self, group=None):
        import torch.distributed as dist
        self.dist = dist if dist.is_available() and dist.is_initialized() else None
        self.group = group
        self.world = self.dist.get_world_size(group) if self.dist else 1
        self.rank = self.dist.get_rank(group) if self.dist else 0

    def all_reduce_sum(self, x):
        if self.world > 1:
            self.dist.all_reduce(x, op=self.dist.ReduceOp.SUM, group=self.group)
        return x

    def all_gather(self, x):
        if self.world == 1:
            return [x]
        out = [torch.empty_like(x) for _ in range(self.world)]
        self.dist.all_gather(out, x, group=self.group)
        return out

    def broadcast(self, x, src):
        if self.world > 1:
            self.dist.broadcast(x, src=self.dist.get_global_rank(self.group, src) if self.group else src,
                                group=self.group)
        return x


class ColumnSplit:
    """The exchange protocol of the column-split greedy over one shard per rank.

    A shard holds this rank's columns and offers: bank(), caches() -> (h, t), live_count(),
    shortlist(Br), solve_rerank(b0, b1) -> re-rank scores of shortlist positions [b0, b1),
    winner_column(j) / empty_column() -> the p x nA solve column of position j,
    take_winner(j, u, owned, score) -> candidate index, maintain_delta() -> (dh, dt),
    apply_cache(dh, dt), finish(e), and the attributes k, B, naive.  Every method that
    returns tensors returns them on the device the process group's backend expects."""

    def __init__(self, shard, comm):
        if shard.naive:
            raise ValueError("the column split runs the cached greedy (naive=False)")
        self.shard, self.comm = shard, comm
        self.rnd = 0
        self.banked = False

    def bank(self):
        self.shard.bank()
        h, t = self.shard.caches()
        self.comm.all_reduce_sum(h)
        self.comm.all_reduce_sum(t)
        self.banked = True

    def step(self):
        """One round; returns the winner's candidate index (the same on every rank)."""
        sh, comm = self.shard, self.comm
        if not self.banked:
            self.bank()
        if self.rnd >= sh.k:
            raise RuntimeError("all k rounds have run")
        Br = min(sh.B, sh.live_count())
        sh.shortlist(Br)
        world, rank = comm.world, comm.rank
        b0, b1 = share(Br, world, rank)
        g = sh.solve_rerank(b0, b1)
        width = -(-Br // world)
        buf = torch.full((width,), -float("inf"), dtype=torch.float64, device=g.device)
        buf[:b1 - b0] = g
        parts = comm.all_gather(buf)
        gq = np.concatenate([parts[r][:share(Br, world, r)[1] - share(Br, world, r)[0]].cpu().numpy()
                             for r in range(world)])
        j = int(np.argmax(gq))
        owner = owner_of(j, Br, world)
        u = sh.winner_column(j) if owner == rank else sh.empty_column()
        comm.broadcast(u, owner)
        e = sh.take_winner(j, u, owner == rank, float(gq[j]))
        if self.rnd + 1 < sh.k:
            dh, dt = sh.maintain_delta()
            comm.all_reduce_sum(dh)
            comm.all_reduce_sum(dt)
            sh.apply_cache(dh, dt)
        sh.finish(e)
        self.rnd += 1
        return e


class DeviceShard(Greedy):
    """This rank's share of a greedy run on its GPU: a Greedy over the sketch columns
    [c0, c1) (its own X / Y bank columns, F and Gc columns), which solves the shortlist
    positions the protocol hands it and maintains its columns with the split kernels."""

    def __init__(self, G, cand, k, s, sketch, c0, c1, **kw):
        Z, F, Gc = sketch
        if not 0 <= c0 < c1 <= Z.shape[1]:
            raise ValueError("each rank needs at least one sketch column")
        cut = (lambda a: a[:, c0:c1]) if isinstance(Z, torch.Tensor) else (lambda a: np.ascontiguousarray(a[:, c0:c1]))
        super().__init__(G, cand, k, s, q=c1 - c0, sketch=(cut(Z), cut(F), cut(Gc)), **kw)
        p, N = self.p, self.N
        self.dh = torch.empty((p, N), dtype=torch.float64, device=self.dev)
        self.dt = torch.empty((p, N), dtype=torch.float64, device=self.dev)
        self.esz = 4 if self.x_f32 else 8

    def caches(self):
        return self.h, self.t

    def live_count(self):
        return int(self.live_h.sum())

    def shortlist(self, Br):
        _lib.check(self.lib.polar_score_topb(self.h.data_ptr(), self.t.data_ptr(), self.tau_d.data_ptr(),
                                             self.om_d.data_ptr(), self.G.sigma, self.p, self.N,
                                             self.live_d.data_ptr(), _OBJ[self.obj], Br, self.short_d.data_ptr(),
                                             self.sscore_d.data_ptr(), None, self.topb_tmp.data_ptr(), self.stream),
                   "score_topb")

    def solve_rerank(self, b0, b1):
        nb = b1 - b0
        if nb <= 0:
            return torch.empty(0, dtype=torch.float64, device=self.dev)
        lib, st = self.lib, self.stream
        _lib.check(lib.polar_fill_incidence(self.n, nb, self.cand_d.data_ptr(), self.short_d.data_ptr() + 8 * b0,
                                            self.es_d.data_ptr(), self.Wb.data_ptr(), self.Bmax, self.ia_d.data_ptr(),
                                            self.ib_d.data_ptr(), st), "fill_incidence")
        inf = []
        _, hh, _ = msolve(self.op, self.Wb[:, :nb], self.tau_d, self.act_d, self.tol, maxit=self.maxit,
                          track=(self.obj != "logdet"), counter=self.cnt, precision=self.prec, out=self.U,
                          out_col=b0, active_pos=self.pos_d, info=inf)
        self.solves.extend((nb, int(i.iterations)) for i in inf)
        _lib.check(lib.polar_rerank(self.U.data_ptr() + self.esz * b0, self.x_f32, self.p, self.nA, self.Bmax,
                                    self.ia_d.data_ptr(), self.ib_d.data_ptr(), nb,
                                    hh.data_ptr() if hh is not None else None, self.om_d.data_ptr(), _OBJ[self.obj],
                                    self.gq_d.data_ptr(), self.best_d.data_ptr(), st), "rerank")
        return self.gq_d[:nb].clone()

    def winner_column(self, j):
        return self.U[:, :, j].contiguous()

    def empty_column(self):
        return torch.empty((self.p, self.nA), dtype=self.U.dtype, device=self.dev)

    def take_winner(self, j, u, owned, score):
        if not owned:
            self.U[:, :, j].copy_(u)
        self.best_d.fill_(j)
        _lib.check(self.lib.polar_select(self.short_d.data_ptr(), self.best_d.data_ptr(), self.es_d.data_ptr(),
                                         self.live_d.data_ptr(), self.win_d.data_ptr(), self.stream), "select")
        win = self.win_d.cpu().numpy()
        e = int(win[4:6].view(np.int64)[0])
        self.seq.append(e)
        self.marg.append(score)
        self.live_h[e] = False
        return e

    def maintain_delta(self):
        q, XY = self.q, self.XY
        _lib.check(self.lib.polar_maintain_split(XY.data_ptr(), 2 * q, XY[:, :, q:].data_ptr(), 2 * q, self.x_f32,
                                                 self.p, self.nA, q, self.U.data_ptr(), self.x_f32, self.Bmax,
                                                 self.win_d.data_ptr(), self.Gd.data_ptr(), self.es_d.data_ptr(),
                                                 self.N, self.dh.data_ptr(), self.dt.data_ptr(),
                                                 self.mtmp.data_ptr(), self.stream), "maintain_split")
        return self.dh, self.dt

    def apply_cache(self, dh, dt):
        _lib.check(self.lib.polar_cache_apply(self.h.data_ptr(), dh.data_ptr(), self.t.data_ptr(), dt.data_ptr(),
                                              self.p * self.N, self.stream), "cache_apply")

    def finish(self, e):
        q = self.q
        _lib.check(self.lib.polar_rank1_rows(self.RHS[:, q:].data_ptr(), 2 * q, q, self.Gd.data_ptr(),
                                             self.cand_d.data_ptr(), self.win_d[4:].data_ptr(), self.stream),
                   "rank1_rows")
        self.op.add(int(self.cand[e, 0]), int(self.cand[e, 1]))
        self.rnd += 1


def polar_split(G, cand, k, s, q=128, B=16, eps=1e-2, tol=1e-7, obj="frac", sketch=None, seed=2026, kind="block",
                *, K=None, precision="fp64", group=None, maxit=100000):
    """polar() with the bank's sketch columns and each round's shortlist columns split over
    the ranks of `group` (the default process group when None; one rank when
    torch.distributed is not initialised).  Every rank passes the same arguments and gets
    the same sequence; marginals are the winners' re-rank scores as in polar()."""
    comm = Comm(group)
    if sketch is None:
        sketch = sketches(G, cand, q, seed, kind)
    qq = int(sketch[0].shape[1])
    if comm.world > qq:
        raise ValueError("more ranks than sketch columns")
    c0, c1 = share(qq, comm.world, comm.rank)
    shard = DeviceShard(G, cand, k, s, sketch, c0, c1, B=B, eps=eps, tol=tol, obj=obj, K=K, precision=precision,
                        maxit=maxit)
    run = ColumnSplit(shard, comm)
    run.bank()
    for _ in range(shard.k):
        run.step()
    out = shard.result()
    out["ranks"] = comm.world
    out["columns"] = (c0, c1)
    return out
