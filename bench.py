"""POLAR solve-and-score benchmark on B200.

Workload (precision config): Chung–Lu n=317,080 (~1.05M edges, exponent 2.4, seed 1),
sigma=1e-2, s=0.5, K=24 poles, q=64 sketch columns, N=200,000 candidate non-edges, B=16,
k=50 rounds, CG tol 1e-7.  The seeded synthetic graph stands in for com-DBLP (same n and
m; the SNAP file is not available here).

One step = one complete k-round greedy POLAR run (bank solve, then per round: proxy score
+ top-B, B-column shortlist solve, re-rank, maintenance).  `value` = mixed-precision
greedy time (device events; inputs resident).  The FP64 path runs once beside it for
parity (same sequence, max relative marginal error).  `e2e` times the public API
(polar_b200.Graph + polar_b200.polar) from host arrays, uploads included.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

Multi-GPU: the greedy does not shard (one graph per greedy); N GPUs run N independent
replicas on graphs of different seeds, with no collective on the data path; value is
the mean greedy time of the replicas (max over ranks of the device time / K).
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "k-round greedy time (mixed precision, FP64 parity)"
UNIT = "s/greedy"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="precision-n317k")
    ap.add_argument("--n", type=int, default=None, help="shrink the graph (debug)")
    ap.add_argument("--N", type=int, default=None)
    ap.add_argument("--k", type=int, default=None)
    ap.add_argument("--no-fp64", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--cpu-iters", type=int, default=1, help="oracle CG iterations timed per width")
    ap.add_argument("--phases", action="store_true")
    return ap.parse_args()


# ---------------------------------------------------------------------------------------
class Clocks:
    """nvidia-smi sampling of SM clocks and throttle reasons during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            threading.Thread(target=self._read, daemon=True).start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [x.strip() for x in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def peak_hbm():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def profiled_traffic(config):
    """DRAM bytes per SpMM launch from the committed ncu summary (null when absent)."""
    p = os.path.join(ROOT, "profiles", "roofline_traffic.json")
    if not os.path.exists(p):
        return None
    with open(p) as f:
        d = json.load(f)
    return d.get(config, {}).get("spmm_dram_bytes_per_launch")


# ---------------------------------------------------------------------------------------
def replica_seed(base_seed, rank):
    """Seed of rank `rank`'s replica graph: replicas run independent greedies."""
    return base_seed + 1000 * rank


def job_seconds(local_s, world, device):
    """Device time of the whole job: the maximum over ranks (all ranks call this in the
    same order; a no-op at one rank)."""
    if world <= 1:
        return local_s
    import torch
    import torch.distributed as dist
    t = torch.tensor([local_s], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    dist.barrier()
    return float(t.item())


def build_inputs(a, rank=0):
    from polar_b200.synth import CONFIGS, candidates, chung_lu
    c = dict(CONFIGS[a.config])
    n = a.n or c["n"]
    N = a.N or c["N"]
    k = a.k or c["k"]
    seed = replica_seed(c["seed"], rank)
    E = chung_lu(n, c["mean_deg"], c["gamma"], seed, dmax=c["dmax"] if n == c["n"] else None,
                 min_degree=c.get("min_degree", 0))
    cand = candidates(n, E, N, seed + 7919)
    return dict(n=n, N=N, k=k, E=E, cand=cand, cfg=c, seed=seed)


def oracle_iteration_costs(inp, sk, tau, active_h, widths, iters):
    """Seconds per multi-shift CG iteration of the oracle (NumPy FP64, the host's BLAS
    threads) at each column width, from `iters` timed iterations."""
    from oracle import polar_oracle as O
    c = inp["cfg"]
    op = O.Op(O.Graph(inp["n"], inp["E"], c["sigma"]))
    out = {}
    rhs = np.concatenate([sk[0], sk[1]], axis=1)
    for w in widths:
        W = rhs[:, :w] if w <= rhs.shape[1] else np.tile(rhs, (1, -(-w // rhs.shape[1])))[:, :w]
        t0 = time.perf_counter()
        try:
            O.msolve(op, W, tau, active_h, 1e-30, maxit=iters)
        except RuntimeError:
            pass
        out[w] = (time.perf_counter() - t0) / iters
    return out


def cpu_estimate(costs, solves, oracle_width=64):
    """Greedy seconds of the oracle for these solves: the oracle runs the bank in chunks
    of `oracle_width` columns (realworld/polar_gpu.py:169-173) and one shortlist solve per
    round; per-iteration cost is interpolated linearly in the column count."""
    ws = sorted(costs)
    t_at = lambda R: float(np.interp(R, ws, [costs[w] for w in ws]))
    total = 0.0
    for R, it in solves:
        if R > oracle_width:
            total += (R // oracle_width) * t_at(oracle_width) * it
        else:
            total += t_at(R) * it
    return total


def run_ours(a):
    import torch
    import torch.distributed as dist

    import polar_b200 as pg
    from polar_b200 import _lib

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=900), device_id=dev)
    lib = _lib.load()
    inp = build_inputs(a, rank)
    n, N, k, E, cand, c = inp["n"], inp["N"], inp["k"], inp["E"], inp["cand"], inp["cfg"]
    G = pg.Graph(n, E, c["sigma"])
    sk = pg.sketches(G, cand, c["q"], 2026)
    kw = dict(q=c["q"], B=c["B"], tol=c["tol"], sketch=sk, K=c["K"])

    def timed_run(prec, **extra):
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        res = pg.polar(G, cand, k, c["s"], precision=prec, **kw, **extra)
        e1.record()
        torch.cuda.synchronize()
        res["device_s"] = e0.elapsed_time(e1) / 1e3
        return res

    fp64 = None if a.no_fp64 else timed_run("fp64")
    for _ in range(a.warmup):
        mixed = timed_run("mixed")

    # ---- timed region: exactly K greedy runs, uninstrumented ----
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    launches0 = lib.polar_launch_count()
    with Clocks(local) as clk:
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record()
        runs = [pg.polar(G, cand, k, c["s"], precision="mixed", phases=a.phases, **kw) for _ in range(a.steps)]
        ev1.record()
        torch.cuda.synchronize()
    launches = lib.polar_launch_count() - launches0
    total_s = job_seconds(ev0.elapsed_time(ev1) / 1e3, world, dev)
    # ---- one more greedy with every solver kernel bracketed by CUDA events (the event
    # nodes serialise the iteration graph, so this run is not part of `value`) ----
    torch.cuda.synchronize()
    lib.polar_set_kernel_timing(1)
    inst = timed_run("mixed")
    ktime = _lib.kernel_timing()
    lib.polar_set_kernel_timing(0)
    per = total_s / a.steps
    mixed = runs[-1]

    # ---- roofline of the dominant kernel (the SpMM of the multi-shift CG: heavy-row and
    # light-row launches together; algorithmic bytes are counted on the light class) ----
    hbm, peak_kind = peak_hbm()
    nl, ms_l, by = ktime["spmm"]
    ms = ms_l + ktime["spmm_heavy"][1]
    achieved = by / (ms / 1e3) / 1e9 if ms > 0 else None
    kernels = {name: {"launches": v[0], "ms": v[1], "share": None,
                      "alg_GBps": (v[2] / (v[1] / 1e3) / 1e9) if v[1] > 0 else None}
               for name, v in ktime.items()}
    ktot = sum(v[1] for v in ktime.values())
    for name in kernels:
        kernels[name]["share"] = ktime[name][1] / ktot if ktot else None

    # ---- end to end through the public API, from host arrays ----
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    G2 = pg.Graph(n, E, c["sigma"])
    res_e2e = pg.polar(G2, cand, k, c["s"], precision="mixed", **kw)
    _ = list(res_e2e["sequence"])
    torch.cuda.synchronize()
    e2e_s = time.perf_counter() - t0
    h2d = E.nbytes + cand.nbytes + sum(np.asarray(x).nbytes for x in sk)
    d2h = 8 * 6 * k + 8 * 2 * k

    parity = {}
    if fp64 is not None:
        mf = np.asarray(fp64["marginals"])
        mm = np.asarray(mixed["marginals"])
        same = fp64["sequence"] == mixed["sequence"]
        upto = len(mf) if same else next(i for i, (x, y) in enumerate(zip(fp64["sequence"], mixed["sequence"]))
                                         if x != y)
        parity = {"same_sequence": same, "rounds_compared": upto,
                  "max_rel_marginal_err": float(np.max(np.abs(mm[:upto] - mf[:upto]) / np.abs(mf[:upto])))
                  if upto else None,
                  "fp64_greedy_s": fp64["device_s"], "mixed_speedup_vs_fp64": fp64["device_s"] / per}

    cpu = None
    if rank == 0 and world == 1 and not a.no_cpu:
        tau, _, _ = pg.poles("frac", c["s"], c["sigma"], G.Lam(k), 1e-2, K=c["K"])
        costs = oracle_iteration_costs(inp, sk, tau, np.unique(cand), (64, c["B"]), a.cpu_iters)
        est = cpu_estimate(costs, mixed["solves"])
        cpu = {"value": est, "unit": UNIT, "cores": os.cpu_count(), "kind": "port",
               "sample": (f"oracle (NumPy FP64 restatement of polar_gpu.py) multi-shift CG timed for "
                          f"{a.cpu_iters} iteration(s) at 64 and {c['B']} columns "
                          f"({costs[64]:.2f} / {costs[c['B']]:.2f} s per iteration, BLAS on all host threads, "
                          f"SciPy SpMM on 1 core), times this greedy's seed iterations per solve "
                          f"({sum(it for _, it in mixed['solves'])} iterations over {len(mixed['solves'])} solves)")}

    if rank == 0:
        line = {
            "metric": METRIC, "value": per, "unit": UNIT, "n_gpus": world, "steps": a.steps, "warmup": a.warmup,
            "ms_per_step": per * 1e3, "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32 vectors, f64 scalars", "data": "synthetic (seeded Chung-Lu stand-in for com-DBLP shape)",
            "config": {"workload": a.config, "n": n, "m": int(len(E)), "N": N, "K": c["K"], "q": c["q"],
                       "B": c["B"], "k": k, "s": c["s"], "sigma": c["sigma"], "tol": c["tol"],
                       "l2": "inputs larger than L2 (X/Y banks 2.8 GB, SpMM block 162 MB)",
                       "parallelism": f"replicas x{world}"},
            "e2e": {"value": e2e_s, "unit": UNIT, "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h)},
            "gpu_launches": int(launches),
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                         "frac": achieved / hbm if achieved else None,
                         "traffic": profiled_traffic(a.config),
                         "kernel": "mk_spmm (CSR SpMM + d.v of the multi-shift CG, heavy + light launches)",
                         "peak_source": peak_kind, "launches": nl, "avg_launch_us": ms * 1e3 / nl if nl else None,
                         "measured": "CUDA events around every solver kernel in one instrumented greedy run "
                                     "right after the timed region (%.3f s with events)" % inst["device_s"]},
            "kernels": kernels,
            "parity": parity,
            "sequence_head": mixed["sequence"][:8],
            "spmv": mixed["spmv"], "p": mixed["p"],
            "clocks": clk.summary(),
            "cpu_baseline": cpu,
        }
        if a.phases:
            line["phases"] = mixed.get("phases")
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


def run_reference(a):
    """The reference's algorithm on the host: the oracle (a NumPy FP64 restatement of
    realworld/polar_gpu.py; the reference itself needs CuPy and a GPU).  Per-iteration
    cost is timed at the bank and shortlist widths; iteration counts come from seed-CG
    runs of a sample of bank columns and shortlist edges (SciPy, FP64)."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    import polar_b200.quadrature as Q
    from oracle import polar_oracle as O
    inp = build_inputs(a, 0)
    c = inp["cfg"]
    OG = O.Graph(inp["n"], inp["E"], c["sigma"])
    sk = O.sketches(OG, inp["cand"], c["q"], 2026)
    tau, _, _ = Q.poles("frac", c["s"], c["sigma"], OG.Lam(inp["k"]), 1e-2, K=c["K"])
    active_h = np.unique(inp["cand"])
    n = inp["n"]

    def seed_iters(w):
        A = OG.M0 + tau[0] * __import__("scipy.sparse", fromlist=["eye"]).eye(n, format="csr")
        r = w.copy()
        d = r.copy()
        rr = r @ r
        stop = c["tol"] * np.sqrt(rr)
        for it in range(100000):
            v = A @ d
            al = rr / (d @ v)
            r -= al * v
            rrn = r @ r
            if np.sqrt(rrn) <= stop:
                return it + 1
            d = r + (rrn / rr) * d
            rr = rrn
        return 100000

    vals = []
    for _ in range(max(1, a.steps)):
        t0 = time.perf_counter()
        costs = oracle_iteration_costs(inp, sk, tau, active_h, (64, c["B"]), a.cpu_iters)
        rhs = np.concatenate([sk[0], sk[1]], axis=1)
        bank_it = max(seed_iters(rhs[:, j].copy()) for j in (0, 1, c["q"], c["q"] + 1))
        short_it = []
        for e in range(2):
            w = np.zeros(n)
            w[inp["cand"][e, 0]] = 1.0
            w[inp["cand"][e, 1]] = -1.0
            short_it.append(seed_iters(w))
        solves = [(2 * c["q"], bank_it)] + [(c["B"], max(short_it))] * inp["k"]
        vals.append(cpu_estimate(costs, solves))
        sample_s = time.perf_counter() - t0
    v = float(np.mean(vals))
    cpu = {"value": v, "unit": UNIT, "cores": os.cpu_count(), "kind": "port",
           "sample": (f"oracle multi-shift CG: {a.cpu_iters} timed iteration(s) at 64 and {c['B']} columns "
                      f"({costs[64]:.2f} / {costs[c['B']]:.2f} s/iteration); iteration counts from seed CG on 4 "
                      f"bank columns ({bank_it}) and 2 shortlist edges ({max(short_it)}), x {inp['k']} rounds; "
                      f"{sample_s:.0f} s of host work per step")}
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": world, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": v * 1e3, "higher_is_better": False, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded Chung-Lu stand-in for com-DBLP shape)",
            "config": {"workload": a.config, "n": n, "m": int(len(inp["E"])), "N": inp["N"], "K": c["K"],
                       "q": c["q"], "B": c["B"], "k": inp["k"], "s": c["s"], "sigma": c["sigma"], "tol": c["tol"]},
            "cpu_baseline": cpu, "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


if __name__ == "__main__":
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)
