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
    ap.add_argument("--no-autotune", action="store_true", help="keep the solver's default SpMM layouts")
    ap.add_argument("--quick", action="store_true", help="full-n4M: one short solve (an ncu-sized case)")
    ap.add_argument("--cache", default=None, help="full-n4M: .npz file holding the generated edge list "
                                                    "(written when absent, read when present)")
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
    tuned = {}
    if not a.no_autotune:
        # SpMM layout per solve width (shortlist B, bank 2q), timed once before any greedy
        from polar_b200 import autotune
        for prec, wide in (("mixed", 128),) + ((("fp64", 64),) if not a.no_fp64 else ()):
            for R in sorted({c["B"], min(2 * c["q"], wide)}):
                t = autotune.tune_msolve(pg.Op(G), R, prec, p=c["K"])
                tuned[f"{prec}_R{R}"] = {"lane_bytes": t["best"][0], "sliced_ell": t["best"][1],
                                         "heavy_thresh": t["best"][2], "us_per_iter": t["us_per_iter"],
                                         "layouts_timed": len(t["table"])}

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
            "dtype": "f32 SpMM input/output and pole iterates; f64 residual, direction and scalars",
            "data": "synthetic (seeded Chung-Lu stand-in for com-DBLP shape)",
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
            "iteration_alg_GBps": (sum(v[2] for v in ktime.values()) / (ktot / 1e3) / 1e9) if ktot else None,
            "parity": parity,
            "sequence_head": mixed["sequence"][:8],
            "spmv": mixed["spmv"], "p": mixed["p"],
            "cg": {"seed_iterations": int(sum(it for _, it in mixed["solves"])), "column_iterations": mixed["spmv"],
                   "seed_iterations_per_s": sum(it for _, it in mixed["solves"]) / per,
                   "column_iterations_per_s": mixed["spmv"] / per},
            "clocks": clk.summary(),
            "cpu_baseline": cpu,
            "autotune": tuned or None,
        }
        if a.phases:
            line["phases"] = mixed.get("phases")
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


def run_batch(a):
    """Many-graphs workload: the bank solves of 48 graphs (2q right-hand sides each, K poles
    from each graph's own s and sigma) in one polar_msolve_batch launch, against the same
    solves one graph at a time through msolve."""
    import torch

    import polar_b200 as pg
    from polar_b200 import _lib
    from polar_b200.batch import msolve_batch
    from polar_b200.synth import CONFIGS, batch_specs, candidates, chung_lu
    torch.cuda.set_device(0)
    dev = torch.device("cuda", 0)
    lib = _lib.load()
    c = CONFIGS["batch48"]
    specs = batch_specs(c["graphs"])
    R = 2 * c["q"]
    t_gen = time.perf_counter()
    ops, Ws, taus, acts, Wh, meta = [], [], [], [], [], []
    gen = torch.Generator(device=dev)
    gen.manual_seed(2026)
    for sp in specs:
        n = min(sp["n"], a.n) if a.n else sp["n"]
        E = chung_lu(n, sp["mean_deg"], sp["gamma"], sp["seed"], min_degree=1)
        cand = candidates(n, E, min(c["N"], n), sp["seed"] + 7919)
        G = pg.Graph(n, E, sp["sigma"])
        tau, _, _ = pg.poles("frac", sp["s"], sp["sigma"], G.Lam(c["k"]), 1e-2, K=c["K"])
        W = torch.randn((n, R), generator=gen, device=dev, dtype=torch.float64) / np.sqrt(c["q"])
        ops.append(pg.Op(G))
        Ws.append(W)
        taus.append(tau)
        acts.append(np.unique(cand))
        meta.append((n, G.nnz))
    t_gen = time.perf_counter() - t_gen
    kw = dict(precision="mixed")

    def batch_once(W_list):
        return msolve_batch(ops, W_list, taus, acts, c["tol"], **kw)

    for _ in range(a.warmup):
        res = batch_once(Ws)
    torch.cuda.synchronize()
    launches0 = lib.polar_launch_count()
    with Clocks(0) as clk:
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(a.steps):
            res = batch_once(Ws)
        e1.record()
        torch.cuda.synchronize()
    launches = lib.polar_launch_count() - launches0
    per = e0.elapsed_time(e1) / 1e3 / a.steps
    iters = [int(it.max()) for _, _, it in res]
    colit = sum(int(it.sum()) for _, _, it in res)
    # the same solves one graph at a time (kernel-per-phase driver, CUDA-graph blocks)
    torch.cuda.synchronize()
    s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s0.record()
    seq = [pg.msolve(ops[g], Ws[g], taus[g], acts[g], c["tol"], **kw) for g in range(len(ops))]
    s1.record()
    torch.cuda.synchronize()
    seq_s = s0.elapsed_time(s1) / 1e3
    err = max(float((X.double() - Xs.double()).abs().max() / Xs.double().abs().max().clamp_min(1e-300))
              for (X, _, _), (Xs, _, _) in zip(res, seq))
    # end to end: host right-hand sides in, host solutions out
    Wh = [W.cpu().numpy() for W in Ws]
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    out = batch_once(Wh)
    Xh = [X.cpu() for X, _, _ in out]
    e2e_s = time.perf_counter() - t0
    h2d = sum(W.nbytes for W in Wh)
    d2h = sum(X.numel() * X.element_size() for X in Xh)
    # bytes moved by the SpMM and vector phases, per seed iteration (algorithmic, FP32)
    alg = sum(it * (4.0 * (n + 1) + 4.0 * nnz + 2 * 4.0 * n * R + 6 * 4.0 * n * R)
              for it, (n, nnz) in zip(iters, meta))
    line = {
        "metric": "batched bank solves of 48 graphs (mixed precision)", "value": per, "unit": "s/batch",
        "n_gpus": 1, "steps": a.steps, "warmup": a.warmup, "ms_per_step": per * 1e3, "higher_is_better": False,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32 SpMM input/output and pole iterates; f64 residual, direction and scalars",
        "data": "synthetic (48 seeded Chung-Lu graphs, Gaussian right-hand sides)",
        "config": {"workload": "batch48", "graphs": len(ops), "n_total": int(sum(m[0] for m in meta)),
                   "nnz_total": int(sum(m[1] for m in meta)), "K": c["K"], "R": R, "N_per_graph": c["N"],
                   "tol": c["tol"], "l2": "inputs larger than L2 (block vectors of all graphs: %.1f GB)"
                   % (sum(m[0] for m in meta) * R * 4 * 3 / 1e9)},
        "sequential_s": seq_s, "batch_speedup_vs_sequential": seq_s / per,
        "max_rel_diff_vs_sequential": err, "seed_iterations": {"max": max(iters), "sum": sum(iters)},
        "column_iterations_per_s": colit / per, "alg_GBps": alg / per / 1e9,
        "e2e": {"value": e2e_s, "unit": "s/batch", "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h)},
        "gpu_launches": int(launches), "clocks": clk.summary(), "host_setup_s": t_gen,
    }
    print(json.dumps(line), flush=True)


def run_full(a):
    """Full-scale solve: the shortlist solve of the n = 4.0M / 34.7M-edge workload (B = 16
    incidence columns, K = 32 poles, tol 1e-6, pole iterates on ~1.57M active rows) in FP64
    and in mixed precision, with the per-kernel table of each; plus the SpMM alone at 16 and
    64 columns.  `--quick` runs only a 48-iteration mixed solve over 32 active rows (the
    small case for an ncu capture of the SpMM)."""
    import torch

    import polar_b200 as pg
    from polar_b200 import _lib
    from polar_b200.synth import CONFIGS, candidates, chung_lu
    torch.cuda.set_device(0)
    dev = torch.device("cuda", 0)
    lib = _lib.load()
    c = CONFIGS["full-n4M"]
    n = a.n or c["n"]
    t_gen = time.perf_counter()
    if a.cache and os.path.exists(a.cache):
        E = np.load(a.cache)["edges"].astype(np.int64)
    else:
        E = chung_lu(n, c["mean_deg"], c["gamma"], c["seed"], dmax=c["dmax"] if n == c["n"] else None,
                     min_degree=c["min_degree"])
        if a.cache:
            np.savez(a.cache, edges=E.astype(np.int32))
    pairs = candidates(n, E, c["B"], c["seed"] + 7919)
    rng = np.random.default_rng(c["seed"])
    # endpoints of N uniform candidate pairs: the active rows of the workload's pole iterates
    Nq = 16 if a.quick else c["N"]
    active = np.unique(np.concatenate([rng.integers(0, n, 2 * Nq), pairs.ravel()]))
    G = pg.Graph(n, E, c["sigma"])
    t_gen = time.perf_counter() - t_gen
    op = pg.Op(G)
    tau, om, _ = pg.poles("frac", c["s"], c["sigma"], G.Lam(c["k"]), 1e-2, K=c["K"])
    R = c["B"]
    W = np.zeros((n, R))
    W[pairs[:, 0], np.arange(R)] = 1.0
    W[pairs[:, 1], np.arange(R)] = -1.0
    Wd = torch.as_tensor(W).to(dev)
    from polar_b200 import solver as S
    act_d, pos_d = S.prepare_active(active, n, dev)
    ia = np.searchsorted(active, pairs[:, 0])
    ib = np.searchsorted(active, pairs[:, 1])

    def solve(prec, maxit=100000):
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        try:
            X, h, it = S.msolve(op, Wd, tau, act_d, c["tol"], maxit=maxit, track=True, precision=prec,
                                active_pos=pos_d)
        except _lib.PolarError as e:
            if e.status != _lib.POLAR_ERR_ITER_CAP or maxit == 100000:
                raise
            return None
        e1.record()
        torch.cuda.synchronize()
        cols = torch.arange(R, device=dev)
        bu = (X[:, torch.as_tensor(ia, device=dev), cols].double()
              - X[:, torch.as_tensor(ib, device=dev), cols].double()).cpu().numpy()
        G_q = (om[:, None] * h.cpu().numpy() / (1.0 + bu)).sum(0)
        return {"seconds": e0.elapsed_time(e1) / 1e3, "iterations": int(it.max()), "G": G_q}

    if a.quick:
        lib.polar_set_kernel_timing(1)
        solve("mixed", maxit=48)
        kt = _lib.kernel_timing()
        lib.polar_set_kernel_timing(0)
        print(json.dumps({"workload": "full-n4M", "quick": True, "n": n, "nnz": G.nnz,
                          "spmm_ms_per_launch": kt["spmm"][1] / max(1, kt["spmm"][0])}), flush=True)
        return
    out = {}
    for prec in ("fp64", "mixed"):
        solve(prec, maxit=16)  # warm-up: graph partitions, workspace, CUDA graphs
        res = solve(prec)
        lib.polar_set_kernel_timing(1)
        inst = solve(prec)
        kt = _lib.kernel_timing()
        lib.polar_set_kernel_timing(0)
        out[prec] = dict(res, kernels={k: {"launches": v[0], "ms": v[1],
                                           "alg_GBps": v[2] / (v[1] / 1e3) / 1e9 if v[1] > 0 else None}
                                       for k, v in kt.items() if v[0]},
                         instrumented_seconds=inst["seconds"])
    G64, G32 = out["fp64"].pop("G"), out["mixed"].pop("G")
    # the SpMM alone (polar_spmm through Op), 16 and 64 columns, both precisions
    hbm, peak_kind = peak_hbm()
    spmm = {}
    for dt, nm in ((torch.float64, "fp64"), (torch.float32, "mixed")):
        for Rc in (16, 64):
            Xs = torch.randn((n, Rc), device=dev, dtype=torch.float64).to(dt)
            op(Xs, 0.0)
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            reps = 10
            e0.record()
            for _ in range(reps):
                op(Xs, 0.0)
            e1.record()
            torch.cuda.synchronize()
            ms = e0.elapsed_time(e1) / reps
            el = 8 if dt == torch.float64 else 4
            alg = 4.0 * (n + 1) + 4.0 * G.nnz + 2.0 * el * n * Rc
            spmm[f"{nm}_R{Rc}"] = {"ms": ms, "alg_GBps": alg / (ms / 1e3) / 1e9,
                                   "frac_of_peak": alg / (ms / 1e3) / 1e9 / hbm}
            del Xs
    line = {"metric": "full-scale shortlist solve (B = 16 columns, K = 32 poles)", "unit": "s/solve",
            "value": out["mixed"]["seconds"], "higher_is_better": False, "n_gpus": 1,
            "config": {"workload": "full-n4M", "n": n, "m": int(len(E)), "nnz": G.nnz, "dmax": G.dmax,
                       "nA": int(len(active)), "K": c["K"], "R": R, "tol": c["tol"], "sigma": c["sigma"], "s": c["s"]},
            "fp64": out["fp64"], "mixed": out["mixed"],
            "mixed_speedup_vs_fp64": out["fp64"]["seconds"] / out["mixed"]["seconds"],
            "max_rel_marginal_err": float(np.max(np.abs(G32 - G64) / np.abs(G64))),
            "spmm_alone": spmm, "peak_GBps": hbm, "peak_source": peak_kind, "host_setup_s": t_gen}
    print(json.dumps(line), flush=True)


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
    if args.impl == "reference" and args.config in ("batch48", "full-n4M"):
        why = {"batch48": "the many-graphs workload has no reference arm: the reference solves one graph per call",
               "full-n4M": "the full-scale solve has no reference arm here: the oracle's FP64 NumPy solve of a "
                           "4M-vertex graph takes hours on the host cores"}[args.config]
        print(json.dumps({"impl": "reference", "unavailable": why}), flush=True)
    elif args.impl == "reference":
        run_reference(args)
    elif args.config == "batch48":
        run_batch(args)
    elif args.config == "full-n4M":
        run_full(args)
    else:
        run_ours(args)
