"""POLAR solve-and-score benchmark on B200.

Default workload (full-n4M): the full-scale greedy.  Chung–Lu n = 3,997,962 (34.7M edges,
exponent 2.1, expected degree capped at 15,000, min degree 1, seed 4), sigma = 1e-2,
s = 0.5, K = 32 poles, q = 64 sketch columns, N = 10^6 uniform non-edge candidates,
B = 16, k = 100 rounds, CG tol 1e-6.  The seeded synthetic graph stands in for
com-LiveJournal (same n and m; the SNAP file is not available here).

One step = one greedy round (realworld/polar_gpu.py:215-251): proxy scores of all N
candidates and the stable top-B shortlist, the B-column multi-shift solve over all K poles,
the re-rank, and the Sherman–Morrison maintenance of the 2q-column banks and h/t caches.
The bank solve (2q = 128 right-hand sides, once per greedy) runs before the warm-up rounds
and is timed separately; `greedy_s` = bank + k x value is the k-round greedy time.
`value` = mixed-precision seconds per round (CUDA events around the K timed rounds; inputs
resident in HBM).  The FP64 path runs the same rounds after it (`parity`: same sequence,
max relative marginal error, FP64 seconds per round and bank, mixed-over-FP64 speed-up).
`e2e` = polar_b200.Graph + polar_b200.Greedy from host arrays (edge list, candidates and
sketch arrays uploaded, bank, K rounds, winners read back), wall clock divided by K.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--config NAME] [--impl reference]
    python bench.py --config full-n4M --solve [--quick]   # one shortlist solve, kernel table
    python bench.py --config batch48                      # many graphs in one call

Multi-GPU: one greedy is one graph and does not shard here; N GPUs run N independent
replicas (sketch seeds 2026 + 1000 rank), no collective on the data path; value is the
mean round time of the replicas (max over ranks of the device time / K).
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

METRIC = "greedy round time, mixed precision (FP64 parity beside)"
UNIT = "s/round"
ITER_FILE = os.path.join(ROOT, "profiles", "iterations_per_round.json")


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="full-n4M")
    ap.add_argument("--n", type=int, default=None, help="shrink the graph (debug)")
    ap.add_argument("--N", type=int, default=None)
    ap.add_argument("--k", type=int, default=None)
    ap.add_argument("--no-fp64", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--cpu-iters", type=int, default=2, help="oracle CG iterations timed for the CPU baseline")
    ap.add_argument("--autotune", default="auto", choices=["auto", "on", "off"],
                    help="SpMM layout tuning of the shortlist width (auto: graphs under 2M vertices)")
    ap.add_argument("--l2", default=None, help="L2 policy MODE:MB for the solver (polar_set_l2_policy)")
    ap.add_argument("--residual", type=int, default=None, choices=[32, 64],
                    help="residual storage of the mixed-precision solve (polar_set_mixed_residual)")
    ap.add_argument("--solve", action="store_true", help="one shortlist solve with its kernel table")
    ap.add_argument("--quick", action="store_true", help="--solve: 48-iteration solves (an ncu-sized case)")
    ap.add_argument("--cache", default=None, help="directory for generated workloads (.npz, reused when present)")
    ap.add_argument("--dense-only", action="store_true", help="diff-n1.13M: only the dense subgraph checks")
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
    """DRAM bytes per shortlist-solve SpMM launch from the committed ncu summary (null when
    absent)."""
    p = os.path.join(ROOT, "profiles", "roofline_traffic.json")
    if not os.path.exists(p):
        return None
    with open(p) as f:
        d = json.load(f)
    return d.get(config, {}).get("spmm_dram_bytes_per_launch")


# ---------------------------------------------------------------------------------------
def replica_seed(base_seed, rank):
    """Sketch seed of rank `rank`'s replica: replicas run independent greedies."""
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


def build_inputs(a):
    """(n, N, k, edges, candidates, config) of the workload, generated from its seeds (or
    read from --cache, where a previous run left them)."""
    from polar_b200.synth import CONFIGS, make_config
    c = dict(CONFIGS[a.config])
    k = a.k or c["k"]
    E, n, cand, c = make_config(a.config, n=a.n, N=a.N, cache=a.cache)
    return dict(n=n, N=len(cand), k=k, E=E, cand=cand, cfg=c)


# ---------------------------------------------------------------------------------------
# CPU side: the reference's algorithm on the host cores, through the oracle (a NumPy FP64
# restatement of realworld/polar_gpu.py).  A round of the full-scale workload takes hours
# there, so a bounded sample is timed for real and scaled by the round's iteration count:
#   s/round = (s per multi-shift CG iteration at B columns) x (seed iterations per round)
#           + (proxy scores and stable top-B over N) + (Sherman–Morrison maintenance)
def host_threads():
    """Host threads this process may run on (the CPU legs use all of them)."""
    try:
        return max(1, len(os.sched_getaffinity(0)))
    except AttributeError:
        return max(1, os.cpu_count() or 1)


def oracle_round_parts(inp, iters, warm=1, on_sample=None, threads=1):
    """Times `iters` multi-shift CG iterations of the oracle on a B-column shortlist solve
    of the workload (full graph, all K poles, all active rows; right-hand sides = the
    incidence vectors of B candidate edges), plus the per-round scoring and maintenance.
    threads: host threads for the oracle's sparse product and shifted updates (the rest of
    an iteration, vector work on n x B blocks, stays on one thread).
    Returns dict(iteration_s list, score_s, maintain_s, sample_s)."""
    import polar_b200.quadrature as Q
    from oracle import polar_oracle as O
    t_all = time.perf_counter()
    c = inp["cfg"]
    n, cand = inp["n"], inp["cand"]
    OG = O.Graph(n, inp["E"], c["sigma"])
    tau, om, _ = Q.poles("frac", c["s"], c["sigma"], OG.Lam(inp["k"]), 1e-2, K=c["K"])
    active = np.unique(cand)
    B = c["B"]
    W = np.zeros((n, B))
    W[cand[:B, 0], np.arange(B)] = 1.0
    W[cand[:B, 1], np.arange(B)] = -1.0
    times = []
    last = [time.perf_counter()]

    def tick(it):
        now = time.perf_counter()
        times.append(now - last[0])
        last[0] = now
        if on_sample is not None and len(times) > warm:
            on_sample(len(times) - warm - 1, times[-1])

    try:
        O.msolve(O.Op(OG, threads=threads), W, tau, active, 1e-300, maxit=iters + warm, on_iteration=tick,
                 threads=threads)
    except RuntimeError:
        pass  # the iteration cap ends the sample
    # scoring over all N candidates and the stable top-B (polar_gpu.py:219-221)
    p, N = len(tau), len(cand)
    rng = np.random.default_rng(0)
    h = rng.random((p, N))
    t = rng.random((p, N))
    t0 = time.perf_counter()
    sc = O.proxy_scores(h, t, om, tau, c["sigma"])
    np.argsort(-sc, kind="stable")[:B]
    score_s = time.perf_counter() - t0
    # maintenance on 1/16 of the active rows, scaled by 16 (its cost is linear in rows)
    nA = len(active)
    ns = max(2, nA // 16)
    q = c["q"]
    X = rng.normal(size=(p, ns, q))
    Y = rng.normal(size=(p, ns, q))
    u = rng.normal(size=(p, ns)) * 1e-3
    es = np.searchsorted(active, cand) % ns
    t0 = time.perf_counter()
    O.maintain(X, Y, h, t, u, rng.normal(size=q), 0, 1, es[:, 0], es[:, 1])
    maintain_s = (time.perf_counter() - t0) * (nA / ns)
    return dict(iteration_s=times[warm:], score_s=score_s, maintain_s=maintain_s, p=p, nA=nA,
                sample_s=time.perf_counter() - t_all)


def committed_iterations(config):
    """Seed iterations of each round's shortlist solve and of the bank, from the FP64 GPU run
    recorded in profiles/iterations_per_round.json (the iteration count is a property of the
    linear systems: the FP64 GPU path matches the reference's own counts within 2)."""
    if not os.path.exists(ITER_FILE):
        return None
    with open(ITER_FILE) as f:
        return json.load(f).get(config)


def cpu_round_estimate(parts, rounds_iters, bank_iters, k, q):
    """s/round and k-round greedy seconds of the oracle from timed parts."""
    it_s = float(np.mean(parts["iteration_s"]))
    per_round = it_s * float(np.mean(rounds_iters)) + parts["score_s"] + parts["maintain_s"]
    # the reference solves the bank in chunks of chunk_width columns (16 above 3e6 rows,
    # realworld/polar_gpu.py:169-173), each costing about a B = 16 iteration per iteration
    bank_s = it_s * bank_iters * (2 * q / 16)
    return per_round, bank_s + k * per_round, it_s


# ---------------------------------------------------------------------------------------
def release_device_memory():
    import torch
    from polar_b200 import solver as S
    S._WS.clear()
    torch.cuda.synchronize()
    torch.cuda.empty_cache()


def run_greedy(a):
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
    if a.l2:
        mode, mb = a.l2.split(":")
        _lib.check(lib.polar_set_l2_policy(int(mode), int(float(mb) * (1 << 20))), "l2 policy")
    if a.residual:
        _lib.check(lib.polar_set_mixed_residual(a.residual), "residual storage")
    t_setup = time.perf_counter()
    inp = build_inputs(a)
    n, N, k, E, cand, c = inp["n"], inp["N"], inp["k"], inp["E"], inp["cand"], inp["cfg"]
    rounds = a.warmup + a.steps
    if rounds + 1 > k:
        raise SystemExit(f"warm-up + steps + 1 instrumented round = {rounds + 1} exceeds the workload's k = {k}")
    t_gen = time.perf_counter() - t_setup
    G = pg.Graph(n, E, c["sigma"])
    sk = pg.sketches(G, cand, c["q"], replica_seed(2026, rank), device=True)
    kw = dict(q=c["q"], B=c["B"], tol=c["tol"], sketch=sk, K=c["K"])
    tuned = {}
    if a.autotune == "on" or (a.autotune == "auto" and n < 2_000_000):
        # SpMM layout of the shortlist width, timed once before any greedy
        from polar_b200 import autotune
        for prec in ("mixed",) + (("fp64",) if not a.no_fp64 else ()):
            t = autotune.tune_msolve(pg.Op(G), c["B"], prec, p=c["K"])
            tuned[f"{prec}_R{c['B']}"] = {"lane_bytes": t["best"][0], "sliced_ell": t["best"][1],
                                          "heavy_thresh": t["best"][2], "us_per_iter": t["us_per_iter"],
                                          "layouts_timed": len(t["table"])}
    setup_s = time.perf_counter() - t_setup

    def ev():
        return torch.cuda.Event(enable_timing=True)

    def banked(prec):
        g = pg.Greedy(G, cand, k, c["s"], precision=prec, **kw)
        torch.cuda.synchronize()
        b0, b1 = ev(), ev()
        b0.record()
        g.bank()
        b1.record()
        torch.cuda.synchronize()
        return g, b0.elapsed_time(b1) / 1e3

    # ---- mixed precision: bank, warm-up rounds, then exactly K timed rounds ----
    g, bank_s = banked("mixed")
    for _ in range(a.warmup):
        g.step()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    launches0 = lib.polar_launch_count()
    with Clocks(local) as clk:
        e0, e1 = ev(), ev()
        e0.record()
        for _ in range(a.steps):
            g.step()
        e1.record()
        torch.cuda.synchronize()
    launches = lib.polar_launch_count() - launches0
    total_s = job_seconds(e0.elapsed_time(e1) / 1e3, world, dev)
    per = total_s / a.steps
    # ---- one more round with every solver kernel bracketed by CUDA events (the event
    # nodes serialise the iteration graph, so this round is not part of `value`) ----
    lib.polar_set_kernel_timing(1)
    i0, i1 = ev(), ev()
    i0.record()
    g.step()
    i1.record()
    torch.cuda.synchronize()
    ktime = _lib.kernel_timing()
    lib.polar_set_kernel_timing(0)
    inst_s = i0.elapsed_time(i1) / 1e3
    mixed = g.result()
    del g
    release_device_memory()

    # ---- FP64: the same rounds ----
    fp64 = None
    if not a.no_fp64:
        g, bank64_s = banked("fp64")
        t64 = []
        for _ in range(rounds + 1):
            r0, r1 = ev(), ev()
            r0.record()
            g.step()
            r1.record()
            torch.cuda.synchronize()
            t64.append(r0.elapsed_time(r1) / 1e3)
        fp64 = dict(g.result(), bank_s=bank64_s, round_s=t64)
        del g
        release_device_memory()

    # ---- roofline of the dominant kernel: the SpMM of the shortlist solves ----
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
    e2e = None
    if not a.no_e2e:
        sk_h = [x.cpu().numpy() for x in sk]
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        G2 = pg.Graph(n, E, c["sigma"])
        g2 = pg.Greedy(G2, cand, k, c["s"], q=c["q"], B=c["B"], tol=c["tol"], sketch=sk_h, K=c["K"],
                       precision="mixed")
        seq2 = [g2.step() for _ in range(a.steps)]
        torch.cuda.synchronize()
        e2e_s = (time.perf_counter() - t0) / a.steps
        h2d = E.nbytes + cand.nbytes + sum(x.nbytes for x in sk_h)
        e2e = {"value": e2e_s, "unit": UNIT, "h2d_bytes_per_step": int(h2d / a.steps),
               "d2h_bytes_per_step": int(8 * 6 + 8 * 2),
               "note": "Graph + Greedy from host arrays: uploads, bank and %d rounds, wall clock / %d"
                       % (a.steps, a.steps), "same_sequence": seq2 == mixed["sequence"][:a.steps]}
        del g2, G2, sk_h
        release_device_memory()

    parity = {}
    if fp64 is not None:
        mf = np.asarray(fp64["marginals"])
        mm = np.asarray(mixed["marginals"])
        same = fp64["sequence"] == mixed["sequence"]
        upto = len(mf) if same else next(i for i, (x, y) in enumerate(zip(fp64["sequence"], mixed["sequence"]))
                                         if x != y)
        per64 = float(np.sum(fp64["round_s"][a.warmup:rounds]) / a.steps)
        parity = {"same_sequence": same, "rounds_compared": upto,
                  "max_rel_marginal_err": float(np.max(np.abs(mm[:upto] - mf[:upto]) / np.abs(mf[:upto])))
                  if upto else None,
                  "fp64_round_s": per64, "fp64_bank_s": fp64["bank_s"],
                  "fp64_greedy_s": fp64["bank_s"] + k * per64,
                  "mixed_speedup_vs_fp64": (fp64["bank_s"] + k * per64) / (bank_s + k * per),
                  "mixed_round_speedup_vs_fp64": per64 / per}

    def shortlist_iters(res):
        return [it for R, it in res["solves"] if R == c["B"]]

    cpu = None
    if rank == 0 and world == 1 and not a.no_cpu:
        nth = host_threads()
        parts = oracle_round_parts(inp, a.cpu_iters, threads=nth)
        ref_iters = shortlist_iters(fp64 if fp64 is not None else mixed)
        bank_iters = max(it for R, it in (fp64 or mixed)["solves"] if R != c["B"])
        est, greedy_est, it_s = cpu_round_estimate(parts, ref_iters, bank_iters, k, c["q"])
        cpu = {"value": est, "unit": UNIT, "cores": nth, "kind": "port",
               "greedy_s": greedy_est,
               "sample": (f"oracle (NumPy FP64 restatement of polar_gpu.py) multi-shift CG on this workload's "
                          f"shortlist solve ({c['B']} columns, {parts['p']} poles, {parts['nA']} active rows): "
                          f"{len(parts['iteration_s'])} timed iterations, {it_s:.2f} s each, x "
                          f"{np.mean(ref_iters):.0f} seed iterations per round (this run's "
                          f"{'FP64' if fp64 is not None else 'mixed'} solves) + scoring {parts['score_s']:.2f} s + "
                          f"maintenance {parts['maintain_s']:.2f} s (timed on 1/16 of the rows); the SciPy SpMM and "
                          f"the shifted updates on {nth} host threads, the other NumPy work on one; "
                          f"{parts['sample_s']:.0f} s of host work")}

    if rank == 0:
        line = {
            "metric": METRIC, "value": per, "unit": UNIT, "n_gpus": world, "steps": a.steps, "warmup": a.warmup,
            "ms_per_step": per * 1e3, "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32 SpMM input/output and pole iterates; f64 residual, direction and scalars",
            "data": "synthetic (seeded Chung-Lu stand-in for the %s shape)" % (
                "com-LiveJournal" if a.config == "full-n4M" else a.config),
            "config": {"workload": a.config, "n": n, "m": int(len(E)), "N": N, "K": c["K"], "q": c["q"],
                       "B": c["B"], "k": k, "s": c["s"], "sigma": c["sigma"], "tol": c["tol"],
                       "step": "one greedy round",
                       "l2": "inputs larger than L2 (X/Y banks %.1f GB, SpMM block %.0f MB)"
                             % (mixed["p"] * len(np.unique(cand)) * 2 * c["q"] * 4 / 1e9, n * c["B"] * 4 / 1e6),
                       "parallelism": f"replicas x{world}"},
            "bank_s": bank_s, "greedy_s": bank_s + k * per,
            "e2e": e2e,
            "gpu_launches": int(launches),
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                         "frac": achieved / hbm if achieved else None,
                         "traffic": profiled_traffic(a.config),
                         "kernel": "mk_spmm (SpMM + d.v of the shortlist multi-shift CG, R = %d)" % c["B"],
                         "peak_source": peak_kind, "launches": nl, "avg_launch_us": ms * 1e3 / nl if nl else None,
                         "measured": "CUDA events around every solver kernel in one instrumented round right "
                                     "after the timed region (%.3f s with events)" % inst_s},
            "kernels": kernels,
            "iteration_alg_GBps": (sum(v[2] for v in ktime.values()) / (ktot / 1e3) / 1e9) if ktot else None,
            "parity": parity,
            "sequence_head": mixed["sequence"][:8],
            "p": mixed["p"],
            "iterations": {"bank": [it for R, it in mixed["solves"] if R != c["B"]],
                           "mixed_per_round": shortlist_iters(mixed),
                           "fp64_per_round": shortlist_iters(fp64) if fp64 else None,
                           "fp64_bank": [it for R, it in fp64["solves"] if R != c["B"]] if fp64 else None},
            "cg": {"seed_iterations_per_s": float(np.mean(shortlist_iters(mixed)[a.warmup:rounds])) / per,
                   "column_iterations_per_s": float(np.mean(shortlist_iters(mixed)[a.warmup:rounds])) * c["B"] / per},
            "clocks": clk.summary(),
            "cpu_baseline": cpu,
            "autotune": tuned or None,
            "host_setup_s": setup_s, "input_generation_s": t_gen,
        }
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


def run_solve(a):
    """One shortlist solve of the workload (B incidence columns, all K poles, pole iterates
    on the endpoints of all N candidates) in FP64 and in mixed precision, each with its
    per-kernel table, plus the SpMM alone (polar_spmm through Op) at B and 4B columns.
    --quick: 48-iteration mixed solves at B and 8B columns (the bank width) for every L2
    policy in --l2 (comma-separated MODE:MB; default 0:0,1:64), printing the SpMM time per
    launch; this is also the small case for an ncu capture of the SpMM."""
    import torch

    import polar_b200 as pg
    from polar_b200 import _lib
    from polar_b200 import solver as S
    torch.cuda.set_device(0)
    dev = torch.device("cuda", 0)
    lib = _lib.load()
    t_gen = time.perf_counter()
    inp = build_inputs(a)
    n, E, cand, c = inp["n"], inp["E"], inp["cand"], inp["cfg"]
    G = pg.Graph(n, E, c["sigma"])
    t_gen = time.perf_counter() - t_gen
    op = pg.Op(G)
    tau, om, _ = pg.poles("frac", c["s"], c["sigma"], G.Lam(inp["k"]), 1e-2, K=c["K"])
    R = c["B"]
    pairs = cand[:R]
    active = np.unique(cand)
    W = np.zeros((n, R))
    W[pairs[:, 0], np.arange(R)] = 1.0
    W[pairs[:, 1], np.arange(R)] = -1.0
    Wd = torch.as_tensor(W).to(dev)
    act_d, pos_d = S.prepare_active(active, n, dev)
    ia = np.searchsorted(active, pairs[:, 0])
    ib = np.searchsorted(active, pairs[:, 1])

    def solve(prec, Wm, maxit=100000, act=(act_d, pos_d)):
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        try:
            X, h, it = S.msolve(op, Wm, tau, act[0], c["tol"], maxit=maxit, track=True, precision=prec,
                                active_pos=act[1])
        except _lib.PolarError as e:
            if e.status != _lib.POLAR_ERR_ITER_CAP or maxit == 100000:
                raise
            return None
        e1.record()
        torch.cuda.synchronize()
        cols = torch.arange(R, device=dev)
        bu = (X[:, torch.as_tensor(ia, device=dev), cols].double()
              - X[:, torch.as_tensor(ib, device=dev), cols].double()).cpu().numpy()
        G_q = (om[:, None] * h[:, :R].cpu().numpy() / (1.0 + bu)).sum(0)
        return {"seconds": e0.elapsed_time(e1) / 1e3, "iterations": int(it.max()), "G": G_q}

    if a.quick:
        # small pole state (active rows: the B pairs' endpoints) and full-height blocks
        small = S.prepare_active(np.unique(pairs), n, dev)
        ia = np.searchsorted(np.unique(pairs), pairs[:, 0])
        ib = np.searchsorted(np.unique(pairs), pairs[:, 1])
        W8 = torch.cat([Wd] * 8, dim=1) + 1e-3 * torch.randn((n, 8 * R), device=dev, dtype=torch.float64)
        out = {}
        for pol in (a.l2 or "0:0,1:64").split(","):
            mode, mb = pol.split(":")
            _lib.check(lib.polar_set_l2_policy(int(mode), int(float(mb) * (1 << 20))), "l2 policy")
            row = {}
            for name, Wm in (("R%d" % R, Wd), ("R%d" % (8 * R), W8)):
                for prec in ("mixed", "fp64"):
                    if prec == "fp64" and Wm.shape[1] > 64:
                        continue
                    # lane widths: the solver's default, and 16 / 64 bytes at the bank width
                    for lb in ((0,) if Wm.shape[1] <= 16 else (0, 16, 64)):
                        lib.polar_set_spmm_lane_bytes(lb)
                        lib.polar_set_kernel_timing(1)
                        try:
                            S.msolve(op, Wm, tau, small[0], c["tol"], maxit=48, track=False, precision=prec,
                                     active_pos=small[1])
                        except _lib.PolarError as e:
                            if e.status != _lib.POLAR_ERR_ITER_CAP:
                                raise
                        kt = _lib.kernel_timing()
                        lib.polar_set_kernel_timing(0)
                        lib.polar_set_spmm_lane_bytes(0)
                        key = f"{prec}_{name}" + (f"_lane{lb}" if lb else "")
                        row[key] = {k2: round(v[1] / max(1, v[0]), 4) for k2, v in kt.items() if v[0]}
            out[pol] = row
        _lib.check(lib.polar_set_l2_policy(0, 64 << 20), "l2 policy")
        # heavy-row threshold of the shortlist width (mixed): rows above it go to warp chunks
        from polar_b200 import autotune
        for prec, Wm in (("mixed", Wd), ("fp64", Wd), ("mixed", W8)):
            thr = {}
            for t in (32, 64, 128, 256, 512, 1024):
                autotune.record(G, prec, Wm.shape[1], (0, 1, t))
                lib.polar_set_kernel_timing(1)
                try:
                    S.msolve(op, Wm, tau, small[0], c["tol"], maxit=48, track=False, precision=prec,
                             active_pos=small[1])
                except _lib.PolarError as e:
                    if e.status != _lib.POLAR_ERR_ITER_CAP:
                        raise
                kt = _lib.kernel_timing()
                lib.polar_set_kernel_timing(0)
                thr[t] = round(kt["spmm"][1] / max(1, kt["spmm"][0]), 4)
            autotune.clear(G)
            out["heavy_thresh_%s_R%d" % (prec, Wm.shape[1])] = thr
        print(json.dumps({"workload": a.config, "quick": True, "n": n, "nnz": G.nnz,
                          "ms_per_launch_by_l2_policy": out}), flush=True)
        return
    out = {}
    for prec in ("fp64", "mixed"):
        solve(prec, Wd, maxit=16)  # warm-up: graph partitions, workspace, CUDA graphs
        res = solve(prec, Wd)
        lib.polar_set_kernel_timing(1)
        inst = solve(prec, Wd)
        kt = _lib.kernel_timing()
        lib.polar_set_kernel_timing(0)
        out[prec] = dict(res, kernels={k2: {"launches": v[0], "ms": v[1],
                                            "alg_GBps": v[2] / (v[1] / 1e3) / 1e9 if v[1] > 0 else None}
                                       for k2, v in kt.items() if v[0]},
                         instrumented_seconds=inst["seconds"])
    G64, G32 = out["fp64"].pop("G"), out["mixed"].pop("G")
    hbm, peak_kind = peak_hbm()
    spmm = {}
    for dt, nm in ((torch.float64, "fp64"), (torch.float32, "mixed")):
        for Rc in (R, 4 * R):
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
    line = {"metric": "shortlist solve (B columns, K poles)", "unit": "s/solve",
            "value": out["mixed"]["seconds"], "higher_is_better": False, "n_gpus": 1,
            "config": {"workload": a.config, "n": n, "m": int(len(E)), "nnz": G.nnz, "dmax": G.dmax,
                       "nA": int(len(active)), "K": c["K"], "R": R, "tol": c["tol"], "sigma": c["sigma"], "s": c["s"]},
            "fp64": out["fp64"], "mixed": out["mixed"],
            "mixed_speedup_vs_fp64": out["fp64"]["seconds"] / out["mixed"]["seconds"],
            "max_rel_marginal_err": float(np.max(np.abs(G32 - G64) / np.abs(G64))),
            "spmm_alone": spmm, "peak_GBps": hbm, "peak_source": peak_kind, "host_setup_s": t_gen}
    print(json.dumps(line), flush=True)


def run_diff(a):
    """Differentiation workload: Chung–Lu n = 1,134,890 (~2.99M edges, exponent 2.2, seed 3),
    sigma = 1e-2, s = 0.5, K = 24 poles; 4,096 candidate non-edges with relaxed weights
    w ~ U[0, 1].  Times FracTrace's two halves on the device (the grouped forward f_s with
    f_{s+1} for d f / d sigma, and the adjoint d f / d w for all 4,096 weights), checks
    sampled adjoint entries against central differences (h = 1e-4) computed from solves
    that do not share the adjoint's, and checks the adjoint against the dense FP64
    eigendecomposition gradient on a 3,000-vertex induced subgraph."""
    import torch

    import polar_b200 as pg
    from polar_b200.adjoint import relaxed_central_difference, relaxed_gradient, relaxed_objective, relaxed_rule
    from oracle import polar_oracle as O
    from polar_b200.synth import candidates
    torch.cuda.set_device(0)
    inp = build_inputs(a)
    n, E, cand, c = inp["n"], inp["E"], inp["cand"], inp["cfg"]
    rng = np.random.default_rng(c["seed"])
    w = rng.uniform(0.0, 1.0, len(cand))
    G = pg.Graph(n, E, c["sigma"])
    tau, om = relaxed_rule(G, c["s"], K=c["K"])
    tol = c["tol"]

    def timed(fn):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        out = fn()
        torch.cuda.synchronize()
        return out, time.perf_counter() - t0

    out = {}
    line = {"metric": "relaxed-weight objective and adjoint (FracTrace halves)", "unit": "s", "higher_is_better": False,
            "n_gpus": 1,
            "config": {"workload": a.config, "n": n, "m": int(len(E)), "candidates": len(cand), "K": c["K"],
                       "s": c["s"], "sigma": c["sigma"], "tol": tol}}
    if not a.dense_only:
        for prec in ("fp64", "mixed"):
            grad, tg = timed(lambda: relaxed_gradient(G, cand, w, c["s"], tau=tau, om=om, tol=tol, precision=prec))
            out[prec] = {"gradient_s": tg, "grad": grad}
        (f, f_next), tf = timed(lambda: relaxed_objective(G, cand, w, c["s"], tau=tau, om=om, tol=tol,
                                                          with_next=True))
        g64 = out["fp64"]["grad"]
        sample = [int(i) for i in rng.choice(np.flatnonzero(w >= 1e-3), 8, replace=False)]
        fd = []
        for i in sample:
            v, t = timed(lambda: relaxed_central_difference(G, cand, w, c["s"], i, 1e-4, tau=tau, om=om, tol=tol))
            fd.append({"i": i, "fd": float(v), "grad": float(g64[i]), "rel_err": float(abs(v - g64[i]) / abs(v)),
                       "seconds": t})
        line.update({"value": out["fp64"]["gradient_s"], "forward_s": tf, "f": float(f),
                     "dsigma": float(-c["s"] * f_next),
                     "gradient_fp64_s": out["fp64"]["gradient_s"], "gradient_mixed_s": out["mixed"]["gradient_s"],
                     "mixed_vs_fp64_max_rel": float(np.max(np.abs(out["mixed"]["grad"] - g64) / np.abs(g64))),
                     "central_differences": fd,
                     "max_rel_err_vs_central_differences": max(x["rel_err"] for x in fd)})
    # dense check: induced subgraph on the 3,000 lowest ids (the hubs and their mutual edges)
    ns = 3000
    Es = E[(E[:, 0] < ns) & (E[:, 1] < ns)]
    cs = candidates(ns, Es, 256, c["seed"] + 11)
    ws = rng.uniform(0.0, 1.0, len(cs))
    Gs = pg.Graph(ns, Es, c["sigma"])
    ts, oms = relaxed_rule(Gs, c["s"], K=c["K"])
    gs = relaxed_gradient(Gs, cs, ws, c["s"], tau=ts, om=oms, tol=1e-12)
    d = O.relaxed_dense(ns, Es, c["sigma"], cs, ws, c["s"], ts, oms)
    # the same check with a fine composite rule (eps = 1e-9): the adjoint converges to the
    # exact gradient as the rule does
    t_fine, om_fine = relaxed_rule(Gs, c["s"], K=None, eps=1e-9)
    gsf = relaxed_gradient(Gs, cs, ws, c["s"], tau=t_fine, om=om_fine, tol=1e-12)
    line["dense_subgraph"] = {
        "n": ns, "m": int(len(Es)), "candidates": len(cs),
        "max_rel_err_vs_rule": float(np.max(np.abs(gs - d["grad_q"]) / np.abs(d["grad_q"]))),
        "max_rel_err_vs_exact": float(np.max(np.abs(gs - d["grad"]) / np.abs(d["grad"]))),
        "fine_rule_poles": int(len(t_fine)),
        "fine_rule_max_rel_err_vs_exact": float(np.max(np.abs(gsf - d["grad"]) / np.abs(d["grad"])))}
    print(json.dumps(line), flush=True)


def run_reference(a):
    """The reference's algorithm on the host cores for the same workload and metric: the
    oracle (a NumPy FP64 restatement of realworld/polar_gpu.py, pinned to the reference's
    own outputs; the reference itself needs CuPy and a GPU).  Each timed step is
    ceil(20 / K) multi-shift CG iterations of the workload's shortlist solve (B columns, all K
    poles, all active rows, full graph), so that at least 20 real iterations are timed; each
    warm-up step is one iteration.  value = s per iteration x the seed iterations of a round
    (the FP64 GPU path's per-round counts, profiles/iterations_per_round.json) + the
    per-round scoring and maintenance, timed once.  Rank 0 alone runs; other ranks exit."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    rec = committed_iterations(a.config)
    if rec is None:
        print(json.dumps({"impl": "reference", "unavailable": "no recorded per-round iteration counts for "
                          f"{a.config} in profiles/iterations_per_round.json"}), flush=True)
        return
    inp = build_inputs(a)
    c = inp["cfg"]
    t0 = time.perf_counter()
    nth = host_threads()
    per_step = -(-20 // max(1, a.steps))
    parts = oracle_round_parts(inp, per_step * a.steps, warm=1 + a.warmup, threads=nth)
    run_s = time.perf_counter() - t0
    per, greedy_s, it_s = cpu_round_estimate(parts, rec["fp64_per_round"], max(rec["fp64_bank"]), inp["k"], c["q"])
    cpu = {"value": per, "unit": UNIT, "cores": nth, "kind": "port", "greedy_s": greedy_s,
           "sample": (f"oracle multi-shift CG on the shortlist solve ({c['B']} columns, {parts['p']} poles, "
                      f"{parts['nA']} active rows): {len(parts['iteration_s'])} timed iterations "
                      f"({a.steps} steps of {per_step}), {it_s:.2f} s each, x "
                      f"{np.mean(rec['fp64_per_round']):.0f} seed iterations per round (FP64 GPU counts) + scoring "
                      f"{parts['score_s']:.2f} s + maintenance {parts['maintain_s']:.2f} s; sparse product and "
                      f"shifted updates on {nth} host threads, other NumPy work on one")}
    line = {"impl": "reference", "metric": METRIC, "value": per, "unit": UNIT, "n_gpus": world, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": per_step * it_s * 1e3, "higher_is_better": False, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded Chung-Lu stand-in for the %s shape)" % (
                "com-LiveJournal" if a.config == "full-n4M" else a.config),
            "config": {"workload": a.config, "n": inp["n"], "m": int(len(inp["E"])), "N": inp["N"], "K": c["K"],
                       "q": c["q"], "B": c["B"], "k": inp["k"], "s": c["s"], "sigma": c["sigma"], "tol": c["tol"],
                       "step": "%d multi-shift CG iterations of a round's shortlist solve (value: s/round)"
                               % per_step},
            "greedy_s": greedy_s, "timed_run_s": run_s,
            "cpu_baseline": cpu, "e2e": {"value": per, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


if __name__ == "__main__":
    args = parse()
    if args.impl == "reference" and args.config in ("batch48", "diff-n1.13M"):
        print(json.dumps({"impl": "reference", "unavailable": {
            "batch48": "the many-graphs workload has no reference arm: the reference solves one graph per call",
            "diff-n1.13M": "the reference has no relaxed-weight objective or adjoint"}[args.config]}), flush=True)
    elif args.impl == "reference":
        run_reference(args)
    elif args.config == "batch48":
        run_batch(args)
    elif args.config == "diff-n1.13M":
        run_diff(args)
    elif args.solve:
        run_solve(args)
    else:
        run_greedy(args)
