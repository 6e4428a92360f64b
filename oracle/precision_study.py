"""Which vectors of the multi-shift CG may be stored in FP32?  Runs oracle.precision_model on
the n = 317,080 Chung-Lu workload (the shortlist solve of 16 incidence columns, K = 24 poles,
tol 1e-7) for each storage scheme and prints seed iterations and the marginal error
against the all-FP64 run.  CPU only; each scheme takes a few minutes.

    python -m oracle.precision_study [--n 317080] [--schemes all32,device,...]
"""
import argparse
import json
import os
import sys
import time

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))

from oracle import precision_model as PM  # noqa: E402
from polar_b200 import quadrature as Q  # noqa: E402
from polar_b200.synth import CONFIGS, candidates, chung_lu  # noqa: E402

SCHEMES = {
    "all32": dict(r=True, d=True, dm=True, v=True, xp=True),
    "r32": dict(r=True),
    "d32": dict(d=True, dm=True),
    "v32": dict(v=True),
    "r64": dict(d=True, dm=True, v=True, xp=True),
    "device": dict(dm=True, v=True, xp=True),
    "device_r32": dict(r=True, dm=True, v=True, xp=True),
    "device_r32_ru50": dict(r=True, dm=True, v=True, xp=True, ru=50),
    "all32_ru50": dict(r=True, d=True, dm=True, v=True, xp=True, ru=50),
}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=CONFIGS["precision-n317k"]["n"])
    ap.add_argument("--schemes", default=",".join(SCHEMES))
    a = ap.parse_args()
    c = CONFIGS["precision-n317k"]
    E = chung_lu(a.n, c["mean_deg"], c["gamma"], c["seed"], min_degree=1)
    A, deg = PM.laplacian(a.n, E)
    tau, om, _ = Q.poles("frac", c["s"], c["sigma"], c["sigma"] + 2 * deg.max() + 4 * c["k"], 1e-2, K=c["K"])
    pairs = candidates(a.n, E, 16, 77)
    t0 = time.time()
    it0, G0 = PM.shortlist_solve(A, deg, c["sigma"], tau, om, pairs, tol=c["tol"])
    print(json.dumps({"scheme": "fp64", "iterations": it0, "seconds": round(time.time() - t0, 1)}), flush=True)
    for name in a.schemes.split(","):
        t0 = time.time()
        it, G = PM.shortlist_solve(A, deg, c["sigma"], tau, om, pairs, tol=c["tol"], **SCHEMES[name])
        err = float(np.max(np.abs(G - G0) / np.abs(G0)))
        print(json.dumps({"scheme": name, "iterations": it, "max_rel_marginal_err": err,
                          "seconds": round(time.time() - t0, 1)}), flush=True)


if __name__ == "__main__":
    main()
