"""Host side of bench.py: the CPU baseline's timed oracle sample and its per-round
arithmetic, on a small workload (no GPU)."""
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT))


def test_oracle_round_parts_small():
    import bench
    from polar_b200.synth import CONFIGS, candidates, chung_lu
    c = dict(CONFIGS["precision-n317k"])
    n, N = 3000, 2000
    E = chung_lu(n, c["mean_deg"], c["gamma"], c["seed"], min_degree=1)
    inp = dict(n=n, N=N, k=10, E=E, cand=candidates(n, E, N, 5), cfg=c)
    seen = []
    parts = bench.oracle_round_parts(inp, 3, on_sample=lambda i, s: seen.append((i, s)))
    assert len(parts["iteration_s"]) == 3 and all(t > 0 for t in parts["iteration_s"])
    assert [i for i, _ in seen] == [0, 1, 2]
    assert parts["p"] == c["K"] and parts["nA"] == len(np.unique(inp["cand"]))
    assert parts["score_s"] > 0 and parts["maintain_s"] > 0
    per, greedy, it_s = bench.cpu_round_estimate(parts, [100, 120], 150, 10, c["q"])
    assert it_s == pytest.approx(np.mean(parts["iteration_s"]))
    assert per == pytest.approx(it_s * 110 + parts["score_s"] + parts["maintain_s"])
    assert greedy == pytest.approx(it_s * 150 * (2 * c["q"] / 16) + 10 * per)
