"""The CPU model of the mixed-precision solver (oracle.precision_model): keeping the residual
and the direction recurrence in FP64, with only the SpMM's copy of the direction, its output
and the shifted iterates in FP32 (the device's mixed scheme), gives a smaller marginal error
than storing every vector in FP32.  CPU only."""
import numpy as np

from oracle import precision_model as PM
from polar_b200 import quadrature as Q
from polar_b200.synth import candidates, chung_lu


def test_device_scheme_beats_all_fp32():
    n = 30000
    E = chung_lu(n, 6.6, 2.4, 1, min_degree=1)
    A, deg = PM.laplacian(n, E)
    tau, om, _ = Q.poles("frac", 0.5, 1e-2, 1e-2 + 2 * deg.max() + 200, 1e-2, K=24)
    pairs = candidates(n, E, 16, 77)
    it0, G0 = PM.shortlist_solve(A, deg, 1e-2, tau, om, pairs)
    it32, G32 = PM.shortlist_solve(A, deg, 1e-2, tau, om, pairs, r=True, d=True, dm=True, v=True, xp=True)
    itd, Gd = PM.shortlist_solve(A, deg, 1e-2, tau, om, pairs, dm=True, v=True, xp=True)
    e32 = np.max(np.abs(G32 - G0) / np.abs(G0))
    ed = np.max(np.abs(Gd - G0) / np.abs(G0))
    assert ed < 0.6 * e32 and ed < 2e-7, (ed, e32)
    assert it0 <= itd <= 1.1 * it0 and it0 <= it32
