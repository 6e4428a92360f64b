"""polar_b200 — B200-native (sm_100a) solve-and-score path of POLAR.

Drop-in for the entry points of realworld/polar_gpu.py that the drivers call
(`import polar_b200 as pg`): Graph, Op, msolve, composite, poles, sketches, polar,
true_marginals, degree_greedy, random_set, chunk_width.  The compute runs in the
hand-written kernels of libpolar.so (include/polar.h) through ctypes; there is no CPU
fallback.  Keyword-only extensions: precision='fp64'|'mixed', K=<fixed pole count>.
Beyond the reference: FracTrace / relaxed_gradient / relaxed_objective, the relaxed-weight
objective f_s(w, sigma) with its adjoint (polar_b200.adjoint); polar_split, the greedy with
its sketch and shortlist columns split over the ranks of a process group (polar_b200.split).
"""
from .quadrature import composite, fixed_rule, poles
from .sketch import sketches, chunk_width
from .synth import chung_lu, candidates

__version__ = "0.1.0"

_DEVICE_NAMES = ("Graph", "Op", "msolve", "Counter", "polar", "Greedy", "true_marginals", "degree_greedy", "random_set",
                 "FracTrace", "relaxed_gradient", "relaxed_objective", "polar_split")


def __getattr__(name):
    # Device-side names load libpolar.so on first use, so host-only helpers (quadrature,
    # sketches, generators) import on machines without a GPU.
    if name in ("Graph", "Op"):
        from . import graph
        return getattr(graph, name)
    if name in ("msolve", "Counter"):
        from . import solver
        return getattr(solver, name)
    if name in ("polar", "Greedy", "true_marginals", "degree_greedy", "random_set"):
        from . import greedy
        return getattr(greedy, name)
    if name == "polar_split":
        from . import split
        return split.polar_split
    if name in ("FracTrace", "relaxed_gradient", "relaxed_objective"):
        from . import adjoint
        return getattr(adjoint, name)
    raise AttributeError(name)


__all__ = ["composite", "fixed_rule", "poles", "sketches", "chunk_width", "chung_lu", "candidates",
           *_DEVICE_NAMES]
