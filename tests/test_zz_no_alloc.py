"""polar_spmm_noalloc (fixed in-library scratch) against polar_spmm (caller scratch), both
through the C ABI.  Collected last so it runs both alone and after every other GPU test.
Needs a B200."""
import ctypes

import numpy as np
import pytest

from polar_b200.synth import chung_lu

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
@pytest.mark.parametrize("R", [5, 16])
def test_noalloc_matches_caller_scratch(prec, R):
    import torch
    import polar_b200 as pg
    from polar_b200 import _lib
    lib = _lib.load()
    n = 4000
    G = pg.Graph(n, chung_lu(n, 6.0, 2.2, 9), 1e-2, heavy_thresh=8)  # many heavy-row chunks
    op = pg.Op(G)
    for a, b in [(0, 5), (17, 3999), (0, 17)]:
        op.add(a, b)
    dt = torch.float64 if prec == "fp64" else torch.float32
    code = _lib.POLAR_FP64 if prec == "fp64" else _lib.POLAR_MIXED
    X = torch.as_tensor(np.random.default_rng(R).normal(size=(n, R)), dtype=dt, device="cuda")
    Y0 = op(X, 0.37)  # polar_spmm with scratch from the caller
    # the graph struct op() hands to polar_spmm for this width (its sliced-ELL layout when
    # R is a power of two), so both entry points run the same kernel
    g = op.struct(sell_rows=lib.polar_sell_rows(code, R))
    stream = torch.cuda.current_stream().cuda_stream
    outs = []
    for _ in range(2):  # two calls in a row reuse the same fixed scratch
        Y = torch.full_like(X, float("nan"))
        _lib.check(lib.polar_spmm_noalloc(ctypes.byref(g), code, R, 0.37, X.data_ptr(), R, Y.data_ptr(), R,
                                          stream), "polar_spmm_noalloc")
        outs.append(Y)
    torch.cuda.synchronize()
    for Y in outs:
        assert torch.equal(Y, Y0)


def test_noalloc_rejects_oversize_scratch():
    import torch
    import polar_b200 as pg
    from polar_b200 import _lib
    lib = _lib.load()
    n = 40000
    G = pg.Graph(n, chung_lu(n, 12.0, 2.2, 3), 1e-2, heavy_thresh=8)
    g = pg.Op(G).struct()
    need = lib.polar_spmm_scratch_bytes(ctypes.byref(g), _lib.POLAR_FP64, 16)
    assert need > 8 << 20
    X = torch.zeros((n, 16), dtype=torch.float64, device="cuda")
    Y = torch.zeros_like(X)
    before = lib.polar_launch_count()
    rc = lib.polar_spmm_noalloc(ctypes.byref(g), _lib.POLAR_FP64, 16, 0.0, X.data_ptr(), 16, Y.data_ptr(), 16,
                                torch.cuda.current_stream().cuda_stream)
    assert rc == _lib.POLAR_ERR_WORKSPACE
    assert b"fixed" in lib.polar_last_error()
    assert lib.polar_launch_count() == before


def test_noalloc_rejects_bad_arguments_before_queueing():
    """Bad sizes and a weights/diagonal mismatch return BAD_ARG before the counter clear is
    queued: a capture of the stream around the rejected calls holds no node."""
    import torch
    from cuda.bindings import runtime as rt
    import polar_b200 as pg
    from polar_b200 import _lib
    lib = _lib.load()
    n = 4000
    G = pg.Graph(n, chung_lu(n, 6.0, 2.2, 9), 1e-2, heavy_thresh=8)
    g = pg.Op(G).struct()
    X = torch.zeros((n, 16), dtype=torch.float64, device="cuda")
    Y = torch.zeros_like(X)
    gw = pg.Op(G).struct()
    gw.d_wts = X.data_ptr()  # weights without a diagonal
    s = torch.cuda.Stream()
    h = s.cuda_stream
    (err,) = rt.cudaStreamBeginCapture(h, rt.cudaStreamCaptureMode.cudaStreamCaptureModeRelaxed)
    assert err == rt.cudaError_t.cudaSuccess
    rcs = [lib.polar_spmm_noalloc(ctypes.byref(g), _lib.POLAR_FP64, 0, 0.0, X.data_ptr(), 16, Y.data_ptr(), 16, h),
           lib.polar_spmm_noalloc(ctypes.byref(g), _lib.POLAR_FP64, 16, 0.0, X.data_ptr(), 8, Y.data_ptr(), 16, h),
           lib.polar_spmm_noalloc(ctypes.byref(g), 9, 16, 0.0, X.data_ptr(), 16, Y.data_ptr(), 16, h),
           lib.polar_spmm_noalloc(ctypes.byref(gw), _lib.POLAR_FP64, 16, 0.0, X.data_ptr(), 16, Y.data_ptr(), 16, h)]
    err, graph = rt.cudaStreamEndCapture(h)
    assert err == rt.cudaError_t.cudaSuccess
    err, _, count = rt.cudaGraphGetNodes(graph, 0)
    rt.cudaGraphDestroy(graph)
    assert rcs == [_lib.POLAR_ERR_BAD_ARG] * 4
    assert count == 0
