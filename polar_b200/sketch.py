"""Sketch inputs Z (n x q), F = C_0^T U (n x q) and Gc (N x q).

Same random stream and construction as realworld/polar_gpu.py:137-165 for the 'block'
and 'gauss' kinds, so a seed reproduces the reference's sketches.  'rademacher' (entries
+-1/sqrt(q); Z centred) is an additional kind drawn in the same order (Z, then the
edge-incidence rows U in 4M-edge chunks, then Gc).  Sketches are inputs of the timed
path; the reference also builds them on the host, outside its timed region.

device=True keeps the random draws on the host (NumPy's generator, same order) and does
the rest on the GPU (libpolar): the sign-fixed QR of every Gaussian q x q block
(polar_block_orth), the centring of Z (polar_center_columns) and F += C_0^T U over the
edge chunks (polar_incidence_apply).  It returns float64 CUDA tensors equal to the host
arrays up to rounding (the QR runs as two-pass Gram-Schmidt instead of Householder).
"""
import numpy as np
import scipy.sparse as sp

__all__ = ["sketches", "block_rows", "chunk_width"]


def block_rows(rows, q, rng, center=False):
    """Rows of independent Haar q x q orthogonal blocks (sign-fixed QR of Gaussians)."""
    nb = -(-rows // q)
    g = rng.normal(size=(nb, q, q))
    Q, Rm = np.linalg.qr(g)
    Q = Q * np.sign(np.diagonal(Rm, axis1=1, axis2=2))[:, None, :]
    out = np.transpose(Q, (0, 2, 1)).reshape(nb * q, q)[:rows]
    if center:
        out = out - out.mean(0)
    return out


def _draw(kind, rows, q, rng, center=False):
    if kind == "gauss":
        out = rng.normal(size=(rows, q)) / np.sqrt(q)
        return out
    if kind == "rademacher":
        out = (rng.integers(0, 2, size=(rows, q), dtype=np.int8) * 2 - 1).astype(np.float64) / np.sqrt(q)
        if center:
            out = out - out.mean(0)
        return out
    if kind == "block":
        return block_rows(rows, q, rng, center=center)
    raise ValueError(f"unknown sketch kind {kind!r}")


def sketches(G, cand, q, seed, kind="block", chunk=4_000_000, *, device=False):
    """(Z, F, Gc) as float64 host arrays (device=True: float64 CUDA tensors on G's device)."""
    if device:
        return _sketches_device(G, cand, q, seed, kind, chunk)
    rng = np.random.default_rng(seed)
    n = G.n
    Z = _draw(kind, n, q, rng, center=(kind != "gauss"))
    F = np.zeros((n, q))
    u, v = G.edges[:, 0], G.edges[:, 1]
    sw = np.sqrt(G.weights)
    for lo in range(0, G.m, chunk):
        hi = min(G.m, lo + chunk)
        U = _draw(kind, hi - lo, q, rng)
        U *= sw[lo:hi, None]
        ne = hi - lo
        C = sp.csr_matrix((np.r_[np.ones(ne), -np.ones(ne)],
                           (np.r_[u[lo:hi], v[lo:hi]], np.r_[np.arange(ne), np.arange(ne)])), shape=(n, ne))
        F += C @ U
    Gc = _draw(kind, len(cand), q, rng)
    return Z, F, Gc


def _sketches_device(G, cand, q, seed, kind, chunk):
    import torch

    from . import _lib
    if kind not in ("block", "gauss", "rademacher"):
        raise ValueError(f"unknown sketch kind {kind!r}")
    lib = _lib.load()
    dev = G.device
    stream = torch.cuda.current_stream(dev).cuda_stream
    rng = np.random.default_rng(seed)
    n = G.n

    def center(out):
        tmp = torch.empty(int(lib.polar_center_columns_tmp_bytes(q)), dtype=torch.uint8, device=dev)
        _lib.check(lib.polar_center_columns(out.data_ptr(), out.shape[0], q, q, tmp.data_ptr(), tmp.numel(), stream),
                   "polar_center_columns")

    def draw(rows, do_center=False, scale=None):
        if kind == "block":
            nb = -(-rows // q)
            g = torch.as_tensor(rng.normal(size=(nb, q, q))).to(dev)
            out = torch.empty((rows, q), dtype=torch.float64, device=dev)
            sc = None if scale is None else torch.as_tensor(np.ascontiguousarray(scale, dtype=np.float64)).to(dev)
            _lib.check(lib.polar_block_orth(g.data_ptr(), rows, q, None if sc is None else sc.data_ptr(),
                                            out.data_ptr(), q, stream), "polar_block_orth")
            if do_center:
                center(out)
            return out
        host = _draw(kind, rows, q, rng)
        if scale is not None:
            host = host * np.asarray(scale, dtype=np.float64)[:, None]
        out = torch.as_tensor(np.ascontiguousarray(host)).to(dev)
        if do_center:
            center(out)
        return out

    Z = draw(n, do_center=(kind != "gauss"))
    F = torch.zeros((n, q), dtype=torch.float64, device=dev)
    u, v = G.edges[:, 0], G.edges[:, 1]
    sw = np.sqrt(G.weights)
    for lo in range(0, G.m, chunk):
        hi = min(G.m, lo + chunk)
        ne = hi - lo
        U = draw(ne, scale=sw[lo:hi])
        C = sp.csr_matrix((np.r_[np.ones(ne, np.int8), -np.ones(ne, np.int8)],
                           (np.r_[u[lo:hi], v[lo:hi]], np.r_[np.arange(ne), np.arange(ne)])), shape=(n, ne))
        C.sort_indices()
        ip = torch.as_tensor(C.indptr.astype(np.int32)).to(dev)
        ix = torch.as_tensor(C.indices.astype(np.int32)).to(dev)
        sg = torch.as_tensor(C.data.astype(np.int8)).to(dev)
        _lib.check(lib.polar_incidence_apply(n, ip.data_ptr(), ix.data_ptr(), sg.data_ptr(), U.data_ptr(), q, q,
                                             F.data_ptr(), q, stream), "polar_incidence_apply")
    Gc = draw(len(cand))
    return Z, F, Gc


def chunk_width(n, p, nA, budget=10e9):
    """The reference's bank width heuristic (realworld/polar_gpu.py:169-173), kept for the
    API; the device path picks its own width from the kernel's column limit."""
    per_col = 8.0 * (10 * n + 4 * p * nA)
    cap = 16 if n > 3e6 else 64
    return int(max(8, min(cap, budget // per_col)))
