"""Graph operator on the device: M0 = L + sigma I as a CSR of neighbour lists, and the
operator view Op = M0 + sum_S w b b^T (+ shift I) used by the solver.

Mirrors realworld/polar_gpu.py:47-80 (Graph, Op).  Layout in HBM:
* indptr int32[n+1], indices int32[nnz] (off-diagonal neighbours only, sorted per row);
  unweighted graphs store no values (weight 1, diagonal = degree + sigma);
* weighted graphs add wts float64[nnz] and diag float64[n];
* rows with more than `heavy_thresh` neighbours are split into chunks of that size
  (hrow, hchunk_off, chunk_row/lo/hi), combined in a fixed order by the kernels;
* edges added by Op.add live in a small side structure (bitset over rows + sorted row
  list + neighbour lists), so the CSR is never rebuilt during the greedy.
"""
import numpy as np
import scipy.sparse as sp
import torch

from . import _lib

__all__ = ["Graph", "Op", "default_device", "csr_from_edges", "sell_slices", "sell_slices_torch"]


def default_device():
    """The current CUDA device; Graph(device='cpu') builds the host structures only
    (for tests of the host logic), and no kernel can run on it."""
    if not torch.cuda.is_available():
        raise RuntimeError("polar_b200 needs a CUDA device (B200, sm_100a); none is available")
    return torch.device("cuda", torch.cuda.current_device())


def _i32(x, dev):
    return torch.as_tensor(np.ascontiguousarray(x, dtype=np.int32)).to(dev)


def sell_slices(indptr, indices, light_mask, S, window=4096):
    """Sliced ELL of the light rows for warps of S rows: rows are sorted by degree
    (descending) within windows of `window` rows, cut into slices of S rows, and each
    slice stores its neighbour lists column-major (index k of row r at off + k*S + r),
    padded with -1 to the slice's largest degree.  Returns (slice_off int32[ns+1],
    slice_rows int32[ns*S] (-1 pads), sidx int32)."""
    rows = np.flatnonzero(light_mask).astype(np.int64)
    if len(rows) == 0:
        return np.zeros(1, np.int32), np.zeros(0, np.int32), np.zeros(0, np.int32)
    deg = (indptr[rows + 1] - indptr[rows]).astype(np.int64)
    win = np.arange(len(rows)) // window
    order = np.lexsort((-deg, win))
    rows = rows[order]
    deg = deg[order]
    ns = -(-len(rows) // S)
    pad = ns * S - len(rows)
    rows_p = np.r_[rows, -np.ones(pad, np.int64)].reshape(ns, S)
    deg_p = np.r_[deg, np.zeros(pad, np.int64)].reshape(ns, S)
    width = deg_p.max(axis=1)
    off = np.zeros(ns + 1, np.int64)
    off[1:] = np.cumsum(width * S)
    sidx = -np.ones(int(off[-1]), np.int64)
    # position of neighbour k of slice row r: off[s] + k*S + r
    rr = np.repeat(np.arange(ns * S), deg_p.ravel())
    s_of = rr // S
    r_in = rr % S
    k_in = np.arange(len(rr)) - np.repeat(np.cumsum(deg_p.ravel()) - deg_p.ravel(), deg_p.ravel())
    src = np.repeat(indptr[np.maximum(rows_p.ravel(), 0)].astype(np.int64), deg_p.ravel()) + k_in
    sidx[off[s_of] + k_in * S + r_in] = indices[src]
    if off[-1] >= 2 ** 31:
        raise ValueError("sliced ELL too large for int32 offsets")
    return off.astype(np.int32), rows_p.ravel().astype(np.int32), sidx.astype(np.int32)


def csr_from_edges(n, u, v):
    """Symmetric unweighted adjacency CSR from an edge list, with torch on the edge arrays'
    device (the ingestion step of realworld/graphs.py:46-58 and polar_gpu.py:48-58, which
    build it with scipy on the host): both directions, sorted by (row, column), repeated
    pairs merged.  Returns (indptr int32[n+1], indices int32[nnz], counts int64[nnz]); a
    count above 1 is a merged repeated edge (a weight above 1)."""
    n = int(n)
    rows = torch.cat([u, v]).to(torch.int64)
    cols = torch.cat([v, u]).to(torch.int64)
    key, _ = torch.sort(rows * n + cols)
    uniq, counts = torch.unique_consecutive(key, return_counts=True)
    r = torch.div(uniq, n, rounding_mode="floor")
    indptr = torch.zeros(n + 1, dtype=torch.int64, device=u.device)
    indptr[1:] = torch.cumsum(torch.bincount(r, minlength=n), 0)
    return indptr.to(torch.int32), (uniq - r * n).to(torch.int32), counts


def sell_slices_torch(indptr, indices, light_mask, S, window=4096):
    """sell_slices with torch on the arrays' device; the same three arrays (as int32
    tensors on that device)."""
    dev = indptr.device
    rows = torch.nonzero(light_mask).flatten()
    if rows.numel() == 0:
        z = torch.zeros(1, dtype=torch.int32, device=dev)
        return z, torch.zeros(0, dtype=torch.int32, device=dev), torch.zeros(0, dtype=torch.int32, device=dev)
    ip = indptr.to(torch.int64)
    deg = ip[rows + 1] - ip[rows]
    dmax = int(deg.max())
    win = torch.arange(rows.numel(), device=dev) // window
    _, order = torch.sort(win * (dmax + 1) + (dmax - deg), stable=True)
    rows = rows[order]
    deg = deg[order]
    ns = -(-rows.numel() // S)
    pad = ns * S - rows.numel()
    rows_p = torch.cat([rows, torch.full((pad,), -1, dtype=torch.int64, device=dev)])
    deg_p = torch.cat([deg, torch.zeros(pad, dtype=torch.int64, device=dev)])
    width = deg_p.view(ns, S).max(dim=1).values
    off = torch.zeros(ns + 1, dtype=torch.int64, device=dev)
    off[1:] = torch.cumsum(width * S, 0)
    sidx = torch.full((int(off[-1]),), -1, dtype=torch.int32, device=dev)
    rr = torch.repeat_interleave(torch.arange(ns * S, device=dev), deg_p)
    start = torch.cumsum(deg_p, 0) - deg_p
    k_in = torch.arange(rr.numel(), device=dev) - torch.repeat_interleave(start, deg_p)
    src = torch.repeat_interleave(ip[rows_p.clamp_min(0)], deg_p) + k_in
    sidx[off[rr // S] + k_in * S + rr % S] = indices[src].to(torch.int32)
    if int(off[-1]) >= 2 ** 31:
        raise ValueError("sliced ELL too large for int32 offsets")
    return off.to(torch.int32), rows_p.to(torch.int32), sidx


def row_blocks(indptr, heavy_thresh, row_cost=4, target=None):
    """Contiguous blocks of light rows (degree <= heavy_thresh) with about `target` work
    each, work = nnz + row_cost per row; heavy rows are never inside a block.  Returns
    int32[nrb, 2] of [first row, one past last row]."""
    deg = np.diff(indptr.astype(np.int64))
    n = len(deg)
    if n == 0:
        return np.zeros((0, 2), np.int32)
    light = deg <= heavy_thresh
    cost = np.where(light, deg + row_cost, 0)
    if target is None:
        target = int(np.clip(cost.sum() / 30000.0, 32, 512))
    run = np.cumsum(~light)                       # run id changes at every heavy row
    cum = np.cumsum(cost) - cost                  # work before row i
    run_start = np.zeros(run.max() + 2, np.int64)
    first = np.r_[True, run[1:] != run[:-1]]
    run_start[run[first]] = cum[first]
    key = run * (1 << 40) + (cum - run_start[run]) // target
    idx = np.flatnonzero(light)
    if len(idx) == 0:
        return np.zeros((0, 2), np.int32)
    k = key[idx]
    brk = np.r_[True, (k[1:] != k[:-1]) | (idx[1:] != idx[:-1] + 1)]
    starts = idx[brk]
    ends = np.r_[idx[np.flatnonzero(brk)[1:] - 1] + 1, idx[-1] + 1]
    return np.stack([starts, ends], axis=1).astype(np.int32)


class _HostM0:
    """Host FP64 CSR of M0 = diag(deg + sigma) - A with the `.get()` the drivers call
    (realworld/run_real.py:49 uses G.M0.get().toarray() for dense oracles)."""

    def __init__(self, G):
        self._G = G
        self._csr = None

    def get(self):
        if self._csr is None:
            G = self._G
            A = sp.csr_matrix((G._data_h, G._indices_h, G._indptr_h), shape=(G.n, G.n))
            M = (sp.diags(G._deg_h + G.sigma) - A).tocsr()
            M.sort_indices()
            self._csr = M
        return self._csr

    @property
    def shape(self):
        return (self._G.n, self._G.n)


class Graph:
    """Graph(n, edges, sigma, weights=None): realworld/polar_gpu.py:47-60.

    Attributes as in the reference: n, sigma, M0 (host CSR via .get()), dmax, m, edges,
    weights; plus the device CSR used by the kernels."""

    def __init__(self, n, edges, sigma, weights=None, *, heavy_thresh=256, device=None):
        self.n = int(n)
        self.sigma = float(sigma)
        self.device = default_device() if device is None else torch.device(device)
        edges = np.asarray(edges, dtype=np.int64).reshape(-1, 2)
        u, v = edges[:, 0], edges[:, 1]
        if len(u) and (u.min() < 0 or v.min() < 0 or max(u.max(), v.max()) >= self.n):
            raise ValueError("edge endpoint out of range")
        w = np.ones(len(u)) if weights is None else np.asarray(weights, np.float64)
        if len(w) != len(u):
            raise ValueError("weights must match edges")
        deg = np.bincount(u, w, self.n) + np.bincount(v, w, self.n)
        self.dmax = float(deg.max()) if self.n else 0.0
        self.m = len(u)
        self.edges = edges
        self.weights = w
        self.M0 = _HostM0(self)
        self._deg_h = deg
        dev = self.device
        self._ind_h = self._dat_h = None
        csr = None
        if weights is None and dev.type == "cuda" and 0 < 2 * len(u) < 2 ** 31:
            # ingestion on the device; repeated edges (merged weights) take the host path
            csr = csr_from_edges(self.n, torch.as_tensor(u).to(dev), torch.as_tensor(v).to(dev))
            if bool((csr[2] > 1).any()):
                csr = None
        if csr is not None:
            self.indptr, self.indices = csr[0], csr[1]
            self._indptr_h = self.indptr.cpu().numpy()
            self.nnz = int(self.indices.numel())
            self.weighted = False
        else:
            A = sp.csr_matrix((np.r_[w, w], (np.r_[u, v], np.r_[v, u])), shape=(self.n, self.n))
            A.sum_duplicates()
            A.sort_indices()
            if A.nnz >= 2 ** 31:
                raise ValueError("graph too large for int32 CSR")
            self._indptr_h = A.indptr.astype(np.int32)
            self._ind_h = A.indices.astype(np.int32)
            self._dat_h = A.data
            self.nnz = int(A.nnz)
            self.weighted = weights is not None and not np.all(self._dat_h == 1.0)
            self.indptr = _i32(self._indptr_h, dev)
            self.indices = _i32(self._ind_h, dev)
        if self.weighted:
            self.wts = torch.as_tensor(self._data_h, dtype=torch.float64).to(dev)
            self.diag = torch.as_tensor(deg + self.sigma, dtype=torch.float64).to(dev)
        else:
            self.wts = None
            self.diag = None
        self._split_heavy(int(heavy_thresh))

    @property
    def _indices_h(self):
        """Host copy of the neighbour indices (read back once when built on the device)."""
        if self._ind_h is None:
            self._ind_h = self.indices.cpu().numpy()
        return self._ind_h

    @property
    def _data_h(self):
        """Host CSR values (unit weights when built on the device)."""
        if self._dat_h is None:
            self._dat_h = np.ones(self.nnz)
        return self._dat_h

    # -- heavy-row split ---------------------------------------------------------------
    CHUNK = 256  # neighbours per heavy-row chunk (one warp per chunk in the solver)

    def _split_heavy(self, thresh):
        """Default partition (threshold `thresh`) plus a cache of partitions for other
        thresholds: rows with more than `thresh` neighbours are cut into chunks of at most
        CHUNK (the kernels' kChunkMax), combined in chunk order by the kernels."""
        self.heavy_thresh = max(1, thresh)
        self._heavy = {}
        hv = self._heavy_parts(self.heavy_thresh)
        self.nheavy, self.nchunks = hv["nheavy"], hv["nchunks"]
        self.hrow, self.hchunk_off = hv["hrow"], hv["hchunk_off"]
        self.chunk_row, self.chunk_lo, self.chunk_hi = hv["chunk_row"], hv["chunk_lo"], hv["chunk_hi"]
        self.rowblk_h, self.nrb, self.rowblk = hv["rowblk_h"], hv["nrb"], hv["rowblk"]

    def _heavy_parts(self, thresh):
        if thresh in self._heavy:
            return self._heavy[thresh]
        ch = self.CHUNK
        degs = np.diff(self._indptr_h.astype(np.int64))
        hrow = np.flatnonzero(degs > thresh).astype(np.int32)
        nch = -(-degs[hrow] // ch) if len(hrow) else np.zeros(0, np.int64)
        off = np.zeros(len(hrow) + 1, np.int64)
        off[1:] = np.cumsum(nch)
        total = int(off[-1])
        chunk_row = np.repeat(np.arange(len(hrow), dtype=np.int32), nch)
        within = np.arange(total, dtype=np.int64) - np.repeat(off[:-1], nch)
        lo = self._indptr_h[hrow].astype(np.int64)
        hi = self._indptr_h[hrow + 1].astype(np.int64) if len(hrow) else np.zeros(0, np.int64)
        c_lo = np.repeat(lo, nch) + within * ch
        c_hi = np.minimum(c_lo + ch, np.repeat(hi, nch))
        dev = self.device
        one = np.zeros(1, np.int32)
        rb = row_blocks(self._indptr_h, thresh)
        hv = dict(thresh=thresh, nheavy=len(hrow), nchunks=total, rowblk_h=rb, nrb=len(rb),
                  rowblk=_i32(rb.ravel() if len(rb) else np.zeros(2, np.int32), dev),
                  hrow=_i32(hrow if len(hrow) else one, dev), hchunk_off=_i32(off, dev),
                  chunk_row=_i32(chunk_row if total else one, dev), chunk_lo=_i32(c_lo if total else one, dev),
                  chunk_hi=_i32(c_hi if total else one, dev))
        self._heavy[thresh] = hv
        return hv

    def Lam(self, k):
        """Spectral upper bound sigma + 2 dmax + 4k (realworld/polar_gpu.py:59-60)."""
        return self.sigma + 2.0 * self.dmax + 4.0 * k

    def _sell(self, thresh, S):
        key = (thresh, S)
        if not hasattr(self, "_sell_cache"):
            self._sell_cache = {}
        if key not in self._sell_cache:
            dev = self.device
            if dev.type == "cuda":
                ip = self.indptr.to(torch.int64)
                off, rows, sidx = sell_slices_torch(self.indptr, self.indices, (ip[1:] - ip[:-1]) <= thresh, S)
                one = torch.zeros(1, dtype=torch.int32, device=dev)
                self._sell_cache[key] = dict(ns=off.numel() - 1, off=off, rows=rows if rows.numel() else one,
                                             idx=sidx if sidx.numel() else one)
            else:
                degs = np.diff(self._indptr_h.astype(np.int64))
                off, rows, sidx = sell_slices(self._indptr_h, self._indices_h, degs <= thresh, S)
                self._sell_cache[key] = dict(ns=len(off) - 1, off=_i32(off, dev),
                                             rows=_i32(rows if len(rows) else np.zeros(1, np.int32), dev),
                                             idx=_i32(sidx if len(sidx) else np.zeros(1, np.int32), dev))
        return self._sell_cache[key]

    def struct(self, extra=None, heavy_thresh=None, sell_rows=0):
        """ctypes polar_graph for this graph (plus an Op's added edges), with the heavy-row
        partition for `heavy_thresh` (default: the graph's own threshold) and, when
        sell_rows > 0 (unweighted graphs), the sliced-ELL layout of the light rows for
        warps of sell_rows rows."""
        hv = self._heavy_parts(self.heavy_thresh if heavy_thresh is None else int(heavy_thresh))
        s = _lib.PolarGraph()
        s.nsl = 0
        s.sell_s = 0
        if sell_rows and not self.weighted:
            sl = self._sell(hv["thresh"], int(sell_rows))
            s.nsl = sl["ns"]
            s.sell_s = int(sell_rows)
            s.d_sl_off = sl["off"].data_ptr()
            s.d_sl_rows = sl["rows"].data_ptr()
            s.d_sl_idx = sl["idx"].data_ptr()
        s.n = self.n
        s.nnz = self.nnz
        s.d_indptr = self.indptr.data_ptr()
        s.d_indices = self.indices.data_ptr() if self.nnz else self.indptr.data_ptr()
        s.d_wts = self.wts.data_ptr() if self.weighted else None
        s.d_diag = self.diag.data_ptr() if self.weighted else None
        s.sigma = self.sigma
        s.nx = 0
        s.heavy_thresh = hv["thresh"]
        s.nheavy = hv["nheavy"]
        s.nchunks = hv["nchunks"]
        s.d_hrow = hv["hrow"].data_ptr()
        s.d_hchunk_off = hv["hchunk_off"].data_ptr()
        s.d_chunk_row = hv["chunk_row"].data_ptr()
        s.d_chunk_lo = hv["chunk_lo"].data_ptr()
        s.d_chunk_hi = hv["chunk_hi"].data_ptr()
        s.nrb = hv["nrb"]
        s.d_rowblk = hv["rowblk"].data_ptr()
        if extra is not None:
            extra.fill(s)
        return s


class _Added:
    """Edges added during the greedy (Op.add), as the side structure the kernels read."""

    def __init__(self, G):
        self.G = G
        self.nbr = {}       # row -> list of (neighbour, weight)
        self.bits_h = np.zeros((G.n + 31) // 32, dtype=np.uint32)
        self.bits_d = torch.zeros(len(self.bits_h), dtype=torch.int32, device=G.device)
        self.dirty = False
        self.weighted = False
        self.rows_d = self.off_d = self.nbr_d = self.wt_d = None

    def add(self, a, b, w):
        for x, y in ((a, b), (b, a)):
            self.nbr.setdefault(x, []).append((y, w))
        if w != 1.0:
            self.weighted = True
        words = sorted({a >> 5, b >> 5})
        for r in (a, b):
            self.bits_h[r >> 5] |= np.uint32(1 << (r & 31))
        idx = torch.as_tensor(np.array(words, dtype=np.int64), device=self.G.device)
        vals = torch.as_tensor(self.bits_h[words].view(np.int32).copy(), device=self.G.device)
        self.bits_d.index_copy_(0, idx, vals)
        self.dirty = True

    def _upload(self):
        rows = np.array(sorted(self.nbr), dtype=np.int32)
        off = np.zeros(len(rows) + 1, dtype=np.int32)
        off[1:] = np.cumsum([len(self.nbr[r]) for r in rows])
        nb = np.array([x for r in rows for x, _ in self.nbr[r]], dtype=np.int32)
        wt = np.array([w for r in rows for _, w in self.nbr[r]], dtype=np.float64)
        dev = self.G.device
        self.rows_d = _i32(rows, dev)
        self.off_d = _i32(off, dev)
        self.nbr_d = _i32(nb, dev)
        self.wt_d = torch.as_tensor(wt).to(dev) if self.weighted else None
        self.dirty = False

    def fill(self, s):
        if not self.nbr:
            return
        if self.dirty:
            self._upload()
        s.nx = len(self.nbr)
        s.d_xbits = self.bits_d.data_ptr()
        s.d_xrow = self.rows_d.data_ptr()
        s.d_xoff = self.off_d.data_ptr()
        s.d_xnbr = self.nbr_d.data_ptr()
        s.d_xwt = self.wt_d.data_ptr() if self.wt_d is not None else None


class Op:
    """y = (M0 + sum_S w b b^T + shift I) x  (realworld/polar_gpu.py:63-80)."""

    def __init__(self, G):
        self.G = G
        self.M0 = G.M0
        self.A = []
        self.B = []
        self._added = _Added(G)
        self._scratch = {}

    def add(self, a, b, w=1.0):
        a, b = int(a), int(b)
        if a == b or not (0 <= a < self.G.n and 0 <= b < self.G.n):
            raise ValueError("added edge must join two distinct vertices")
        self.A.append(a)
        self.B.append(b)
        self._added.add(a, b, float(w))

    def struct(self, heavy_thresh=None, sell_rows=0):
        return self.G.struct(self._added, heavy_thresh=heavy_thresh, sell_rows=sell_rows)

    def __call__(self, x, shift=0.0):
        """Apply to an (n, R) or (n,) float64/float32 CUDA tensor; returns a new tensor."""
        squeeze = x.dim() == 1
        X = x.reshape(self.G.n, -1)
        if X.dtype not in (torch.float64, torch.float32):
            raise TypeError("x must be float64 or float32")
        if not X.is_cuda:
            raise TypeError("x must be a CUDA tensor")
        X = X.contiguous()
        R = X.shape[1]
        prec = _lib.POLAR_MIXED if X.dtype == torch.float32 else _lib.POLAR_FP64
        maxc = 128 if prec == _lib.POLAR_MIXED else 64
        Y = torch.empty_like(X)
        lib = _lib.load()
        stream = torch.cuda.current_stream(X.device).cuda_stream
        g = self.struct()
        key = (prec, X.device.index)
        if key not in self._scratch:
            nb = lib.polar_spmm_scratch_bytes(g, prec, maxc)
            buf = torch.empty(max(nb, 256), dtype=torch.uint8, device=X.device)
            _lib.check(lib.polar_spmm_scratch_init(g, prec, maxc, buf.data_ptr(), stream), "spmm scratch")
            self._scratch[key] = buf
        scratch = self._scratch[key]
        for lo in range(0, R, maxc):
            hi = min(R, lo + maxc)
            xs = X[:, lo:hi]
            ys = Y[:, lo:hi]
            # unweighted graphs: the sliced-ELL layout of the solver for this width (the
            # library uses it when the width is a power of two)
            gw = self.struct(sell_rows=lib.polar_sell_rows(prec, hi - lo)) if not self.G.weighted else g
            _lib.check(lib.polar_spmm(gw, prec, hi - lo, float(shift), xs.data_ptr(), R, ys.data_ptr(), R,
                                      scratch.data_ptr(), stream), "polar_spmm")
        return Y.reshape(-1) if squeeze else Y
