// Row-group CSR-Laplacian SpMM building blocks (sm_100a).
//
// X is read with ordinary (coherent) loads and never through a const __restrict__
// pointer: inside the persistent solver X is rewritten by other CTAs between grid
// barriers, and the non-coherent read-only path could return stale rows.
//
// A "row group" is G consecutive lanes of a warp that together own one matrix row and
// all ld = G*VEC columns of the dense block; lane g holds columns [g*VEC, g*VEC+VEC).
// Neighbour indices are read cooperatively (G per step, coalesced) and broadcast with
// shuffles; each neighbour row of X is one VEC-wide vector load per lane.
//
// Operator (realworld/polar_gpu.py:47-80): y_i = (deg_i + sigma + shift) x_i
//   - sum_{j in N(i)} w_ij x_j + sum_{added (i,k)} w_ik (x_i - x_k).
#pragma once
#include "common.cuh"

#ifndef POLAR_PANEL_BYTES
#define POLAR_PANEL_BYTES 512  // column panel of the SpMM (bytes of one row's panel)
#endif

namespace polar {

constexpr int kChunkMax = 256;  // neighbours per heavy-row chunk (the graph partition's CHUNK)

template <typename T> struct AccOf;
template <> struct AccOf<float> { using type = float; };
template <> struct AccOf<double> { using type = double; };

struct RowGroup {
  int G;         // lanes per row (power of two, <= 32)
  int lg;        // lane index inside the group
  unsigned mask; // lanes of this group
  int col;       // first column owned by this lane
};

template <int VEC>
POLAR_D RowGroup make_row_group(int ld) {
  RowGroup r;
  r.G = ld / VEC;
  const int lane = threadIdx.x & 31;
  r.lg = lane & (r.G - 1);
  const int base = lane - r.lg;
  r.mask = (r.G == 32) ? 0xffffffffu : (((1u << r.G) - 1u) << base);
  r.col = r.lg * VEC;
  return r;
}

// acc[v] += sum_{k in [lo,hi)} w_k * X[idx_k][col+v]
// Lanes with on == false (all their columns converged) still take part in the index
// shuffles but issue no loads.  Groups of 4+ lanes read a batch of G indices
// cooperatively and broadcast them by shuffles; narrower groups read the next 4 indices
// directly (the same addresses for the group's lanes, served by L1) so 4 gathers are in
// flight per lane.
template <typename T, int VEC, bool WEIGHTED, typename AA = typename AccOf<T>::type>
POLAR_D void gather_rows(const polar_graph& g, const RowGroup& rg, int lo, int hi, const T* X,
                         int ld, AA (&acc)[VEC], bool on = true) {
  using A = AA;
  if (rg.G < 4) {
    if (!on) return;
    int k = lo;
    for (; k + 4 <= hi; k += 4) {
      int jj[4];
      A ww[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        jj[u] = __ldg(g.d_indices + k + u);
        ww[u] = WEIGHTED ? (A)__ldg(g.d_wts + k + u) : A(1);
      }
      T xv[4][VEC];
#pragma unroll
      for (int u = 0; u < 4; ++u) vload<T, VEC>(xv[u], X + (size_t)jj[u] * ld + rg.col);
#pragma unroll
      for (int u = 0; u < 4; ++u)
#pragma unroll
        for (int v = 0; v < VEC; ++v) acc[v] = WEIGHTED ? fma(ww[u], (A)xv[u][v], acc[v]) : acc[v] + (A)xv[u][v];
    }
    for (; k < hi; ++k) {
      const int jj = __ldg(g.d_indices + k);
      const A ww = WEIGHTED ? (A)__ldg(g.d_wts + k) : A(1);
      T xv[VEC];
      vload<T, VEC>(xv, X + (size_t)jj * ld + rg.col);
#pragma unroll
      for (int v = 0; v < VEC; ++v) acc[v] = WEIGHTED ? fma(ww, (A)xv[v], acc[v]) : acc[v] + (A)xv[v];
    }
    return;
  }
  for (int k0 = lo; k0 < hi; k0 += rg.G) {
    const int k = k0 + rg.lg;
    int j = 0;
    A w = A(1);
    if (k < hi) {
      j = __ldg(g.d_indices + k);
      if (WEIGHTED) w = (A)__ldg(g.d_wts + k);
    }
    const int cnt = min(rg.G, hi - k0);
    int t = 0;
    for (; t + 4 <= cnt; t += 4) {
      int jj[4];
      A ww[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        jj[u] = __shfl_sync(rg.mask, j, t + u, rg.G);
        ww[u] = WEIGHTED ? __shfl_sync(rg.mask, w, t + u, rg.G) : A(1);
      }
      if (on) {
        T xv[4][VEC];
#pragma unroll
        for (int u = 0; u < 4; ++u) vload<T, VEC>(xv[u], X + (size_t)jj[u] * ld + rg.col);
#pragma unroll
        for (int u = 0; u < 4; ++u)
#pragma unroll
          for (int v = 0; v < VEC; ++v) acc[v] = WEIGHTED ? fma(ww[u], (A)xv[u][v], acc[v]) : acc[v] + (A)xv[u][v];
      }
    }
    for (; t < cnt; ++t) {
      const int jj = __shfl_sync(rg.mask, j, t, rg.G);
      const A ww = WEIGHTED ? __shfl_sync(rg.mask, w, t, rg.G) : A(1);
      if (on) {
        T xv[VEC];
        vload<T, VEC>(xv, X + (size_t)jj * ld + rg.col);
#pragma unroll
        for (int v = 0; v < VEC; ++v) acc[v] = WEIGHTED ? fma(ww, (A)xv[v], acc[v]) : acc[v] + (A)xv[v];
      }
    }
  }
}

// Added-edge contribution for row i: acc += sum w x_k, returns sum w (to add to diag).
template <typename T, int VEC, typename AA = typename AccOf<T>::type>
POLAR_D double added_terms(const polar_graph& g, const RowGroup& rg, int i, const T* X, int ld,
                           AA (&acc)[VEC], bool on = true) {
  using A = AA;
  if (g.nx == 0 || !on) return 0.0;
  const uint32_t bits = __ldg(g.d_xbits + (i >> 5));
  if (!((bits >> (i & 31)) & 1u)) return 0.0;
  int lo = 0, hi = g.nx - 1;
  while (lo < hi) {  // first xrow >= i
    const int mid = (lo + hi) >> 1;
    if (__ldg(g.d_xrow + mid) < i) lo = mid + 1; else hi = mid;
  }
  double wsum = 0.0;
  const int b = __ldg(g.d_xoff + lo), e = __ldg(g.d_xoff + lo + 1);
  for (int k = b; k < e; ++k) {
    const int j = __ldg(g.d_xnbr + k);
    const double w = g.d_xwt ? __ldg(g.d_xwt + k) : 1.0;
    T xv[VEC];
    vload<T, VEC>(xv, X + (size_t)j * ld + rg.col);
#pragma unroll
    for (int v = 0; v < VEC; ++v) acc[v] = fma((A)w, (A)xv[v], acc[v]);
    wsum += w;
  }
  return wsum;
}

// Finishes row i from its own entries xi (already loaded): y = (diag + shift) x_i - acc.
// ADD = false leaves out the added edges (the caller applies them afterwards).
template <typename T, int VEC, bool ADD = true, typename AA = typename AccOf<T>::type>
POLAR_D void finish_row_pre(const polar_graph& g, const RowGroup& rg, int i, int deg, double shift, const T* X,
                            int ld, AA (&acc)[VEC], T* Y, int ldy, const T (&xi)[VEC],
                            T (&yi)[VEC], bool store = true) {
  using A = AA;
  if (!store) {
#pragma unroll
    for (int v = 0; v < VEC; ++v) yi[v] = T(0);
    return;
  }
  double wadd = 0.0;
  if constexpr (ADD) wadd = added_terms<T, VEC, AA>(g, rg, i, X, ld, acc);
  const double dg = (g.d_diag ? __ldg(g.d_diag + i) : (double)deg + g.sigma) + wadd + shift;
#pragma unroll
  for (int v = 0; v < VEC; ++v) yi[v] = (T)fma((A)dg, (A)xi[v], -acc[v]);
  vstore<T, VEC>(Y + (size_t)i * ldy + rg.col, yi);
}

// Finishes row i: y = (diag + shift) x_i - acc.  Returns x_i in xi (for d^T v).
template <typename T, int VEC, bool ADD = true, typename AA = typename AccOf<T>::type>
POLAR_D void finish_row(const polar_graph& g, const RowGroup& rg, int i, int deg, double shift,
                        const T* X, int ld, AA (&acc)[VEC], T* Y,
                        int ldy, T (&xi)[VEC], T (&yi)[VEC], bool store = true) {
  using A = AA;
  if (!store) {  // lane idle: nothing to compute
#pragma unroll
    for (int v = 0; v < VEC; ++v) xi[v] = yi[v] = T(0);
    return;
  }
  double wadd = 0.0;
  if constexpr (ADD) wadd = added_terms<T, VEC, AA>(g, rg, i, X, ld, acc);
  const double dg = (g.d_diag ? __ldg(g.d_diag + i) : (double)deg + g.sigma) + wadd + shift;
  vload<T, VEC>(xi, X + (size_t)i * ld + rg.col);
#pragma unroll
  for (int v = 0; v < VEC; ++v) yi[v] = (T)fma((A)dg, (A)xi[v], -acc[v]);
  if (store) vstore<T, VEC>(Y + (size_t)i * ldy + rg.col, yi);
}

// ---------------------------------------------------------------------------------------
// CSR stream over one row block [r0, r1) of light rows: the row group walks the block's
// nonzeros in batches of G, with the next index batch in flight, issues the G neighbour
// gathers of a batch before consuming any, and closes rows as the stream crosses their
// ends (empty rows included).  G <= 32.  With DOT, dacc += x_i . y_i per column.
template <typename T, int VEC, bool WEIGHTED, bool DOT>
POLAR_D void stream_block(const polar_graph& g, const RowGroup& rg, int r0, int r1, const T* X, int ld, T* Y,
                          int ldy, double shift, bool on, double (&dacc)[VEC]) {
  using A = typename AccOf<T>::type;
  const int G = rg.G;
  const int kend = __ldg(g.d_indptr + r1);
  int row = r0;
  int rowbeg = __ldg(g.d_indptr + r0);
  int rowend = __ldg(g.d_indptr + r0 + 1);
  const int kbeg = rowbeg;
  T xi[VEC];
  if (on) vload<T, VEC>(xi, X + (size_t)row * ld + rg.col);
  A acc[VEC];
#pragma unroll
  for (int v = 0; v < VEC; ++v) acc[v] = A(0);
  auto close_row = [&]() {
    if (on) {
      const double wadd = added_terms<T, VEC>(g, rg, row, X, ld, acc);
      const double dg = (g.d_diag ? __ldg(g.d_diag + row) : (double)(rowend - rowbeg) + g.sigma) + wadd + shift;
      T yi[VEC];
#pragma unroll
      for (int v = 0; v < VEC; ++v) yi[v] = (T)fma((A)dg, (A)xi[v], -acc[v]);
      vstore<T, VEC>(Y + (size_t)row * ldy + rg.col, yi);
      if (DOT)
#pragma unroll
        for (int v = 0; v < VEC; ++v) dacc[v] += (double)xi[v] * (double)yi[v];
    }
#pragma unroll
    for (int v = 0; v < VEC; ++v) acc[v] = A(0);
    ++row;
    if (row < r1) {
      rowbeg = rowend;
      rowend = __ldg(g.d_indptr + row + 1);
      if (on) vload<T, VEC>(xi, X + (size_t)row * ld + rg.col);
    }
  };
  int jc = 0, jn = 0;
  A wc = A(1), wn = A(1);
  {
    const int k = kbeg + rg.lg;
    if (k < kend) {
      jc = __ldg(g.d_indices + k);
      if (WEIGHTED) wc = (A)__ldg(g.d_wts + k);
    }
    const int k2 = k + G;
    if (k2 < kend) {
      jn = __ldg(g.d_indices + k2);
      if (WEIGHTED) wn = (A)__ldg(g.d_wts + k2);
    }
  }
  for (int kb = kbeg; kb < kend; kb += G) {
    const int cnt = min(G, kend - kb);
    const int jb = jc;
    const A wb = wc;
    jc = jn;
    wc = wn;
    {
      const int k3 = kb + 2 * G + rg.lg;
      jn = 0;
      if (k3 < kend) {
        jn = __ldg(g.d_indices + k3);
        if (WEIGHTED) wn = (A)__ldg(g.d_wts + k3);
      }
    }
    for (int s0 = 0; s0 < cnt; s0 += 8) {
      T xv[8][VEC];
      A ww[8];
#pragma unroll
      for (int u = 0; u < 8; ++u) {
        if (s0 + u < cnt) {
          const int j = __shfl_sync(rg.mask, jb, s0 + u, G);
          ww[u] = WEIGHTED ? __shfl_sync(rg.mask, wb, s0 + u, G) : A(1);
          if (on) vload<T, VEC>(xv[u], X + (size_t)j * ld + rg.col);
        }
      }
#pragma unroll
      for (int u = 0; u < 8; ++u) {
        if (s0 + u < cnt) {
          const int k = kb + s0 + u;
          while (k >= rowend) close_row();
          if (on)
#pragma unroll
            for (int v = 0; v < VEC; ++v)
              acc[v] = WEIGHTED ? fma(ww[u], (A)xv[u][v], acc[v]) : acc[v] + (A)xv[u][v];
        }
      }
    }
  }
  while (row < r1) close_row();
}

// ---------------------------------------------------------------------------------------
// P1: v = (M + shift I) d, processed in 128-byte column panels (32 FP32 / 16 FP64
// columns).  One pass over the CSR per panel keeps the gathered panel of d (n x 128 B)
// resident in L2.  Row groups of G = panel/VEC lanes; a warp owns 32/G consecutive rows at
// a time (independent gather chains).  Per-warp column sums of d.v accumulate in shared
// memory (red[warp][c]) in a fixed order.
template <typename T, int VEC, bool WEIGHTED, bool DOT>
POLAR_D void spmm_phase(const polar_graph& g, int ld, double shift, const T* X, T* Y, int ldy,
                        typename AccOf<T>::type* chunk_part, int* hcount, double* red, const int* act,
                        int vb = -1, int vnb = -1) {
  // (vb, vnb): this CTA's index among the CTAs sharing the work, and their count
  // (default: blockIdx.x of gridDim.x)
  using A = typename AccOf<T>::type;
  constexpr int PANEL = POLAR_PANEL_BYTES / sizeof(T);
  const int pw = ld < PANEL ? ld : PANEL;
  const int npanel = ld / pw;
  RowGroup rg;
  rg.G = pw / VEC;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  rg.lg = lane & (rg.G - 1);
  const int gbase = lane - rg.lg;
  rg.mask = (rg.G == 32) ? 0xffffffffu : (((1u << rg.G) - 1u) << gbase);
  const int gpw = 32 / rg.G;
  const int grp = lane / rg.G;
  const int wpb = blockDim.x >> 5;
  const int gwarp = (vb < 0 ? (int)blockIdx.x : vb) * wpb + warp;
  const int nwarps = (vnb < 0 ? (int)gridDim.x : vnb) * wpb;
  const int gid = gwarp * gpw + grp;
  const int GT = nwarps * gpw;
  if (DOT) {
    for (int c = lane; c < ld; c += 32) red[warp * ld + c] = 0.0;
    __syncwarp();
  }
  for (int pnl = 0; pnl < npanel; ++pnl) {
    rg.col = pnl * pw + rg.lg * VEC;
    bool on = act == nullptr;
    if (act)
#pragma unroll
      for (int v = 0; v < VEC; ++v) on |= act[rg.col + v] != 0;
    double dacc[VEC];
#pragma unroll
    for (int v = 0; v < VEC; ++v) dacc[v] = 0.0;
    // Heavy rows: each chunk adds its own share of d_i . v_i (-d_i . partial; the first
    // chunk also the diagonal and added-edge terms).  Chunk -> row group is fixed, so the
    // dot product does not depend on which group finishes the row.
    for (int ch = gid; ch < g.nchunks; ch += GT) {
      const int h = __ldg(g.d_chunk_row + ch);
      const int lo = __ldg(g.d_chunk_lo + ch), hi = __ldg(g.d_chunk_hi + ch);
      const int i = __ldg(g.d_hrow + h);
      const int c0 = __ldg(g.d_hchunk_off + h), c1 = __ldg(g.d_hchunk_off + h + 1);
      A acc[VEC];
#pragma unroll
      for (int v = 0; v < VEC; ++v) acc[v] = A(0);
      gather_rows<T, VEC, WEIGHTED>(g, rg, lo, hi, X, ld, acc, on);
      T xi[VEC];
      if (on) {
        vstore<A, VEC>(chunk_part + (size_t)ch * ld + rg.col, acc);
        vload<T, VEC>(xi, X + (size_t)i * ld + rg.col);
        if (DOT)
#pragma unroll
          for (int v = 0; v < VEC; ++v) dacc[v] -= (double)xi[v] * (double)acc[v];
      }
      if (DOT && ch == c0 && on) {
        A ex[VEC];
#pragma unroll
        for (int v = 0; v < VEC; ++v) ex[v] = A(0);
        const double wadd = added_terms<T, VEC>(g, rg, i, X, ld, ex);
        const int deg = __ldg(g.d_indptr + i + 1) - __ldg(g.d_indptr + i);
        const double dg = (g.d_diag ? __ldg(g.d_diag + i) : (double)deg + g.sigma) + wadd + shift;
#pragma unroll
        for (int v = 0; v < VEC; ++v) dacc[v] += (double)xi[v] * (dg * (double)xi[v] - (double)ex[v]);
      }
      __threadfence();
      __syncwarp(rg.mask);
      int* cnt = hcount + (size_t)h * npanel + pnl;
      int old = 0;
      if (rg.lg == 0) old = atomicAdd(cnt, 1);
      old = __shfl_sync(rg.mask, old, 0, rg.G);
      if (old == c1 - c0 - 1) {
        __threadfence();
        A sum[VEC];
#pragma unroll
        for (int v = 0; v < VEC; ++v) sum[v] = A(0);
        if (on) {
          for (int c2 = c0; c2 < c1; ++c2) {
            A pv[VEC];
            vload_cg<A, VEC>(pv, chunk_part + (size_t)c2 * ld + rg.col);
#pragma unroll
            for (int v = 0; v < VEC; ++v) sum[v] += pv[v];
          }
        }
        const int deg = __ldg(g.d_indptr + i + 1) - __ldg(g.d_indptr + i);
        T xf[VEC], yi[VEC];
        finish_row<T, VEC>(g, rg, i, deg, shift, X, ld, sum, Y, ldy, xf, yi, on);
        if (rg.lg == 0) *cnt = 0;
      }
    }
    // light rows: CSR stream over row blocks
    for (int b = gid; b < g.nrb; b += GT)
      stream_block<T, VEC, WEIGHTED, DOT>(g, rg, __ldg(g.d_rowblk + 2 * b), __ldg(g.d_rowblk + 2 * b + 1), X, ld, Y,
                                          ldy, shift, on, dacc);
    if (DOT) {
      for (int o = rg.G; o < 32; o <<= 1)
#pragma unroll
        for (int v = 0; v < VEC; ++v) dacc[v] += __shfl_xor_sync(0xffffffffu, dacc[v], o);
      if (lane < rg.G)
#pragma unroll
        for (int v = 0; v < VEC; ++v) red[warp * ld + rg.col + v] += dacc[v];
      __syncwarp();
    }
  }
}


}  // namespace polar
