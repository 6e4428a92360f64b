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

namespace polar {

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
// shuffles but issue no loads.
template <typename T, int VEC, bool WEIGHTED>
POLAR_D void gather_rows(const polar_graph& g, const RowGroup& rg, int lo, int hi, const T* X,
                         int ld, typename AccOf<T>::type (&acc)[VEC], bool on = true) {
  using A = typename AccOf<T>::type;
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
template <typename T, int VEC>
POLAR_D double added_terms(const polar_graph& g, const RowGroup& rg, int i, const T* X, int ld,
                           typename AccOf<T>::type (&acc)[VEC], bool on = true) {
  using A = typename AccOf<T>::type;
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

// Finishes row i: y = (diag + shift) x_i - acc.  Returns x_i in xi (for d^T v).
template <typename T, int VEC>
POLAR_D void finish_row(const polar_graph& g, const RowGroup& rg, int i, int deg, double shift,
                        const T* X, int ld, typename AccOf<T>::type (&acc)[VEC], T* Y,
                        int ldy, T (&xi)[VEC], T (&yi)[VEC], bool store = true) {
  using A = typename AccOf<T>::type;
  if (!store) {  // lane idle: nothing to compute
#pragma unroll
    for (int v = 0; v < VEC; ++v) xi[v] = yi[v] = T(0);
    return;
  }
  const double wadd = added_terms<T, VEC>(g, rg, i, X, ld, acc);
  const double dg = (g.d_diag ? __ldg(g.d_diag + i) : (double)deg + g.sigma) + wadd + shift;
  vload<T, VEC>(xi, X + (size_t)i * ld + rg.col);
#pragma unroll
  for (int v = 0; v < VEC; ++v) yi[v] = (T)fma((A)dg, (A)xi[v], -acc[v]);
  if (store) vstore<T, VEC>(Y + (size_t)i * ldy + rg.col, yi);
}

}  // namespace polar
