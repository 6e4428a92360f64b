// Multi-kernel multi-shift CG (sm_100a): one high-occupancy kernel per phase; the host
// queues M iterations plus the deferred shifted update, then checks convergence once.
//
// Per iteration (realworld/polar_gpu.py:100-125):
//   mk_spmm   v = (M + tau_0 I) d, partial d.v per CTA; the last CTA to finish reduces
//             the partials in a fixed order and writes a = rr / d.v
//   mk_resid  r <- r - a v, r on the active rows -> history slot, partial r.r; the last
//             CTA computes beta, chi and convergence for every column
//   mk_dir    zeta recurrences / tracker / freezing for all (pole, column) items and the
//             step coefficients; d <- r + beta d
// and after M iterations (or convergence)
//   mk_flush  deferred shifted update of X and P from the history (final pass writes
//             the output block)
// Kernels take SolvePrm by value in the constant parameter space (__grid_constant__), so
// field reads are uniform constant loads that no store can alias.  Reductions are
// deterministic (fixed grids, fixed summation order).
#include <cuda_runtime.h>

#include <cstdlib>
#include <map>
#include <vector>
#include <mutex>
#include <thread>
#include <tuple>
#include <type_traits>

#include "common.cuh"
#include "graph_ops.cuh"
#include "host_util.h"
#include "msolve_mk.h"
#include "sell_spmm.cuh"
#include "solver_core.cuh"

namespace polar {

// ctl: [0] status [1] err [2] where [3] any [4] ran [5] nsteps [6] first
//      [7] cnt_init [8] cnt_spmm [9] cnt_resid [10] cnt_dir [11] cnt_flush
enum { C_STATUS = 0, C_ERR, C_WHERE, C_ANY, C_RAN, C_NSTEPS, C_FIRST, C_CNT0, C_CNT1, C_CNT3, C_CNT4, C_CNT5 };

POLAR_D bool last_cta(int* cnt) {
  __shared__ int s_last;
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) {
    const int t = atomicAdd(cnt, 1);
    s_last = (t == (int)gridDim.x - 1) ? 1 : 0;
    if (s_last) {
      *cnt = 0;
      __threadfence();
    }
  }
  __syncthreads();
  return s_last != 0;
}

constexpr size_t kFlushSmemMax = 200 * 1024;
// cp.async ring of the SpMM's slice pass per warp: stages x POLAR_SELL_BYTES x 32 lanes
constexpr int kSellRingWarp = POLAR_SELL_STAGES * POLAR_SELL_BYTES * 32;

POLAR_D bool solve_live(const int* ctl, const long long* stats, long long maxit) {
  return ld_volatile_i32(ctl + C_ANY) != 0 && stats[0] < maxit && ld_volatile_i32(ctl + C_ERR) == 0;
}

// ---- init: r = d = W, r.r --------------------------------------------------------------
template <typename T, int VEC>
__global__ void __launch_bounds__(kBlock) mk_init(const __grid_constant__ SolvePrm<T> P) {

  __shared__ double red[kWarps * kMaxLd];
  __shared__ double s_col[kMaxLd];
  const int ld = P.ld;
  const RowGroup rg = make_row_group<VEC>(ld);
  const long long tid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long nth = (long long)gridDim.x * blockDim.x;
  const long long nvec = (long long)P.n * rg.G;
  const int lgG = __ffs(rg.G) - 1;
  double acc[VEC];
#pragma unroll
  for (int v = 0; v < VEC; ++v) acc[v] = 0.0;
  for (long long e = tid; e < nvec; e += nth) {
    const long long i = e >> lgG;
    double wd[VEC];
#pragma unroll
    for (int v = 0; v < VEC; ++v) {
      const int c = rg.col + v;
      wd[v] = (c < P.R) ? __ldg(P.W + (size_t)i * P.ldw + c) : 0.0;
    }
    store_res<T, VEC>(P, wd, (size_t)i * ld + rg.col);
#pragma unroll
    for (int v = 0; v < VEC; ++v) acc[v] += wd[v] * wd[v];
    store_dir<T, VEC>(P, wd, (size_t)i * ld + rg.col);
  }
  reduce_cols_to_part<VEC>(acc, rg.G, ld, red, P.part + (size_t)blockIdx.x * ld);
  if (last_cta(P.ctl + C_CNT0)) {
    reduce_partials(P.part, gridDim.x, ld, red, s_col);
    const bool anyv = init_step(P, s_col);
    if (threadIdx.x == 0) {
      P.ctl[C_ANY] = anyv ? 1 : 0;
      P.ctl[C_RAN] = 0;
      P.ctl[C_NSTEPS] = 0;
      P.ctl[C_FIRST] = 1;
      P.stats[0] = 0;
      P.stats[1] = 0;
    }
  }
}

// ---- edges added by the greedy (Op.add): v += sum_S w b b^T d, d.v += d^T (that) ------------
// Run by the SpMM's last CTA after every row of v is final.  Thread item = (added-edge
// row, column); each row's change is its own term w (d_r - d_k) summed over its added
// neighbours in list order, and the d.v correction x_r (v_new - v_old) is summed per column
// over the rows in a fixed order in `tmp` (shared, kWarps * kMaxLd doubles).
template <typename T>
POLAR_D void apply_added_edges(const SolvePrm<T>& P, double* tmp, double* s_col) {
  const polar_graph& g = P.g;
  const int ld = P.ld;
  const int tile = (kWarps * kMaxLd) / ld;
  double colsum = 0.0;
  for (int r0 = 0; r0 < g.nx; r0 += tile) {
    const int nr = min(tile, g.nx - r0);
    __syncthreads();
    for (int q = threadIdx.x; q < nr * ld; q += blockDim.x) {
      const int rr = q / ld, c = q - rr * ld;
      const int ix = r0 + rr;
      const int r = __ldg(g.d_xrow + ix);
      const int b = __ldg(g.d_xoff + ix), e = __ldg(g.d_xoff + ix + 1);
      const double dr = (double)P.d[(size_t)r * ld + c];
      double delta = 0.0;
      for (int k = b; k < e; ++k) {
        const double w = g.d_xwt ? __ldg(g.d_xwt + k) : 1.0;
        delta += w * (dr - (double)P.d[(size_t)__ldg(g.d_xnbr + k) * ld + c]);
      }
      T* vp = P.v + (size_t)r * ld + c;
      const T vold = *vp;
      const T vnew = (T)((double)vold + delta);
      *vp = vnew;
      tmp[rr * ld + c] = dr * ((double)vnew - (double)vold);
    }
    __syncthreads();
    if (threadIdx.x < ld)
      for (int rr = 0; rr < nr; ++rr) colsum += tmp[rr * ld + threadIdx.x];
  }
  __syncthreads();
  if (threadIdx.x < ld) s_col[threadIdx.x] += colsum;
  __syncthreads();
}

// ---- v = (M + tau_0 I) d and d.v -------------------------------------------------------
#ifndef POLAR_SPMM_MINB
#define POLAR_SPMM_MINB 2  // resident 512-thread CTAs per SM requested for the SpMM kernel
#endif
// Bytes of gathered rows in flight per lane: the gather batch is this many bytes over the
// lane's share of a row (at least one neighbour).  Larger batches spill at 64 registers.
#ifndef POLAR_STREAM_U
#define POLAR_STREAM_U 4  // row items in flight per thread in the d update
#endif
#ifndef POLAR_RESID_U
#define POLAR_RESID_U 2   // same for the r update with FP64 vectors (more spills at 64 registers)
#endif
#ifndef POLAR_RESID_U32
#define POLAR_RESID_U32 1  // same with FP32 v: one item at a time was 6 % faster at n = 4.0M, R = 16
#endif
#ifndef POLAR_STREAM_MINB
#define POLAR_STREAM_MINB 2  // resident 512-thread CTAs per SM requested for the r and d updates
#endif
// SpMM accumulator: FP64 row sums for FP32 vectors unless POLAR_SPMM_ACC64 = 0.  A
// Laplacian row (deg + sigma + shift) x_i - sum_j x_j cancels heavily for smooth vectors, so
// the neighbour sum is kept unrounded until that final combination (one rounding per row
// instead of one per neighbour).  This bounds the mixed path's marginal error below 1e-6.
#ifndef POLAR_SPMM_ACC64
#define POLAR_SPMM_ACC64 1
#endif
template <typename T> struct SpmmAcc { using type = double; };
template <> struct SpmmAcc<float> { using type = std::conditional<POLAR_SPMM_ACC64 != 0, double, float>::type; };

// CPL: columns per lane (several 16-byte accesses when wider); row group = ld / CPL lanes.
// MODE 1: heavy chunks only (partials of d.v to part_h, no reduction); MODE 2: light rows
// by row groups (after a MODE 1 launch); MODE 3 (unweighted graphs with a sliced-ELL copy):
// heavy chunks and then the light rows' slices in one launch.  In modes 2 and 3 the last
// CTA reduces the partial arrays.  Separate instantiations give each path its own
// register budget.
template <typename T, int CPL, bool W, int MODE>
__global__ void __launch_bounds__(kBlock, POLAR_SPMM_MINB) mk_spmm(const __grid_constant__ SolvePrm<T> P) {

  pdl_wait();
  pdl_launch();
  if (!solve_live(P.ctl, P.stats, P.maxit)) return;
  using A = typename SpmmAcc<T>::type;
  A* const chunk_part = reinterpret_cast<A*>(P.chunk_part);
  __shared__ double red[kWarps * kMaxLd];
  __shared__ double s_col[kMaxLd];
  const polar_graph& g = P.g;
  const int ld = P.ld;
  const double shift = __ldg(P.tau);
  const RowGroup rg = make_row_group<CPL>(ld);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int gpw = 32 / rg.G;
  const int gid = (blockIdx.x * kWarps + warp) * gpw + lane / rg.G;
  const int GT = gridDim.x * kWarps * gpw;
  bool on = false;
#pragma unroll
  for (int v = 0; v < CPL; ++v) on |= P.act[rg.col + v] != 0;
  // heavy chunks then light-row slices (sell_spmm.cuh); MODE 3 accumulates d.v in the
  // warp's row of `red` (heavy chunks first, then slices)
  double* wred = red + warp * ld;
  if (MODE == 3) {
    for (int c = lane; c < ld; c += 32) wred[c] = 0.0;
    __syncwarp();
  }
  const GatherHints hp = make_gather_hints(P.l2_mode, P.hot_rows, P.d, (size_t)ld * sizeof(T), P.n);
  const int wid = blockIdx.x * kWarps + warp;
  const int nw = gridDim.x * kWarps;
  if (MODE == 1 || MODE == 3) {
    __shared__ int s_idx[kWarps][kChunkMax];
    double dacc[CPL];
#pragma unroll
    for (int v = 0; v < CPL; ++v) dacc[v] = 0.0;
    heavy_chunk_pass<T, CPL, W, A>(
        g, rg, wid, nw, P.d, ld, ld, on, s_idx[warp], chunk_part, P.hcount, hp,
        [&](int i, int cnt, auto& acc, auto& xi) {
          T yi[CPL];
          finish_row_pre<T, CPL, false, A>(g, rg, i, cnt, shift, P.d, ld, acc, P.v, ld, xi, yi, on);
          if (on)
#pragma unroll
            for (int v = 0; v < CPL; ++v) dacc[v] += (double)xi[v] * (double)yi[v];
        },
        [&](int i, bool first, auto& acc, auto& xi) {
          // each chunk adds its share of d_i . v_i; the first also the diagonal term
#pragma unroll
          for (int v = 0; v < CPL; ++v) dacc[v] -= (double)xi[v] * (double)acc[v];
          if (first) {
            const int deg = __ldg(g.d_indptr + i + 1) - __ldg(g.d_indptr + i);
            const double dg = (g.d_diag ? __ldg(g.d_diag + i) : (double)deg + g.sigma) + shift;
#pragma unroll
            for (int v = 0; v < CPL; ++v) dacc[v] += (double)xi[v] * (dg * (double)xi[v]);
          }
        },
        [&](int i, int deg, auto& sum) {
          T xf[CPL], yi[CPL];
          finish_row<T, CPL, false, A>(g, rg, i, deg, shift, P.d, ld, sum, P.v, ld, xf, yi, on);
        });
    if (MODE == 1) {
      // heavy-only launch: partial d.v per CTA, reduced by the light launch's last CTA
      reduce_cols_to_part<CPL>(dacc, rg.G, ld, red, P.part_h + (size_t)blockIdx.x * ld);
      return;
    }
    // MODE 3: fold the heavy rows' d.v into the warp's row (fixed xor pattern)
    for (int o = rg.G; o < 32; o <<= 1)
#pragma unroll
      for (int v = 0; v < CPL; ++v) dacc[v] += __shfl_xor_sync(0xffffffffu, dacc[v], o);
    if (lane < rg.G)
#pragma unroll
      for (int v = 0; v < CPL; ++v) wred[rg.col + v] += dacc[v];
    __syncwarp();
  }
  if (MODE == 3) {
    // light rows in sliced ELL.  The row's own entries are read after its gathers; d.v
    // leaves the registers: after each slice the products x_i y_i are summed over the
    // warp's rows per column in FP64 (fixed xor pattern) and added to the warp's row of red.
    constexpr int DC = CPL < 4 ? CPL : 4;  // columns per FP64 reduction pass
    auto row_end = [&](int row, int deg, auto& acc, auto& xi, bool go) {
      // y_i = (deg + sigma + shift) x_i - acc, formed in place in acc
      if (go) {
        const double dg = (double)deg + g.sigma + shift;
        T yv[CPL];
#pragma unroll
        for (int v = 0; v < CPL; ++v) yv[v] = (T)fma((A)dg, (A)xi[v], -acc[v]);
        vstore_hint<T, CPL>(P.v + (size_t)row * ld + rg.col, yv, hp.stream);
#pragma unroll
        for (int v = 0; v < CPL; ++v) acc[v] = (A)yv[v];
      }
#pragma unroll
      for (int v0 = 0; v0 < CPL; v0 += DC) {
        double pr[DC];
#pragma unroll
        for (int v = 0; v < DC; ++v) pr[v] = go ? (double)xi[v0 + v] * (double)acc[v0 + v] : 0.0;
        for (int o = rg.G; o < 32; o <<= 1)
#pragma unroll
          for (int v = 0; v < DC; ++v) pr[v] += __shfl_xor_sync(0xffffffffu, pr[v], o);
        if (lane < rg.G)
#pragma unroll
          for (int v = 0; v < DC; ++v) wred[rg.col + v0 + v] += pr[v];
      }
    };
    if constexpr (POLAR_SELL_ASYNC != 0 && (CPL * sizeof(T)) % 16 == 0) {
      extern __shared__ __align__(16) unsigned char spmm_ring[];
      sell_slice_pass_async<T, CPL, A>(g, rg, wid, nw, P.d, ld, on, hp, spmm_ring + (size_t)warp * kSellRingWarp,
                                       row_end);
    } else {
      sell_slice_pass<T, CPL, A>(g, rg, wid, nw, P.d, ld, on, hp, row_end);
    }
    reduce_red_to_part(red, ld, P.part + (size_t)blockIdx.x * ld);
  } else {
    // MODE 2: light rows, one row group per row; the row's own entries are loaded with its
    // indices
    double dl[CPL];
#pragma unroll
    for (int v = 0; v < CPL; ++v) dl[v] = 0.0;
    for (int i = gid; i < g.n; i += GT) {
      const int lo = __ldg(g.d_indptr + i), hi = __ldg(g.d_indptr + i + 1);
      if (hi - lo > g.heavy_thresh) continue;
      T xi[CPL], yi[CPL];
      if (on) vload<T, CPL>(xi, P.d + (size_t)i * ld + rg.col);
      A acc[CPL];
#pragma unroll
      for (int v = 0; v < CPL; ++v) acc[v] = A(0);
      gather_rows<T, CPL, W, A>(g, rg, lo, hi, P.d, ld, acc, on);
      finish_row_pre<T, CPL, false, A>(g, rg, i, hi - lo, shift, P.d, ld, acc, P.v, ld, xi, yi, on);
      if (!on)
#pragma unroll
        for (int v = 0; v < CPL; ++v) xi[v] = T(0);
#pragma unroll
      for (int v = 0; v < CPL; ++v) dl[v] += (double)xi[v] * (double)yi[v];
    }
    reduce_cols_to_part<CPL>(dl, rg.G, ld, red, P.part + (size_t)blockIdx.x * ld);
  }
  if (last_cta(P.ctl + C_CNT1)) {
    reduce_partials(P.part, gridDim.x, ld, red, s_col);
    if (P.nbh > 0) {
      __shared__ double s_h[kMaxLd];
      reduce_partials(P.part_h, P.nbh, ld, red, s_h);
      for (int c = threadIdx.x; c < ld; c += blockDim.x) s_col[c] = s_h[c] + s_col[c];
      __syncthreads();
    }
    if (g.nx > 0) apply_added_edges(P, red, s_col);
    for (int c = threadIdx.x; c < ld; c += blockDim.x) {
      const int a_on = P.act[c];
      const double a = a_on ? P.rr[c] / s_col[c] : 0.0;
      if (a_on && !isfinite(a)) atomicCAS(P.ctl + C_ERR, 0, (int)POLAR_ERR_NONFINITE);
      P.ag[c] = a;
    }
  }
}

// ---- r <- r - a v, history, r.r, column scalars -----------------------------------------
template <typename T, int VEC>
__global__ void __launch_bounds__(kBlock, POLAR_STREAM_MINB) mk_resid(const __grid_constant__ SolvePrm<T> P, int slot) {

  pdl_wait();
  pdl_launch();
  if (!solve_live(P.ctl, P.stats, P.maxit)) return;
  __shared__ double red[kWarps * kMaxLd];
  __shared__ double s_col[kMaxLd];
  const int ld = P.ld, nA = P.nA;
  const RowGroup rg = make_row_group<VEC>(ld);
  const long long tid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long nth = (long long)gridDim.x * blockDim.x;
  const long long nvec = (long long)P.n * rg.G;
  const int lgG = __ffs(rg.G) - 1;
  double a_c[VEC], racc[VEC];
  bool on[VEC], any_on = false;
#pragma unroll
  for (int v = 0; v < VEC; ++v) {
    a_c[v] = P.ag[rg.col + v];
    on[v] = P.act[rg.col + v] != 0;
    any_on |= on[v];
    racc[v] = 0.0;
  }
  if (any_on) {
    T* hslot = P.hist + (size_t)slot * nA * ld;
    constexpr int U = sizeof(T) == 4 ? POLAR_RESID_U32 : POLAR_RESID_U;
    for (long long e0 = tid; e0 < nvec; e0 += U * nth) {
      double rv[U][VEC];
      T vv[U][VEC];
      long long ii[U];
      int ai[U];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const long long e = e0 + u * nth;
        ii[u] = e < nvec ? (e >> lgG) : -1;
        if (ii[u] >= 0) {
          load_res<T, VEC>(P, rv[u], (size_t)ii[u] * ld + rg.col);
          vload<T, VEC>(vv[u], P.v + (size_t)ii[u] * ld + rg.col);
          ai[u] = __ldg(P.active_pos + ii[u]);
        }
      }
#pragma unroll
      for (int u = 0; u < U; ++u) {
        if (ii[u] < 0) continue;
        T rt[VEC];
#pragma unroll
        for (int v = 0; v < VEC; ++v)
          if (on[v]) rv[u][v] = rv[u][v] - a_c[v] * (double)vv[u][v];
        store_res<T, VEC>(P, rv[u], (size_t)ii[u] * ld + rg.col);
#pragma unroll
        for (int v = 0; v < VEC; ++v) {
          racc[v] += rv[u][v] * rv[u][v];
          rt[v] = (T)rv[u][v];
        }
        if (ai[u] >= 0) vstore_cs<T, VEC>(hslot + (size_t)ai[u] * ld + rg.col, rt);
      }
    }
  }
  reduce_cols_to_part<VEC>(racc, rg.G, ld, red, P.part + (size_t)blockIdx.x * ld);
  if (last_cta(P.ctl + C_CNT3)) {
    reduce_partials(P.part, gridDim.x, ld, red, s_col);
    const bool anyv = column_step(P, s_col);
    if (threadIdx.x == 0) {
      P.ctl[C_ANY] = anyv ? 1 : 0;
      P.ctl[C_RAN] = 1;
      P.stats[0] += 1;
    }
  }
}

// ---- pole recurrences + d <- r + beta d -------------------------------------------------
template <typename T, int VEC>
__global__ void __launch_bounds__(kBlock, POLAR_STREAM_MINB) mk_dir(const __grid_constant__ SolvePrm<T> P, int slot) {

  pdl_wait();
  pdl_launch();
  if (ld_volatile_i32(P.ctl + C_RAN) == 0) return;
  const int ld = P.ld;
  const long long tid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long nth = (long long)gridDim.x * blockDim.x;
  const double shift0 = __ldg(P.tau);
  if (P.cmp) {
    // pole items spread over the CTAs, one half-warp per item (lane = history index)
    const int hw = threadIdx.x >> 4, hl = threadIdx.x & 15;
    const unsigned hmask = 0xffffu << (threadIdx.x & 16);
    const long long items = (long long)P.p * ld;
    for (long long q = blockIdx.x + (long long)gridDim.x * hw; q < items; q += (long long)gridDim.x * (blockDim.x >> 4))
      pole_step_unit(P, q, hl, hmask, slot, shift0);
  } else {
    for (long long q = tid; q < (long long)P.p * ld; q += nth) pole_step(P, q, slot, shift0);
  }
  const bool more = ld_volatile_i32(P.ctl + C_ANY) != 0 && P.stats[0] < P.maxit;
  if (more) {
    const RowGroup rg = make_row_group<VEC>(ld);
    const long long nvec = (long long)P.n * rg.G;
    const int lgG = __ffs(rg.G) - 1;
    double be_c[VEC];
    bool on[VEC], any_on = false;
#pragma unroll
    for (int v = 0; v < VEC; ++v) {
      be_c[v] = P.beg[rg.col + v];
      on[v] = P.upd[rg.col + v] != 0;
      any_on |= on[v];
    }
    if (any_on) {
      const uint64_t pol_hot = l2_policy(P.l2_mode ? 1 : 0);
      const uint64_t pol_norm = l2_policy(0);
      // FP64 r doubles the registers of a row item: fewer items in flight for wide FP32 rows
      constexpr int U = (sizeof(T) == 4 && VEC >= 4 && POLAR_STREAM_U > 2) ? 2 : POLAR_STREAM_U;
      for (long long e0 = tid; e0 < nvec; e0 += U * nth) {
        double rv[U][VEC], dv[U][VEC];
        long long ii[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
          const long long e = e0 + u * nth;
          ii[u] = e < nvec ? (e >> lgG) : -1;
          if (ii[u] >= 0) {
            load_res<T, VEC>(P, rv[u], (size_t)ii[u] * ld + rg.col);
            load_dir<T, VEC>(P, dv[u], (size_t)ii[u] * ld + rg.col);
          }
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
          if (ii[u] < 0) continue;
#pragma unroll
          for (int v = 0; v < VEC; ++v)
            if (on[v]) dv[u][v] = rv[u][v] + be_c[v] * dv[u][v];
          store_dir_hint<T, VEC>(P, dv[u], (size_t)ii[u] * ld + rg.col, row_policy(P, ii[u], pol_hot, pol_norm),
                                 pol_norm);
        }
      }
    }
  }
  if (last_cta(P.ctl + C_CNT4)) {
    if (threadIdx.x == 0) {
      P.ctl[C_NSTEPS] = slot + 1;
      P.ctl[C_RAN] = 0;
    }
  }
}

// ---- deferred shifted update (final pass writes the output) -----------------------------
template <typename T, int E>
// The composed coefficients of a column chunk take up to ~150 KB of shared memory, so one
// CTA is resident per SM; the 64-register bound still schedules the full-scale pass
// (DRAM-bound, ~14.5 GB per launch at n = 4M) better than a 128-register one (measured
// 2.08 ms against 2.57 ms per launch).
__global__ void __launch_bounds__(kBlock, 2) mk_flush(const __grid_constant__ SolvePrm<T> P, int force_final) {
  extern __shared__ __align__(16) unsigned char flush_sm[];

  pdl_wait();
  pdl_launch();
  const int nsteps = ld_volatile_i32(P.ctl + C_NSTEPS);
  const bool first = ld_volatile_i32(P.ctl + C_FIRST) != 0;
  const bool done = ld_volatile_i32(P.ctl + C_ANY) == 0 || ld_volatile_i32(P.ctl + C_ERR) != 0;
  const bool final_pass = force_final || done;
  if (!final_pass && nsteps == 0) return;
  const long long tid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long nth = (long long)gridDim.x * blockDim.x;
  if (P.cmp && composed_smem_bytes<T>(P.ld, P.p) <= kFlushSmemMax)
    shifted_update_composed<T, E>(P, nsteps, first, final_pass, reinterpret_cast<T*>(flush_sm));
  else if (flush_smem_bytes<T>(P.ld, P.p, kHist) <= kFlushSmemMax)
    shifted_update_smem<T, E>(P, nsteps, first, final_pass, reinterpret_cast<T*>(flush_sm));
  else
    shifted_update<T, E>(P, nsteps, first, final_pass, tid, nth);
  if (final_pass && P.track && P.h_out)
    for (long long q = tid; q < (long long)P.p * P.ld; q += nth) {
      const int j = (int)(q / P.ld), c = (int)(q % P.ld);
      if (c < P.R) P.h_out[(size_t)j * P.R + c] = P.hs[q];
    }
  if (last_cta(P.ctl + C_CNT5)) {
    if (threadIdx.x == 0) {
      P.ctl[C_NSTEPS] = 0;
      P.ctl[C_FIRST] = 0;
      P.stats[1] += 1;
    }
  }
}

// ---------------------------------------------------------------------------------------
template <typename F>
static int occ_grid(F* fn, int block);

// Kernel launch with programmatic stream serialization (on unless POLAR_PDL=0): inside the
// captured iteration block each kernel's launch overlaps its predecessor's tail.
static bool pdl_on() {
  static const bool on = [] {
    const char* e = getenv("POLAR_PDL");
    return !(e && e[0] == '0');
  }();
  return on;
}

template <typename... KArgs, typename... Args>
static void launch_k(void (*k)(KArgs...), int grid, int block, size_t smem, cudaStream_t st, Args... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(block);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = pdl_on() ? 1 : 0;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  cudaLaunchKernelEx(&cfg, k, args...);
}

// True when the SpMM runs as one sliced-ELL launch (MODE 3).
template <typename T, bool W>
static bool spmm_merged(int cpl, const SolvePrm<T>& P) {
  const int gpw = 32 / (P.ld / cpl);
  return !W && P.g.nsl > 0 && P.g.sell_s == gpw;
}

// Dynamic shared memory of the merged SpMM launch: the slice pass's cp.async ring when it
// is built in (the attribute is raised once per instantiation).
template <typename T, int CPL>
static size_t ring_bytes() {
  if (POLAR_SELL_ASYNC == 0 || (CPL * sizeof(T)) % 16 != 0) return 0;
  return (size_t)kWarps * kSellRingWarp;
}

template <typename T, int CPL, bool W>
static void ring_attribute() {
  static bool done = false;
  if (!done && ring_bytes<T, CPL>() > 0) {
    cudaFuncSetAttribute(mk_spmm<T, CPL, W, 3>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)ring_bytes<T, CPL>());
  }
  done = true;
}

// SpMM launch for a runtime choice of columns per lane.
template <typename T, bool W>
struct SpmmLaunch {
  template <int CPL>
  static int grid() {
    ring_attribute<T, CPL, W>();
    int dev = 0, sms = 0, nb = 0, nb3 = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, mk_spmm<T, CPL, W, 2>, kBlock, 0);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb3, mk_spmm<T, CPL, W, 3>, kBlock, ring_bytes<T, CPL>());
    if (nb3 < nb) nb = nb3;
    if (nb < 1) nb = 1;
    return nb * sms;
  }
  // part 1: heavy-row launch, part 2: light-row launch
  template <int CPL>
  static void go(int part, int g, const SolvePrm<T>& P, cudaStream_t st) {
    if (part == 1) {
      if (P.nbh > 0) launch_k(mk_spmm<T, CPL, W, 1>, P.nbh, kBlock, 0, st, P);
      return;
    }
    if (spmm_merged<T, W>(CPL, P))
      launch_k(mk_spmm<T, CPL, W, 3>, g, kBlock, ring_bytes<T, CPL>(), st, P);
    else
      launch_k(mk_spmm<T, CPL, W, 2>, g, kBlock, 0, st, P);
  }
};

static int g_spmm_cpl_bytes = 0;  // 0: automatic

template <typename T>
static int spmm_cpl(int ld, int vec) {
  // 32 bytes per lane for rows of 512 bytes or more, otherwise one 16-byte access
  int bytes = g_spmm_cpl_bytes ? g_spmm_cpl_bytes : (ld * (int)sizeof(T) >= 512 ? 32 : 16);
  int cpl = bytes / (int)sizeof(T);
  if (cpl < vec) cpl = vec;
  if (cpl > ld) cpl = ld;
  while (ld / cpl > 32) cpl *= 2;
  return cpl;
}

static int g_sell = 1;
int mk_spmm_lanes(int precision, int ld);

int mk_sell_rows(int precision, int ld) {
  if (!g_sell) return 0;
  return 32 / mk_spmm_lanes(precision, ld);
}

int mk_spmm_lanes(int precision, int ld) {
  if (precision == POLAR_MIXED) return ld / spmm_cpl<float>(ld, ld >= 4 ? 4 : ld);
  return ld / spmm_cpl<double>(ld, ld >= 2 ? 2 : ld);
}

template <typename T, bool W>
static int spmm_grid(int cpl) {
  using L = SpmmLaunch<T, W>;
  switch (cpl) {
    case 1: return L::template grid<1>();
    case 2: return L::template grid<2>();
    case 4: return L::template grid<4>();
    case 8: return L::template grid<8>();
    default: return sizeof(T) == 4 ? L::template grid<16>() : L::template grid<8>();
  }
}

template <typename T, bool W>
static void spmm_go(int part, int cpl, int g, const SolvePrm<T>& P, cudaStream_t st) {
  using L = SpmmLaunch<T, W>;
  switch (cpl) {
    case 1: L::template go<1>(part, g, P, st); break;
    case 2: L::template go<2>(part, g, P, st); break;
    case 4: L::template go<4>(part, g, P, st); break;
    case 8: L::template go<8>(part, g, P, st); break;
    default:
      if (sizeof(T) == 4) L::template go<16>(part, g, P, st);
      else L::template go<8>(part, g, P, st);
  }
}

template <typename F>
static int occ_grid(F* fn, int block) {
  int dev = 0, sms = 0, nb = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, fn, block, 0);
  if (nb < 1) nb = 1;
  return nb * sms;
}

template <typename T, int E>
static size_t flush_smem_for(const SolvePrm<T>& P) {
  if (P.cmp && composed_smem_bytes<T>(P.ld, P.p) <= kFlushSmemMax) return composed_smem_bytes<T>(P.ld, P.p);
  const size_t b = flush_smem_bytes<T>(P.ld, P.p, kHist);
  return b <= kFlushSmemMax ? b : 0;
}

template <typename T, int E>
static int flush_grid(const SolvePrm<T>& P, size_t smem) {
  static bool attr = false;
  if (!attr) {
    cudaFuncSetAttribute(mk_flush<T, E>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kFlushSmemMax);
    attr = true;
  }
  int dev = 0, sms = 0, nb = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, mk_flush<T, E>, kBlock, smem);
  if (nb < 1) nb = 1;
  const int nch = P.ld / flush_cw<T>(P.ld);
  int g = nb * sms;
  g -= g % nch;
  return g < nch ? nch : g;
}

template <typename T, int VEC, bool W, int E>
int mk_grid_max() {
  int g = 0;
  for (int cpl = 1; cpl <= 16 / (int)(sizeof(T) / 4); cpl *= 2) {
    const int gc = spmm_grid<T, W>(cpl);
    g = g > gc ? g : gc;
  }
  g = g > occ_grid(mk_resid<T, VEC>, kBlock) ? g : occ_grid(mk_resid<T, VEC>, kBlock);
  g = g > occ_grid(mk_init<T, VEC>, kBlock) ? g : occ_grid(mk_init<T, VEC>, kBlock);
  return g;
}

// Launch helper: counts the launch and, with timing on, brackets it with events and
// records its algorithmic bytes.
template <typename F>
static void timed(int cls, double bytes, cudaStream_t st, F&& launch) {
  count_launch();
  if (!timing_on()) {
    launch();
    return;
  }
  TimedLaunch t{cls, bytes, timing_event(), timing_event()};
  cudaEventRecord(t.a, st);
  launch();
  cudaEventRecord(t.b, st);
  timing_push(t);
}

// One solve of the kernel-per-phase driver as a restartable object: start() clears the
// history, launches the initialisation and captures the iteration block (M iterations and
// one deferred-update pass) as a CUDA graph; launch() queues one block on the solve's
// stream; check() (after that stream has drained the block) reads the control words and
// decides whether the solve is done.  mk_solve runs one object to completion; the batched
// driver keeps one per problem, each on its own stream, so small solves overlap.
// grid_frac in (0, 1] scales every grid (the kernels stride over any grid), so that
// concurrent solves share the SMs.
template <typename T, int VEC, bool W, int E>
struct MkSolver {
  struct GraphTimed {
    int cls;
    double bytes;
    cudaEvent_t a, b;
  };
  SolvePrm<T> P;
  cudaStream_t st = nullptr;
  cudaStream_t cs = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  std::vector<GraphTimed> gt;
  bool timing = false;
  int g5 = 1, per_block = 0;
  size_t s5 = 0;
  double b_flush = 0.0;
  int ctl[8] = {0};
  long long stats[2] = {0, 0};
  bool done = false;
  MkResult res{};

  static int scaled(int g, double f, int mult) {
    int x = (int)(g * f + 0.5);
    if (x < mult) x = mult;
    x -= x % mult;
    return x < mult ? mult : x;
  }

  int start(const SolvePrm<T>& P0, cudaStream_t stream, double grid_frac) {
    P = P0;
    st = stream;
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const double f = grid_frac > 0.0 && grid_frac < 1.0 ? grid_frac : 1.0;
    // heavy chunks run in their own launch when there are any (one warp per chunk, at most
    // two CTAs per SM), except on the sliced-ELL path, whose launch takes them first
    {
      const int want = (P.g.nchunks + kWarps - 1) / kWarps;
      const int cap = scaled(2 * sms, f, 1);
      P.nbh = P.g.nchunks > 0 ? (want < cap ? want : cap) : 0;
      if (P.nbh > kMaxHeavyCtas) P.nbh = kMaxHeavyCtas;
    }
    const double s = sizeof(T), n = P.n, R = P.R, nA = P.nA;
    // algorithmic bytes per launch (unweighted CSR: values implicit, diagonal from indptr)
    const double b_spmm = 4.0 * (n + 1) + 4.0 * P.g.nnz + 2.0 * s * n * R;
    // r is FP64, or FP32 with r32; mixed precision keeps the direction's FP32 remainder
    const double rb = P.r32 ? 4.0 : 8.0;
    const double b_resid = (2.0 * rb + s) * n * R + s * nA * R;
    const double b_dir = (rb + 16.0) * n * R;  // r + direction (8) in, direction (8) out
    b_flush = (4.0 * P.p + kHist) * s * nA * R;
    const int g0 = scaled(occ_grid(mk_init<T, VEC>, kBlock), f, 1);
    const int cpl = spmm_cpl<T>(P.ld, VEC);
    if (spmm_merged<T, W>(cpl, P)) P.nbh = 0;
    const int g1 = scaled(spmm_grid<T, W>(cpl), f, 1);
    const int g3 = scaled(occ_grid(mk_resid<T, VEC>, kBlock), f, 1);
    const int g4 = scaled(occ_grid(mk_dir<T, VEC>, kBlock), f, 1);
    s5 = flush_smem_for<T, E>(P);
    g5 = scaled(flush_grid<T, E>(P, s5), f, P.ld / flush_cw<T>(P.ld));
    res.grid = g1;
    // the composed flush multiplies every history slot (zero coefficients for unused ones)
    cudaError_t e = cudaMemsetAsync(P.hist, 0, sizeof(T) * (size_t)kHist * P.nA * P.ld, st);
    if (e != cudaSuccess) return set_cuda_error("history clear", e);
    timed(KC_INIT, (16.0 + s) * n * R, st, [&] { mk_init<T, VEC><<<g0, kBlock, 0, st>>>(P); });
    e = cudaGetLastError();
    if (e != cudaSuccess) return set_cuda_error("mk_init", e);
    // One block = M iterations and one deferred-update pass, captured once per solve as a
    // CUDA graph (the parameters are fixed for the whole solve) and launched until
    // convergence.  With kernel timing on, each kernel node is bracketed by event nodes.
    timing = timing_on();
    auto node = [&](cudaStream_t x, int cls, double bytes, auto&& launch) {
      if (timing) {
        GraphTimed t{cls, bytes, nullptr, nullptr};
        cudaEventCreate(&t.a);
        cudaEventCreate(&t.b);
        // inside capture only an external record becomes an event-record node
        cudaEventRecordWithFlags(t.a, x, cudaEventRecordExternal);
        launch(x);
        cudaEventRecordWithFlags(t.b, x, cudaEventRecordExternal);
        gt.push_back(t);
      } else {
        launch(x);
      }
    };
    e = cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
      cs = nullptr;
      return set_cuda_error("capture stream", e);
    }
    e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) return set_cuda_error("begin capture", e);
    for (int k = 0; k < kHist; ++k) {
      if (P.nbh > 0) node(cs, KC_HEAVY, 0.0, [&](cudaStream_t x) { spmm_go<T, W>(1, cpl, g1, P, x); });
      node(cs, KC_SPMM, b_spmm, [&](cudaStream_t x) { spmm_go<T, W>(2, cpl, g1, P, x); });
      node(cs, KC_RESID, b_resid, [&](cudaStream_t x) { launch_k(mk_resid<T, VEC>, g3, kBlock, 0, x, P, k); });
      node(cs, KC_DIR, b_dir, [&](cudaStream_t x) { launch_k(mk_dir<T, VEC>, g4, kBlock, 0, x, P, k); });
    }
    node(cs, KC_FLUSH, b_flush, [&](cudaStream_t x) { launch_k(mk_flush<T, E>, g5, kBlock, s5, x, P, 0); });
    e = cudaStreamEndCapture(cs, &graph);
    if (e == cudaSuccess) e = cudaGraphInstantiate(&exec, graph, 0);
    if (e != cudaSuccess) return set_cuda_error("graph build", e);
    per_block = (P.nbh > 0 ? 4 : 3) * kHist + 1;
    return POLAR_OK;
  }

  int launch() {
    cudaError_t e = cudaGraphLaunch(exec, st);
    count_launch(per_block);
    if (e != cudaSuccess) return set_cuda_error("msolve block", e);
    return POLAR_OK;
  }

  // Reads the control words once the stream has executed the last launched block (the
  // copies are ordered after it).  Sets `done` and fills `res`.
  int check() {
    cudaError_t e = cudaMemcpyAsync(ctl, P.ctl, sizeof(ctl), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(stats, P.stats, sizeof(stats), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return set_cuda_error("msolve block", e);
    if (timing)
      for (auto& t : gt) {
        float ms = 0.f;
        if (cudaEventElapsedTime(&ms, t.a, t.b) == cudaSuccess)
          timing_add(t.cls, t.bytes, ms);
        else
          cudaGetLastError();
      }
    if (ctl[C_ERR] != 0 || ctl[C_ANY] == 0) {
      done = true;
    } else if (stats[0] >= P.maxit) {
      timed(KC_FLUSH, b_flush, st, [&] { mk_flush<T, E><<<g5, kBlock, s5, st>>>(P, 1); });
      e = cudaMemcpyAsync(ctl, P.ctl, sizeof(ctl), cudaMemcpyDeviceToHost, st);
      if (e == cudaSuccess) e = cudaMemcpyAsync(stats, P.stats, sizeof(stats), cudaMemcpyDeviceToHost, st);
      if (e == cudaSuccess) e = cudaStreamSynchronize(st);
      if (e != cudaSuccess) return set_cuda_error("msolve sync", e);
      done = true;
    }
    if (done) {
      res.err = ctl[C_ERR];
      res.capped = ctl[C_ERR] == 0 && ctl[C_ANY] != 0;
      res.iterations = stats[0];
      res.flushes = stats[1];
    }
    return POLAR_OK;
  }

  void cleanup() {
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    if (cs) cudaStreamDestroy(cs);
    for (auto& t : gt) {
      cudaEventDestroy(t.a);
      cudaEventDestroy(t.b);
    }
    exec = nullptr;
    graph = nullptr;
    cs = nullptr;
    gt.clear();
  }
};

template <typename T, int VEC, bool W, int E>
int mk_solve(const SolvePrm<T>& P0, SolvePrm<T>* dev_prm, cudaStream_t st, MkResult* out) {
  (void)dev_prm;
  MkSolver<T, VEC, W, E> S;
  int rc = S.start(P0, st, 1.0);
  while (rc == POLAR_OK && !S.done) {
    rc = S.launch();
    if (rc == POLAR_OK) rc = S.check();
  }
  if (S.timing) timing_collect();
  S.cleanup();
  if (rc != POLAR_OK) return rc;
  *out = S.res;
  return POLAR_OK;
}

// Many solves at once: one MkSolver per problem, each on its own stream (ordered after
// the caller's stream) with grids scaled by its share of the work.  The host polls the
// streams and relaunches each solve's block as soon as its previous one has drained, so
// a short solve never waits for a long one.
template <typename T, int VEC, bool W, int E>
int mk_solve_batch(const std::vector<SolvePrm<T>>& Ps, const std::vector<double>& frac, cudaStream_t st,
                   std::vector<MkResult>& out) {
  const int np = (int)Ps.size();
  std::vector<MkSolver<T, VEC, W, E>> S(np);
  std::vector<cudaStream_t> ss(np, nullptr);
  std::vector<cudaEvent_t> ev(np, nullptr);
  cudaEvent_t ready = nullptr;
  int rc = POLAR_OK;
  cudaError_t e = cudaEventCreateWithFlags(&ready, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaEventRecord(ready, st);
  if (e != cudaSuccess) rc = set_cuda_error("batch start event", e);
  for (int b = 0; b < np && rc == POLAR_OK; ++b) {
    e = cudaStreamCreateWithFlags(&ss[b], cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ev[b], cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(ss[b], ready, 0);
    if (e != cudaSuccess) {
      rc = set_cuda_error("batch stream", e);
      break;
    }
    rc = S[b].start(Ps[b], ss[b], frac[b]);
  }
  std::vector<char> queued(np, 0);
  for (int b = 0; b < np && rc == POLAR_OK; ++b) {
    rc = S[b].launch();
    if (rc == POLAR_OK && cudaEventRecord(ev[b], ss[b]) != cudaSuccess) rc = set_cuda_error("batch event", cudaGetLastError());
    queued[b] = 1;
  }
  int live = np;
  while (rc == POLAR_OK && live > 0) {
    bool progressed = false;
    for (int b = 0; b < np && rc == POLAR_OK; ++b) {
      if (!queued[b]) continue;
      const cudaError_t q = cudaEventQuery(ev[b]);
      if (q == cudaErrorNotReady) continue;
      if (q != cudaSuccess) {
        rc = set_cuda_error("batch poll", q);
        break;
      }
      progressed = true;
      queued[b] = 0;
      rc = S[b].check();
      if (rc != POLAR_OK) break;
      if (S[b].done) {
        --live;
        continue;
      }
      rc = S[b].launch();
      if (rc == POLAR_OK && cudaEventRecord(ev[b], ss[b]) != cudaSuccess) rc = set_cuda_error("batch event", cudaGetLastError());
      queued[b] = 1;
    }
    if (!progressed) std::this_thread::yield();
  }
  // the caller's stream waits for every problem's stream
  for (int b = 0; b < np; ++b)
    if (ss[b]) {
      if (cudaEventRecord(ev[b], ss[b]) == cudaSuccess) cudaStreamWaitEvent(st, ev[b], 0);
    }
  if (timing_on()) timing_collect();
  out.assign(np, MkResult{});
  for (int b = 0; b < np; ++b) {
    // drain every stream before its graph is destroyed (also after an error elsewhere)
    if (ss[b] && cudaStreamSynchronize(ss[b]) != cudaSuccess && rc == POLAR_OK)
      rc = set_cuda_error("batch drain", cudaGetLastError());
    out[b] = S[b].res;
    S[b].cleanup();
    if (ev[b]) cudaEventDestroy(ev[b]);
    if (ss[b]) cudaStreamDestroy(ss[b]);
  }
  if (ready) cudaEventDestroy(ready);
  return rc;
}

}  // namespace polar

extern "C" void polar_set_spmm_lane_bytes(int bytes) { polar::g_spmm_cpl_bytes = bytes; }
extern "C" void polar_set_sell(int on) { polar::g_sell = on; }

namespace polar {

#define POLAR_MK_INST(T, VEC, W, E)                                                                 \
  template int mk_solve<T, VEC, W, E>(const SolvePrm<T>&, SolvePrm<T>*, cudaStream_t, MkResult*); \
  template int mk_solve_batch<T, VEC, W, E>(const std::vector<SolvePrm<T>>&, const std::vector<double>&, \
                                            cudaStream_t, std::vector<MkResult>&);                   \
  template int mk_grid_max<T, VEC, W, E>();

POLAR_MK_INST(float, 4, false, POLAR_E32)
POLAR_MK_INST(float, 4, true, POLAR_E32)
POLAR_MK_INST(float, 2, false, POLAR_E32)
POLAR_MK_INST(float, 2, true, POLAR_E32)
POLAR_MK_INST(float, 1, false, POLAR_E32)
POLAR_MK_INST(float, 1, true, POLAR_E32)
POLAR_MK_INST(double, 2, false, POLAR_E64)
POLAR_MK_INST(double, 2, true, POLAR_E64)
POLAR_MK_INST(double, 1, false, POLAR_E64)
POLAR_MK_INST(double, 1, true, POLAR_E64)

}  // namespace polar
