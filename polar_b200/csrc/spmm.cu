// Standalone operator apply: Y = (M + shift I) X  (realworld/spmm.py:4-25, polar_gpu.py:71-80).
//
// The same row-group SpMM as the solver's P1 phase, as an ordinary launch.  Heavy rows
// are split into chunks whose partial sums are combined by the last chunk to finish, in
// chunk order, so the result does not depend on scheduling.
#include <cuda_runtime.h>

#include "common.cuh"
#include "graph_ops.cuh"
#include "host_util.h"
#include "sell_spmm.cuh"

namespace polar {

constexpr int kSpmmBlock = 256;
#ifndef POLAR_PANEL_MINB
#define POLAR_PANEL_MINB 1
#endif

template <typename T, int VEC, bool WEIGHTED>
__global__ void __launch_bounds__(kSpmmBlock) spmm_kernel(polar_graph g, int R, int G, double shift, const T* X,
                                                          int ldx, T* Y, int ldy,
                                                          typename AccOf<T>::type* part, int* hcount) {
  using A = typename AccOf<T>::type;
  RowGroup rg;
  rg.G = G;
  const int lane = threadIdx.x & 31;
  rg.lg = lane & (G - 1);
  const int base = lane - rg.lg;
  rg.mask = (G == 32) ? 0xffffffffu : (((1u << G) - 1u) << base);
  rg.col = rg.lg * VEC;
  const bool on = rg.col < R;
  if (!on) rg.col = 0;  // idle lanes still take part in the index shuffles
  const int gpw = 32 / G;
  const int gid = (blockIdx.x * (kSpmmBlock / 32) + (threadIdx.x >> 5)) * gpw + lane / G;
  const int GT = gridDim.x * (kSpmmBlock / 32) * gpw;
  const int ldp = G * VEC;

  for (int ch = gid; ch < g.nchunks; ch += GT) {
    const int h = g.d_chunk_row[ch];
    A acc[VEC];
#pragma unroll
    for (int v = 0; v < VEC; ++v) acc[v] = A(0);
    gather_rows<T, VEC, WEIGHTED>(g, rg, g.d_chunk_lo[ch], g.d_chunk_hi[ch], X, ldx, acc);
    vstore<A, VEC>(part + (size_t)ch * ldp + rg.lg * VEC, acc);
    __threadfence();
    __syncwarp(rg.mask);
    int old = 0;
    if (rg.lg == 0) old = atomicAdd(hcount + h, 1);
    old = __shfl_sync(rg.mask, old, 0, G);
    const int c0 = g.d_hchunk_off[h], c1 = g.d_hchunk_off[h + 1];
    if (old == c1 - c0 - 1) {
      __threadfence();
      A sum[VEC];
#pragma unroll
      for (int v = 0; v < VEC; ++v) sum[v] = A(0);
      for (int c2 = c0; c2 < c1; ++c2) {
        A pv[VEC];
        vload_cg<A, VEC>(pv, part + (size_t)c2 * ldp + rg.lg * VEC);
#pragma unroll
        for (int v = 0; v < VEC; ++v) sum[v] += pv[v];
      }
      const int i = g.d_hrow[h];
      T xi[VEC], yi[VEC];
      finish_row<T, VEC>(g, rg, i, g.d_indptr[i + 1] - g.d_indptr[i], shift, X, ldx, sum, Y, ldy, xi, yi, on);
      if (rg.lg == 0) hcount[h] = 0;
    }
  }
  for (int i = gid; i < g.n; i += GT) {
    const int lo = g.d_indptr[i], hi = g.d_indptr[i + 1];
    if (hi - lo > g.heavy_thresh) continue;
    A acc[VEC];
#pragma unroll
    for (int v = 0; v < VEC; ++v) acc[v] = A(0);
    gather_rows<T, VEC, WEIGHTED>(g, rg, lo, hi, X, ldx, acc);
    T xi[VEC], yi[VEC];
    finish_row<T, VEC>(g, rg, i, hi - lo, shift, X, ldx, acc, Y, ldy, xi, yi, on);
  }
}

// Panel/stream path (same code as the solver's SpMM phase) for power-of-two R with
// vector-aligned strides; persistent-size grid so panels sweep the GPU in step.
template <typename T, int VEC, bool WEIGHTED>
__global__ void __launch_bounds__(512, POLAR_PANEL_MINB) spmm_panel_kernel(polar_graph g, int R, double shift, const T* X, int ldx,
                                                         T* Y, int ldy, typename AccOf<T>::type* part, int* hcount) {
  (void)ldx;
  spmm_phase<T, VEC, WEIGHTED, false>(g, R, shift, X, Y, ldy, part, hcount, nullptr, nullptr);
}

// Sliced-ELL path (unweighted graphs with the layout for this width): the solver's SpMM
// passes with the standalone row finish (diagonal, shift and the greedy's added edges per
// row), FP64 row sums, the same L2 policies.  R == ld, a power of two.
template <typename T, int CPL>
__global__ void __launch_bounds__(512, 2) spmm_sell_kernel(polar_graph g, int ld, double shift, const T* X,
                                                           int ldx, T* Y, int ldy, double* part, int* hcount,
                                                           int l2_mode, int hot_rows) {
  using A = double;
  __shared__ int s_idx[16][kChunkMax];
  const RowGroup rg = make_row_group<CPL>(ld);
  const int warp = threadIdx.x >> 5;
  const int wid = blockIdx.x * 16 + warp;
  const int nw = gridDim.x * 16;
  const GatherHints hp = make_gather_hints(l2_mode, hot_rows, X, (size_t)ldx * sizeof(T), g.n);
  heavy_chunk_pass<T, CPL, false, A>(
      g, rg, wid, nw, X, ldx, ld, true, s_idx[warp], part, hcount, hp,
      [&](int i, int cnt, auto& acc, auto& xi) {
        T yi[CPL];
        finish_row_pre<T, CPL, true, A>(g, rg, i, cnt, shift, X, ldx, acc, Y, ldy, xi, yi, true);
      },
      [&](int, bool, auto&, auto&) {},
      [&](int i, int deg, auto& sum) {
        T xf[CPL], yi[CPL];
        finish_row<T, CPL, true, A>(g, rg, i, deg, shift, X, ldx, sum, Y, ldy, xf, yi, true);
      });
  auto row_end = [&](int row, int deg, auto& acc, auto& xi, bool go) {
    if (!go) return;
    const double wadd = added_terms<T, CPL, A>(g, rg, row, X, ldx, acc);
    const double dg = (double)deg + g.sigma + wadd + shift;
    T yv[CPL];
#pragma unroll
    for (int v = 0; v < CPL; ++v) yv[v] = (T)fma((A)dg, (A)xi[v], -acc[v]);
    vstore_hint<T, CPL>(Y + (size_t)row * ldy + rg.col, yv, hp.stream);
  };
  if constexpr (POLAR_SELL_ASYNC != 0 && (CPL * sizeof(T)) % 16 == 0) {
    extern __shared__ __align__(16) unsigned char sell_ring[];
    sell_slice_pass_async<T, CPL, A>(g, rg, wid, nw, X, ldx, true, hp,
                                     sell_ring + (size_t)warp * POLAR_SELL_STAGES * POLAR_SELL_BYTES * 32, row_end);
  } else {
    sell_slice_pass<T, CPL, A>(g, rg, wid, nw, X, ldx, true, hp, row_end);
  }
}

template <typename T, int CPL>
static int launch_spmm_sell(const polar_graph& g, int ld, double shift, const void* X, int ldx, void* Y, int ldy,
                            void* scratch, int precision, cudaStream_t st) {
  double* part = reinterpret_cast<double*>(scratch);
  int* hcount = reinterpret_cast<int*>(reinterpret_cast<char*>(scratch) + spmm_counter_offset(&g, precision));
  // the async slice pass's ring (16 warps of 512 threads), when built in
  const size_t ring = (POLAR_SELL_ASYNC != 0 && (CPL * sizeof(T)) % 16 == 0)
                          ? (size_t)16 * POLAR_SELL_STAGES * POLAR_SELL_BYTES * 32 : 0;
  static bool attr = false;
  if (!attr && ring > 0)
    cudaFuncSetAttribute(spmm_sell_kernel<T, CPL>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ring);
  attr = true;
  int dev = 0, sms = 0, nb = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, spmm_sell_kernel<T, CPL>, 512, ring);
  if (nb < 1) nb = 1;
  const long long hot = (long long)(l2_hot_bytes_setting() / ((size_t)ld * sizeof(T)));
  spmm_sell_kernel<T, CPL><<<nb * sms, 512, ring, st>>>(g, ld, shift, (const T*)X, ldx, (T*)Y, ldy, part, hcount,
                                                         l2_mode_setting(), (int)(hot < g.n ? hot : g.n));
  count_launch();
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return set_cuda_error("spmm launch", e);
  return POLAR_OK;
}

// The sliced-ELL launch for this call, or nothing (used = false) when the row-loop
// kernels apply: weighted graphs, no layout for this width, widths that are not a power of
// two, or blocks that are not 16-byte aligned.
template <typename T>
static int try_spmm_sell(const polar_graph& g, int precision, int R, double shift, const void* X, int ldx, void* Y,
                         int ldy, void* scratch, cudaStream_t st, bool* used) {
  *used = false;
  const int vmin = 16 / (int)sizeof(T);  // one 16-byte vector per lane at least
  if (g.d_wts || g.nsl <= 0 || R < vmin || (R & (R - 1)) != 0) return POLAR_OK;
  const int lanes = mk_spmm_lanes(precision, R);
  const int cpl = R / lanes;
  if (g.sell_s != 32 / lanes) return POLAR_OK;
  const size_t es = sizeof(T);
  if ((uintptr_t)X % 16 || (uintptr_t)Y % 16 || ((size_t)ldx * es) % 16 || ((size_t)ldy * es) % 16) return POLAR_OK;
  *used = true;
  switch (cpl) {
    case 2: return launch_spmm_sell<T, 2>(g, R, shift, X, ldx, Y, ldy, scratch, precision, st);
    case 4: return launch_spmm_sell<T, 4>(g, R, shift, X, ldx, Y, ldy, scratch, precision, st);
    case 8: return launch_spmm_sell<T, 8>(g, R, shift, X, ldx, Y, ldy, scratch, precision, st);
    case 16:
      if (sizeof(T) == 4) return launch_spmm_sell<T, 16>(g, R, shift, X, ldx, Y, ldy, scratch, precision, st);
      break;
  }
  *used = false;
  return POLAR_OK;
}

static int spmm_vec(int precision, int R, int ldx, int ldy, const void* X, const void* Y) {
  const int maxv = precision == POLAR_MIXED ? 4 : 2;
  const size_t es = precision == POLAR_MIXED ? 4 : 8;
  for (int v = maxv; v > 1; v >>= 1) {
    if (R % v == 0 && ldx % v == 0 && ldy % v == 0 && ((uintptr_t)X % (v * es)) == 0 &&
        ((uintptr_t)Y % (v * es)) == 0)
      return v;
  }
  return 1;
}

template <typename T, int VEC, bool W>
static int launch_spmm_panel(const polar_graph& g, int R, double shift, const void* X, int ldx, void* Y, int ldy,
                             void* scratch, cudaStream_t st) {
  using A = typename AccOf<T>::type;
  A* part = reinterpret_cast<A*>(scratch);
  int* hcount = reinterpret_cast<int*>(reinterpret_cast<char*>(scratch) +
                                       spmm_counter_offset(&g, sizeof(T) == 4 ? POLAR_MIXED : POLAR_FP64));
  int dev = 0, sms = 0, nb = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, spmm_panel_kernel<T, VEC, W>, 512, 0);
  if (nb < 1) nb = 1;
  spmm_panel_kernel<T, VEC, W><<<nb * sms, 512, 0, st>>>(g, R, shift, (const T*)X, ldx, (T*)Y, ldy, part, hcount);
  count_launch();
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return set_cuda_error("spmm launch", e);
  return POLAR_OK;
}

template <typename T, int VEC, bool W>
static int launch_spmm(const polar_graph& g, int R, double shift, const void* X, int ldx, void* Y, int ldy,
                       void* scratch, cudaStream_t st) {
  using A = typename AccOf<T>::type;
  const int G = next_pow2((R + VEC - 1) / VEC);
  const int ldp = G * VEC;
  A* part = reinterpret_cast<A*>(scratch);
  int* hcount = reinterpret_cast<int*>(reinterpret_cast<char*>(scratch) +
                                       spmm_counter_offset(&g, sizeof(T) == 4 ? POLAR_MIXED : POLAR_FP64));
  (void)ldp;
  const int gpb = (kSpmmBlock / 32) * (32 / G);
  long long groups_needed = (long long)g.n + g.nchunks;
  long long blocks = (groups_needed + gpb - 1) / gpb;
  int dev = 0, sms = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const long long cap = (long long)sms * 16;
  if (blocks > cap) blocks = cap;
  if (blocks < 1) blocks = 1;
  spmm_kernel<T, VEC, W><<<(int)blocks, kSpmmBlock, 0, st>>>(g, R, G, shift, (const T*)X, ldx, (T*)Y, ldy, part, hcount);
  count_launch();
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return set_cuda_error("spmm launch", e);
  return POLAR_OK;
}

}  // namespace polar

using namespace polar;

namespace polar {

size_t spmm_counter_offset(const polar_graph* g, int precision) {
  (void)precision;  // chunk partials: up to 128 columns of FP64 row sums in either precision
  return ((size_t)(g->nchunks > 0 ? g->nchunks : 1) * 128 * 8 + 255) & ~size_t(255);
}

int spmm_check_args(const polar_graph* g, int precision, int R, const void* d_X, int ldx, const void* d_Y,
                    int ldy) {
  if (!g || !d_X || !d_Y) return set_error(POLAR_ERR_BAD_ARG, "null pointer");
  if (precision != POLAR_FP64 && precision != POLAR_MIXED) return set_error(POLAR_ERR_BAD_ARG, "precision");
  if (R < 1 || ldx < R || ldy < R) return set_error(POLAR_ERR_BAD_ARG, "bad sizes");
  const int vec = spmm_vec(precision, R, ldx, ldy, d_X, d_Y);
  if ((R + vec - 1) / vec > 32) return set_error(POLAR_ERR_BAD_ARG, "R too large for one pass; split columns");
  if ((g->d_wts == nullptr) != (g->d_diag == nullptr)) return set_error(POLAR_ERR_BAD_ARG, "weights and diag go together");
  return POLAR_OK;
}

}  // namespace polar

extern "C" size_t polar_spmm_scratch_bytes(const polar_graph* g, int precision, int R) {
  (void)R;
  if (!g) return 0;
  return spmm_counter_offset(g, precision) + (((size_t)(g->nheavy > 0 ? g->nheavy : 1) * 4 * 8 + 255) & ~size_t(255));
}

extern "C" int polar_spmm_scratch_init(const polar_graph* g, int precision, int R, void* d_scratch,
                                       polar_stream_t stream) {
  clear_error();
  if (!g || !d_scratch) return set_error(POLAR_ERR_BAD_ARG, "null pointer");
  cudaError_t e = cudaMemsetAsync(d_scratch, 0, polar_spmm_scratch_bytes(g, precision, R), (cudaStream_t)stream);
  if (e != cudaSuccess) return set_cuda_error("cudaMemsetAsync", e);
  return POLAR_OK;
}

extern "C" int polar_spmm(const polar_graph* g, int precision, int R, double shift, const void* d_X, int ldx,
                          void* d_Y, int ldy, void* d_scratch, polar_stream_t stream) {
  clear_error();
  if (!d_scratch) return set_error(POLAR_ERR_BAD_ARG, "null pointer");
  const int rc = spmm_check_args(g, precision, R, d_X, ldx, d_Y, ldy);
  if (rc != POLAR_OK) return rc;
  const int vec = spmm_vec(precision, R, ldx, ldy, d_X, d_Y);
  const bool w = g->d_wts != nullptr;
  cudaStream_t st = (cudaStream_t)stream;
  {
    bool used = false;
    const int rs = precision == POLAR_MIXED
                       ? try_spmm_sell<float>(*g, precision, R, shift, d_X, ldx, d_Y, ldy, d_scratch, st, &used)
                       : try_spmm_sell<double>(*g, precision, R, shift, d_X, ldx, d_Y, ldy, d_scratch, st, &used);
    if (used || rs != POLAR_OK) return rs;
  }
  const bool pow2 = (R & (R - 1)) == 0;
  if (pow2 && ldx == R && precision == POLAR_MIXED && vec == 4)
    return w ? launch_spmm_panel<float, 4, true>(*g, R, shift, d_X, ldx, d_Y, ldy, d_scratch, st)
             : launch_spmm_panel<float, 4, false>(*g, R, shift, d_X, ldx, d_Y, ldy, d_scratch, st);
  if (pow2 && ldx == R && precision == POLAR_FP64 && vec == 2)
    return w ? launch_spmm_panel<double, 2, true>(*g, R, shift, d_X, ldx, d_Y, ldy, d_scratch, st)
             : launch_spmm_panel<double, 2, false>(*g, R, shift, d_X, ldx, d_Y, ldy, d_scratch, st);
  if (precision == POLAR_MIXED) {
    if (vec == 4) return w ? launch_spmm<float, 4, true>(*g, R, shift, d_X, ldx, d_Y, ldy, d_scratch, st)
                           : launch_spmm<float, 4, false>(*g, R, shift, d_X, ldx, d_Y, ldy, d_scratch, st);
    if (vec == 2) return w ? launch_spmm<float, 2, true>(*g, R, shift, d_X, ldx, d_Y, ldy, d_scratch, st)
                           : launch_spmm<float, 2, false>(*g, R, shift, d_X, ldx, d_Y, ldy, d_scratch, st);
    return w ? launch_spmm<float, 1, true>(*g, R, shift, d_X, ldx, d_Y, ldy, d_scratch, st)
             : launch_spmm<float, 1, false>(*g, R, shift, d_X, ldx, d_Y, ldy, d_scratch, st);
  }
  if (precision != POLAR_FP64) return set_error(POLAR_ERR_BAD_ARG, "precision");
  if (vec == 2) return w ? launch_spmm<double, 2, true>(*g, R, shift, d_X, ldx, d_Y, ldy, d_scratch, st)
                         : launch_spmm<double, 2, false>(*g, R, shift, d_X, ldx, d_Y, ldy, d_scratch, st);
  return w ? launch_spmm<double, 1, true>(*g, R, shift, d_X, ldx, d_Y, ldy, d_scratch, st)
           : launch_spmm<double, 1, false>(*g, R, shift, d_X, ldx, d_Y, ldy, d_scratch, st);
}
