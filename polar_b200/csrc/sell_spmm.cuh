// Sliced-ELL CSR-Laplacian SpMM passes shared by the solver's SpMM (mk_spmm) and the
// standalone operator apply (polar_spmm) on unweighted graphs (sm_100a).
//
// A launch runs the heavy-row chunks first and then the slices of light rows:
//  * heavy rows (degree above the partition's threshold) are cut into chunks of at most
//    kChunkMax neighbours, one warp per chunk.  The warp stages the chunk's indices in
//    shared memory with one coalesced pass; row group grp then takes neighbours grp,
//    grp + gpw, ... in batches of independent gathers, and the groups combine by shuffles
//    in a fixed pattern.  A row held in one chunk is finished by the warp; longer rows leave
//    per-chunk partials that the last chunk to arrive sums in chunk order, so results do
//    not depend on scheduling;
//  * light rows come in slices of gpw degree-sorted rows (the graph's sl_* arrays): a
//    warp reads neighbour k of all its rows with one coalesced load and issues predicated
//    gather batches, so short rows have all their gathers in flight; the next slice's
//    descriptors are fetched while this one is gathered, and a row's degree is the count
//    of its valid entries.
// Row sums are accumulated in A (FP64 for FP32 vectors unless the build says otherwise).
// The caller finishes rows through callbacks, which is where the solver forms d.v and the
// standalone apply adds the greedy's added edges.
#pragma once
#include "graph_ops.cuh"

#ifndef POLAR_HEAVY_BYTES
#define POLAR_HEAVY_BYTES 64  // bytes of gathered rows in flight per lane in a heavy chunk
#endif
#ifndef POLAR_SELL_BYTES
#define POLAR_SELL_BYTES 64   // same for a slice of light rows
#endif

#ifndef POLAR_SELL_ASYNC
#define POLAR_SELL_ASYNC 0  // 1: the slice pass gathers through cp.async into shared memory
#endif
#ifndef POLAR_SELL_STAGES
#define POLAR_SELL_STAGES 2  // batches of the cp.async ring per lane
#endif

namespace polar {

// 16-byte asynchronous copy global -> shared (L2 only); src_bytes 0 fills zeros and reads
// nothing.  The zero-fill form carries no L2 cache-policy operand.
POLAR_D void cp_async16(void* smem, const void* gmem, int src_bytes) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(s), "l"(gmem), "r"(src_bytes) : "memory");
}
POLAR_D void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
POLAR_D void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

#ifndef POLAR_RANGE_POLICY
#define POLAR_RANGE_POLICY 0  // 1: one address-range policy for all gathers (no per-gather choice)
#endif
#ifndef POLAR_SELL_DEG_INDPTR
#define POLAR_SELL_DEG_INDPTR 0  // 1: a slice row's degree from indptr, not counted per neighbour
#endif

// L2 policies of one pass: rows below hot_rows are the most gathered rows of a
// degree-ordered graph (kept with evict_last), the rest `cold`; `stream` for data read or
// written once.  With POLAR_RANGE_POLICY the gather policy is one address-range policy over
// the gathered block (evict_last on its first hot_rows rows, the secondary priority on the
// rest), so a gather needs no choice between policies.
struct GatherHints {
  uint64_t hot, cold, stream;
  int hot_rows;
  POLAR_D uint64_t row(long long i) const {
#if POLAR_RANGE_POLICY
    (void)i;
    return hot;
#else
    return i < hot_rows ? hot : cold;
#endif
  }
};

// Range policy over [base, base + total): primary evict_last on the first `primary` bytes,
// secondary evict_first (or unchanged) on the rest.  Sizes are 32-bit; blocks of 4 GB or
// more fall back to the fractional policy.
POLAR_D uint64_t l2_range_policy(const void* base, size_t primary, size_t total, bool cold_first) {
  uint64_t p;
  const unsigned ps = (unsigned)primary, ts = (unsigned)total;
  if (cold_first)
    asm volatile("createpolicy.range.global.L2::evict_last.L2::evict_first.b64 %0, [%1], %2, %3;"
                 : "=l"(p) : "l"(base), "r"(ps), "r"(ts));
  else
    asm volatile("createpolicy.range.global.L2::evict_last.L2::evict_unchanged.b64 %0, [%1], %2, %3;"
                 : "=l"(p) : "l"(base), "r"(ps), "r"(ts));
  return p;
}

// mode 0: no hints (evict_normal everywhere); 1: hot rows evict_last, streams evict_first;
// 2: as 1 with cold gathers evict_first.  `X`, `row_bytes`, `n`: the gathered block (used
// by the range form).
POLAR_D GatherHints make_gather_hints(int mode, int hot_rows, const void* X = nullptr, size_t row_bytes = 0,
                                      long long n = 0) {
  GatherHints h;
  h.hot = l2_policy(mode ? 1 : 0);
  h.cold = l2_policy(mode == 2 ? 2 : 0);
  h.stream = l2_policy(mode ? 2 : 0);
  h.hot_rows = hot_rows;
#if POLAR_RANGE_POLICY
  const size_t total = row_bytes * (size_t)n;
  if (mode && X && total > 0 && total < (size_t(1) << 32))
    h.hot = l2_range_policy(X, row_bytes * (size_t)hot_rows, total, mode == 2);
  else
    h.hot = h.cold;
#else
  (void)X;
  (void)row_bytes;
  (void)n;
#endif
  return h;
}

// Heavy chunks [wid, wid + nw, ...).  X rows have stride ldx; chunk partials have stride ldp.
// single(i, deg, acc, xi): a row held in one chunk (row-group leader lanes, grp == 0);
// partial(i, first, acc, xi): after a multi-chunk row's partial is stored (grp == 0, on);
// fin(i, deg, sum): the last-arriving chunk with the row's combined sum (grp == 0).
// xi is row i's own entries (loaded for grp == 0 when on).  s_idx: this warp's kChunkMax ints.
template <typename T, int CPL, bool W, typename A, typename Single, typename Partial, typename Final>
POLAR_D void heavy_chunk_pass(const polar_graph& g, const RowGroup& rg, int wid, int nw, const T* X, int ldx, int ldp,
                              bool on, int* s_idx, A* chunk_part, int* hcount, const GatherHints& hp,
                              Single&& single, Partial&& partial, Final&& fin) {
  constexpr int LB = CPL * (int)sizeof(T);
  constexpr int U = (POLAR_HEAVY_BYTES / LB) > 1 ? (POLAR_HEAVY_BYTES / LB) : 1;
  const int lane = threadIdx.x & 31;
  const int gpw = 32 / rg.G;
  const int grp = lane / rg.G;
  for (int ch = wid; ch < g.nchunks; ch += nw) {
    const int h = __ldg(g.d_chunk_row + ch);
    const int lo = __ldg(g.d_chunk_lo + ch), hi = __ldg(g.d_chunk_hi + ch);
    const int i = __ldg(g.d_hrow + h);
    const int c0 = __ldg(g.d_hchunk_off + h), c1 = __ldg(g.d_hchunk_off + h + 1);
    const bool one = (c1 - c0) == 1;
    T xi[CPL];
    if (on && grp == 0) vload<T, CPL>(xi, X + (size_t)i * ldx + rg.col);
    const int cnt = hi - lo;
    __syncwarp();
#pragma unroll
    for (int q = 0; q < kChunkMax / 32; ++q) {
      const int k = 32 * q + lane;
      if (k < cnt) s_idx[k] = ld_hint_i32(g.d_indices + lo + k, hp.stream);
    }
    __syncwarp();
    A acc[CPL];
#pragma unroll
    for (int v = 0; v < CPL; ++v) acc[v] = A(0);
    const int nu = cnt > grp ? (cnt - grp + gpw - 1) / gpw : 0;
    const int numax = (cnt + gpw - 1) / gpw;
    for (int u0 = 0; u0 < numax; u0 += U) {
      T xv[U][CPL];
      A wv[U];
#pragma unroll
      for (int uu = 0; uu < U; ++uu)
        if (on && u0 + uu < nu) {
          const int t = grp + gpw * (u0 + uu);
          const int j = s_idx[t];
          vload_hint<T, CPL>(xv[uu], X + (size_t)j * ldx + rg.col, hp.row(j));
          wv[uu] = W ? (A)__ldg(g.d_wts + lo + t) : A(1);
        }
#pragma unroll
      for (int uu = 0; uu < U; ++uu)
        if (on && u0 + uu < nu) {
#pragma unroll
          for (int v = 0; v < CPL; ++v) acc[v] = W ? fma(wv[uu], (A)xv[uu][v], acc[v]) : acc[v] + (A)xv[uu][v];
        }
    }
    for (int o = rg.G; o < 32; o <<= 1)
#pragma unroll
      for (int v = 0; v < CPL; ++v) acc[v] += __shfl_xor_sync(0xffffffffu, acc[v], o);
    if (one) {
      if (grp == 0) single(i, cnt, acc, xi);
      continue;
    }
    if (on && grp == 0) {
      vstore<A, CPL>(chunk_part + (size_t)ch * ldp + rg.col, acc);
      partial(i, ch == c0, acc, xi);
    }
    __threadfence();
    __syncwarp();
    int old = 0;
    if (lane == 0) old = atomicAdd(hcount + h, 1);
    old = __shfl_sync(0xffffffffu, old, 0);
    if (old == c1 - c0 - 1 && grp == 0) {
      __threadfence();
      A sum[CPL];
#pragma unroll
      for (int v = 0; v < CPL; ++v) sum[v] = A(0);
      if (on)
        for (int c2 = c0; c2 < c1; ++c2) {
          A pv[CPL];
          vload_cg<A, CPL>(pv, chunk_part + (size_t)c2 * ldp + rg.col);
#pragma unroll
          for (int v = 0; v < CPL; ++v) sum[v] += pv[v];
        }
      const int deg = __ldg(g.d_indptr + i + 1) - __ldg(g.d_indptr + i);
      fin(i, deg, sum);
      if (lane == 0) hcount[h] = 0;
    }
    __syncwarp();
  }
}

// Slices [wid, wid + nw, ...) of the light rows (g.sell_s == 32 / rg.G rows each).
// row_end(row, deg, acc, xi, go) is called by EVERY lane once per slice (it may shuffle):
// row = this row group's row (-1 for a pad), xi = its own entries (valid when go),
// go = a real row and on.
// Latency: a slice's work is a chain index load -> gathers -> accumulate per batch, so the
// indices of the next batch (or of the next slice's first batch) are loaded while this
// batch's gathers are in flight, and the row's own entries are loaded at the slice start.
template <typename T, int CPL, typename A, typename RowEnd>
POLAR_D void sell_slice_pass(const polar_graph& g, const RowGroup& rg, int wid, int nw, const T* X, int ldx, bool on,
                             const GatherHints& hp, RowEnd&& row_end) {
  constexpr int LB = CPL * (int)sizeof(T);
  constexpr int U = (POLAR_SELL_BYTES / LB) > 1 ? (POLAR_SELL_BYTES / LB) : 1;
  const int lane = threadIdx.x & 31;
  const int grp = lane / rg.G;
  const int S = 32 / rg.G;
  // descriptors (offset, width, row) of the current and the next slice, and the index
  // batch queued for the current slice
  int off = 0, w = 0, row = -1;
  int jj[U];
  auto fetch_desc = [&](int sl, int& o, int& wd, int& r) {
    o = __ldg(g.d_sl_off + sl);
    wd = (__ldg(g.d_sl_off + sl + 1) - o) / S;
    r = __ldg(g.d_sl_rows + (size_t)sl * S + grp);
  };
  auto fetch_idx = [&](int o, int wd, int k, int (&dst)[U]) {
    const int* sp = g.d_sl_idx + o + grp;
#pragma unroll
    for (int u = 0; u < U; ++u) dst[u] = (k + u < wd) ? ld_hint_i32(sp + (size_t)(k + u) * S, hp.stream) : -1;
  };
  if (wid < g.nsl) {
    fetch_desc(wid, off, w, row);
    fetch_idx(off, w, 0, jj);
  }
  for (int sl = wid; sl < g.nsl; sl += nw) {
    const int sn = sl + nw;
    int off_n = 0, w_n = 0, row_n = -1;
    if (sn < g.nsl) fetch_desc(sn, off_n, w_n, row_n);
    const bool go = row >= 0 && on;
    T xi[CPL];
    if (go) vload_hint<T, CPL>(xi, X + (size_t)row * ldx + rg.col, hp.row(row));
    A acc[CPL];
#pragma unroll
    for (int v = 0; v < CPL; ++v) acc[v] = A(0);
#if POLAR_SELL_DEG_INDPTR
    const int deg = row >= 0 ? __ldg(g.d_indptr + row + 1) - __ldg(g.d_indptr + row) : 0;
#else
    int deg = 0;
#endif
    for (int k = 0; k < w; k += U) {
      T xv[U][CPL];
#pragma unroll
      for (int u = 0; u < U; ++u)
        if (go && jj[u] >= 0) vload_hint<T, CPL>(xv[u], X + (size_t)jj[u] * ldx + rg.col, hp.row(jj[u]));
      int jn[U];
      if (k + U < w)
        fetch_idx(off, w, k + U, jn);
      else if (sn < g.nsl)
        fetch_idx(off_n, w_n, 0, jn);
      else
#pragma unroll
        for (int u = 0; u < U; ++u) jn[u] = -1;
#pragma unroll
      for (int u = 0; u < U; ++u)
        if (jj[u] >= 0) {
#if !POLAR_SELL_DEG_INDPTR
          ++deg;
#endif
          if (go)
#pragma unroll
            for (int v = 0; v < CPL; ++v) acc[v] += (A)xv[u][v];
        }
#pragma unroll
      for (int u = 0; u < U; ++u) jj[u] = jn[u];
    }
    if (w == 0 && sn < g.nsl) fetch_idx(off_n, w_n, 0, jj);
    row_end(row, deg, acc, xi, go);
    off = off_n;
    w = w_n;
    row = row_n;
  }
}

// The slice pass with its gathers in flight as cp.async copies into a per-lane ring in
// shared memory (`ring`: this warp's POLAR_SELL_STAGES * U * 32 * LB bytes, laid out
// [stage][u][lane] so that each batch is written and read conflict-free), so that no
// register holds a gather in flight: the next batch (of this slice, or the next slice's
// first) is issued before the current one is waited for and summed.  Each lane reads only
// what it copied, so no barrier is needed; the sums are formed in the same order as
// sell_slice_pass, so results are identical.
template <typename T, int CPL, typename A, typename RowEnd>
POLAR_D void sell_slice_pass_async(const polar_graph& g, const RowGroup& rg, int wid, int nw, const T* X, int ldx,
                                   bool on, const GatherHints& hp, unsigned char* ring, RowEnd&& row_end) {
  constexpr int LB = CPL * (int)sizeof(T);
  constexpr int U = (POLAR_SELL_BYTES / LB) > 1 ? (POLAR_SELL_BYTES / LB) : 1;
  constexpr int NC = LB / 16;  // 16-byte copies per lane per gathered row
  constexpr int NS = POLAR_SELL_STAGES;
  static_assert(LB % 16 == 0, "lane share of a row must be whole 16-byte copies");
  const int lane = threadIdx.x & 31;
  const int grp = lane / rg.G;
  const int S = 32 / rg.G;
  auto slot = [&](int stage, int u, int c) -> unsigned char* {
    return ring + ((size_t)((stage * U + u) * NC + c) * 32 + lane) * 16;
  };
  auto fetch_desc = [&](int sl, int& o, int& wd, int& r) {
    o = __ldg(g.d_sl_off + sl);
    wd = (__ldg(g.d_sl_off + sl + 1) - o) / S;
    r = __ldg(g.d_sl_rows + (size_t)sl * S + grp);
  };
  auto fetch_idx = [&](int o, int wd, int k, int (&dst)[U]) {
    const int* sp = g.d_sl_idx + o + grp;
#pragma unroll
    for (int u = 0; u < U; ++u) dst[u] = (k + u < wd) ? ld_hint_i32(sp + (size_t)(k + u) * S, hp.stream) : -1;
  };
  auto issue = [&](const int (&jj)[U], bool go, int stage) {
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const bool ok = go && jj[u] >= 0;
      const T* src = ok ? X + (size_t)jj[u] * ldx + rg.col : X;
#pragma unroll
      for (int c = 0; c < NC; ++c)
        cp_async16(slot(stage, u, c), reinterpret_cast<const unsigned char*>(src) + 16 * c, ok ? 16 : 0);
    }
    cp_async_commit();
  };
  int off = 0, w = 0, row = -1;
  int jj[U];
  int stage = 0;
  if (wid < g.nsl) {
    fetch_desc(wid, off, w, row);
    fetch_idx(off, w, 0, jj);
    issue(jj, row >= 0 && on, 0);
  }
  for (int sl = wid; sl < g.nsl; sl += nw) {
    const int sn = sl + nw;
    int off_n = 0, w_n = 0, row_n = -1;
    if (sn < g.nsl) fetch_desc(sn, off_n, w_n, row_n);
    const bool go = row >= 0 && on;
    T xi[CPL];
    if (go) vload_hint<T, CPL>(xi, X + (size_t)row * ldx + rg.col, hp.row(row));
    A acc[CPL];
#pragma unroll
    for (int v = 0; v < CPL; ++v) acc[v] = A(0);
    int deg = 0;
    const int nb = w > 0 ? (w + U - 1) / U : 1;  // an empty slice still owns its one issued batch
    for (int b = 0; b < nb; ++b) {
      // issue the following batch: this slice's next, or the next slice's first
      int jn[U];
      const int nst = (stage + 1) % NS;
      if (b + 1 < nb) {
        fetch_idx(off, w, (b + 1) * U, jn);
        issue(jn, go, nst);
      } else if (sn < g.nsl) {
        fetch_idx(off_n, w_n, 0, jn);
        issue(jn, row_n >= 0 && on, nst);
      } else {
#pragma unroll
        for (int u = 0; u < U; ++u) jn[u] = -1;
        cp_async_commit();  // empty group keeps one group per batch
      }
      cp_async_wait<1>();  // the current batch has landed
#pragma unroll
      for (int u = 0; u < U; ++u)
        if (jj[u] >= 0) {
          ++deg;
          if (go) {
            T xv[CPL];
#pragma unroll
            for (int c = 0; c < NC; ++c) {
              VecU<T, 16 / (int)sizeof(T)> q;
              q.v = *reinterpret_cast<const typename VecType<T, 16 / (int)sizeof(T)>::type*>(slot(stage, u, c));
#pragma unroll
              for (int e = 0; e < 16 / (int)sizeof(T); ++e) xv[c * (16 / (int)sizeof(T)) + e] = q.a[e];
            }
#pragma unroll
            for (int v = 0; v < CPL; ++v) acc[v] += (A)xv[v];
          }
        }
#pragma unroll
      for (int u = 0; u < U; ++u) jj[u] = jn[u];
      stage = nst;
    }
    row_end(row, deg, acc, xi, go);
    off = off_n;
    w = w_n;
    row = row_n;
  }
  cp_async_wait<0>();
}

}  // namespace polar
