// Shared state and device helpers of the multi-shift CG solvers (sm_100a):
// parameter block, deterministic column reductions, and the deferred shifted update.
#pragma once
#include "common.cuh"
#include "graph_ops.cuh"

namespace polar {

constexpr int kBlock = 512;
constexpr int kWarps = kBlock / 32;
constexpr int kMaxLd = 128;
constexpr int kHist = 16;  // M: iterations per deferred shifted-update pass
constexpr int kNC = 2 + 2 * kHist;     // composed coefficients per (pole, column)
constexpr int kMaxHeavyCtas = 1024;    // bound of the heavy-row launch (partials buffer rows)
#ifndef POLAR_E32
#define POLAR_E32 2  // active rows per thread in the deferred update, FP32 iterates
#endif
#ifndef POLAR_E64
#define POLAR_E64 1  // same, FP64 iterates
#endif

template <typename T> struct SolvePrm {
  polar_graph g;
  int n, R, ld, p, nA;
  double tol;
  long long maxit;
  int track;
  const double* W;
  int ldw;
  const double* tau;
  const int* active;
  const int* active_pos;
  void* Xout;
  int x_f32, ldx;
  double* h_out;
  long long* iters_out;
  // workspace.  The residual r and the direction recurrence are kept to FP64 accuracy in
  // every precision: rounding either to FP32 every iteration breaks the local
  // orthogonality and conjugacy of the CG recurrence enough to cost ~25 % more iterations
  // on badly conditioned Laplacians.  d is the SpMM's gathered input in T.  With
  // T = float the direction is the pair d + dlo (dlo = the FP32 remainder of the FP64
  // value, 48 significant bits together), so the SpMM reads d alone and the recurrence
  // reads both; dlo == nullptr: d is the direction itself.  v, the history and the
  // shifted iterates are T.
  double* r;
  float* r32;  // mixed precision with a rounded residual: r in FP32 here (r unused); else null
  float* dlo;
  T *d, *v, *hist, *Pb, *Xb;
  typename AccOf<T>::type* chunk_part;
  int* hcount;
  double* part;
  double* part_h;  // per-CTA d.v partials of the heavy-row launch
  int nbh;         // CTAs of the heavy-row launch (0: none)
  double *rr, *stop, *ap, *bp, *ag, *beg, *chig;
  int *act, *upd;
  double *z, *zp, *hs, *ip, *pn;
  int *live, *pflag;
  T *ca, *cz, *cb;
  double* cmp;  // composed deferred-update coefficients per (pole, column): alpha, beta, gamma[M], delta[M]
  int* ctl;  // [0]=status [1]=err [2]=where [3]=any  [4..5]=barrier count/gen
  long long* stats;  // [0]=iterations [1]=flushes [2..7]=phase ns (CTA 0 view)
  uint64_t timeout_ns;
  // L2 policy of the kernel-per-phase driver: rows [0, hot_rows) of d are gathered and
  // stored with evict_last; l2_mode 0: no hints, 1: cold gathers evict_normal, streamed
  // data evict_first, 2: cold gathers evict_first as well.
  int hot_rows;
  int l2_mode;
};

// Policy for a gather or store of row i of d.
template <typename T>
POLAR_D uint64_t row_policy(const SolvePrm<T>& P, long long i, uint64_t hot, uint64_t cold) {
  return i < P.hot_rows ? hot : cold;
}

// Residual of one row item: the FP64 r, or the FP32 residual when r32 is set.
template <typename T, int VEC>
POLAR_D void load_res(const SolvePrm<T>& P, double (&out)[VEC], size_t o) {
  if (P.r32) {
    float t[VEC];
    vload<float, VEC>(t, P.r32 + o);
#pragma unroll
    for (int v = 0; v < VEC; ++v) out[v] = (double)t[v];
  } else {
    vload<double, VEC>(out, P.r + o);
  }
}

// Stores a residual row item; with r32 it is rounded first and `x` receives the stored
// value, so that norms and recurrences use the residual as stored.
template <typename T, int VEC>
POLAR_D void store_res(const SolvePrm<T>& P, double (&x)[VEC], size_t o) {
  if (P.r32) {
    float t[VEC];
#pragma unroll
    for (int v = 0; v < VEC; ++v) {
      t[v] = (float)x[v];
      x[v] = (double)t[v];
    }
    vstore<float, VEC>(P.r32 + o, t);
  } else {
    vstore<double, VEC>(P.r + o, x);
  }
}

// Direction of one row item in FP64: d (+ dlo when the remainder is kept).  store_dir
// writes d = (T)x and, with a remainder, dlo = (float)(x - d).
template <typename T, int VEC>
POLAR_D void load_dir(const SolvePrm<T>& P, double (&out)[VEC], size_t o) {
  T hi[VEC];
  vload<T, VEC>(hi, P.d + o);
#pragma unroll
  for (int v = 0; v < VEC; ++v) out[v] = (double)hi[v];
  if (P.dlo) {
    float lo[VEC];
    vload<float, VEC>(lo, P.dlo + o);
#pragma unroll
    for (int v = 0; v < VEC; ++v) out[v] += (double)lo[v];
  }
}

template <typename T, int VEC>
POLAR_D void store_dir(const SolvePrm<T>& P, const double (&in)[VEC], size_t o) {
  T hi[VEC];
#pragma unroll
  for (int v = 0; v < VEC; ++v) hi[v] = (T)in[v];
  vstore<T, VEC>(P.d + o, hi);
  if (P.dlo) {
    float lo[VEC];
#pragma unroll
    for (int v = 0; v < VEC; ++v) lo[v] = (float)(in[v] - (double)hi[v]);
    vstore<float, VEC>(P.dlo + o, lo);
  }
}

// store_dir with L2 policies: `dpol` for the SpMM's copy d (evict_last on the gathered
// prefix keeps it resident into the next SpMM), `lopol` for the remainder.
template <typename T, int VEC>
POLAR_D void store_dir_hint(const SolvePrm<T>& P, const double (&in)[VEC], size_t o, uint64_t dpol, uint64_t lopol) {
  T hi[VEC];
#pragma unroll
  for (int v = 0; v < VEC; ++v) hi[v] = (T)in[v];
  vstore_hint<T, VEC>(P.d + o, hi, dpol);
  if (P.dlo) {
    float lo[VEC];
#pragma unroll
    for (int v = 0; v < VEC; ++v) lo[v] = (float)(in[v] - (double)hi[v]);
    vstore_hint<float, VEC>(P.dlo + o, lo, lopol);
  }
}

// ---------------------------------------------------------------------------------------
template <int VEC>
POLAR_D void reduce_cols_to_part(double (&acc)[VEC], int G, int ld, double* red, double* out_row) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int o = G; o < 32; o <<= 1)
#pragma unroll
    for (int v = 0; v < VEC; ++v) acc[v] += __shfl_xor_sync(0xffffffffu, acc[v], o);
  if (lane < G)
#pragma unroll
    for (int v = 0; v < VEC; ++v) red[warp * ld + lane * VEC + v] = acc[v];
  __syncthreads();
  for (int c = threadIdx.x; c < ld; c += blockDim.x) {
    double s = 0.0;
    for (int w = 0; w < kWarps; ++w) s += red[w * ld + c];
    out_row[c] = s;
  }
}

// Sum of per-CTA partials part[b][c] over b in a fixed order (deterministic).
POLAR_D void reduce_partials(const double* part, int nblk, int ld, double* tmp, double* out) {
  const int S = blockDim.x / ld;
  const int t = threadIdx.x, c = t % ld, s = t / ld;
  if (s < S) {
    // strip s sums blocks s, s + S, ... in that order; eight loads are issued before the
    // adds so the strip costs about one L2 round trip per eight partials
    constexpr int B = 8;
    double acc = 0.0;
    for (int b0 = s; b0 < nblk; b0 += B * S) {
      double v[B];
#pragma unroll
      for (int u = 0; u < B; ++u) {
        const int b = b0 + u * S;
        v[u] = b < nblk ? __ldcg(part + (size_t)b * ld + c) : 0.0;
      }
#pragma unroll
      for (int u = 0; u < B; ++u) acc += v[u];
    }
    tmp[s * ld + c] = acc;
  }
  __syncthreads();
  if (t < ld) {
    double acc = 0.0;
    for (int s2 = 0; s2 < S; ++s2) acc += tmp[s2 * ld + t];
    out[t] = acc;
  }
  __syncthreads();
}

// Sum red[warp][c] over the CTA's warps in order -> this CTA's partial row.
POLAR_D void reduce_red_to_part(const double* red, int ld, double* out_row) {
  __syncthreads();
  for (int c = threadIdx.x; c < ld; c += blockDim.x) {
    double s = 0.0;
    for (int w = 0; w < kWarps; ++w) s += red[w * ld + c];
    out_row[c] = s;
  }
}

// ---------------------------------------------------------------------------------------
// Deferred shifted update over `nsteps` recorded iterations.  Thread item = (tile of E
// active rows, column c); the E rows share the per-(pole, step, column) coefficients and
// the history values stay in registers across all poles.  Poles are double-buffered: the
// loads of pole j+1 are in flight while pole j is updated.
template <typename T, int E>
struct PoleBuf {
  T x[E], p[E];
  bool on;
};

template <typename T, int E>
POLAR_D void pole_load(const SolvePrm<T>& P, PoleBuf<T, E>& b, int j, int a0, int c, int nsteps, bool first,
                       bool final_pass, const T (&w0)[E]) {
  const int ld = P.ld, nA = P.nA;
  b.on = P.pflag[j * ld + c] != 0 && nsteps > 0;
  const bool need = first || final_pass || b.on;
  const size_t base = ((size_t)j * nA + a0) * ld + c;
#pragma unroll
  for (int e = 0; e < E; ++e) {
    const bool ok = need && a0 + e < nA;
    b.x[e] = first ? T(0) : (ok ? P.Xb[base + (size_t)e * ld] : T(0));
    b.p[e] = first ? w0[e] : ((ok && b.on) ? P.Pb[base + (size_t)e * ld] : T(0));
  }
}

template <typename T, int E>
POLAR_D void pole_apply(const SolvePrm<T>& P, PoleBuf<T, E>& b, int j, int a0, int c, int nsteps, bool first,
                        bool final_pass, const T (&hv)[E][kHist]) {
  const int ld = P.ld, nA = P.nA, p = P.p;
  if (!first && !final_pass && !b.on) return;
  const size_t base = ((size_t)j * nA + a0) * ld + c;
  if (b.on) {
#pragma unroll
    for (int k = 0; k < kHist; ++k) {
      if (k < nsteps) {
        const size_t ci = ((size_t)k * p + j) * ld + c;
        const T aj = P.ca[ci], zn = P.cz[ci], bj = P.cb[ci];
        if (aj != T(0) || zn != T(0)) {
#pragma unroll
          for (int e = 0; e < E; ++e) {
            b.x[e] = fma(aj, b.p[e], b.x[e]);
            b.p[e] = fma(zn, hv[e][k], bj * b.p[e]);
          }
        }
      }
    }
    if (!final_pass) {
#pragma unroll
      for (int e = 0; e < E; ++e)
        if (a0 + e < nA) P.Pb[base + (size_t)e * ld] = b.p[e];
    }
  }
  if (final_pass) {
    if (c < P.R) {
#pragma unroll
      for (int e = 0; e < E; ++e) {
        if (a0 + e < nA) {
          const size_t o = ((size_t)j * nA + a0 + e) * P.ldx + c;
          if (P.x_f32) reinterpret_cast<float*>(P.Xout)[o] = (float)b.x[e];
          else reinterpret_cast<double*>(P.Xout)[o] = (double)b.x[e];
        }
      }
    }
  } else {
#pragma unroll
    for (int e = 0; e < E; ++e)
      if (a0 + e < nA) P.Xb[base + (size_t)e * ld] = b.x[e];
  }
}

template <typename T, int E>
POLAR_D void shifted_update(const SolvePrm<T>& P, int nsteps, bool first, bool final_pass, long long tid,
                            long long nth) {
  const int ld = P.ld, nA = P.nA, p = P.p;
  const int ntile = (nA + E - 1) / E;
  const long long items = (long long)ntile * ld;
  for (long long item = tid; item < items; item += nth) {
    const int tile = (int)(item / ld), c = (int)(item % ld);
    const int a0 = tile * E;
    T hv[E][kHist];
#pragma unroll
    for (int e = 0; e < E; ++e)
#pragma unroll
      for (int k = 0; k < kHist; ++k)
        hv[e][k] = (k < nsteps && a0 + e < nA) ? P.hist[((size_t)k * nA + a0 + e) * ld + c] : T(0);
    T w0[E];
#pragma unroll
    for (int e = 0; e < E; ++e)
      w0[e] = (first && a0 + e < nA && c < P.R) ? (T)__ldg(P.W + (size_t)__ldg(P.active + a0 + e) * P.ldw + c)
                                                : T(0);
    PoleBuf<T, E> A, B;
    pole_load<T, E>(P, A, 0, a0, c, nsteps, first, final_pass, w0);
    for (int j = 0; j < p; j += 2) {
      if (j + 1 < p) pole_load<T, E>(P, B, j + 1, a0, c, nsteps, first, final_pass, w0);
      pole_apply<T, E>(P, A, j, a0, c, nsteps, first, final_pass, hv);
      if (j + 2 < p) pole_load<T, E>(P, A, j + 2, a0, c, nsteps, first, final_pass, w0);
      if (j + 1 < p) pole_apply<T, E>(P, B, j + 1, a0, c, nsteps, first, final_pass, hv);
    }
  }
}


// Block-cooperative deferred update.  CTA b owns the 128-byte column chunk
// cc = b % nch (CW columns) and strides over row tiles; it stages the chunk's step
// coefficients of every pole (3 x nsteps x p x CW values) in shared memory once, so the
// inner loop reads them from smem.  Thread = (column cl, E rows spaced blockDim/CW apart);
// a warp reads whole 128-byte row segments of X, P and the history.
template <typename T>
POLAR_HD int flush_cw(int ld) {
  const int cw = 128 / (int)sizeof(T);
  return ld < cw ? ld : cw;
}

template <typename T>
POLAR_HD size_t flush_smem_bytes(int ld, int p, int nsteps) {
  return (size_t)3 * nsteps * p * flush_cw<T>(ld) * sizeof(T);
}

template <typename T, int E>
POLAR_D void shifted_update_smem(const SolvePrm<T>& P, int nsteps, bool first, bool final_pass, T* sm) {
  const int ld = P.ld, nA = P.nA, p = P.p;
  const int cw = flush_cw<T>(ld);
  const int nch = ld / cw;
  const int cc = blockIdx.x % nch;
  const int bstride = gridDim.x / nch;
  const int brank = blockIdx.x / nch;
  const int cl = threadIdx.x % cw;
  const int rthr = threadIdx.x / cw;
  const int rows_per_pass = blockDim.x / cw;
  const int TR = rows_per_pass * E;
  const int c = cc * cw + cl;
  // stage coefficients: sm[plane][k][j][cl]
  const int per_plane = nsteps * p * cw;
  for (int i = threadIdx.x; i < per_plane; i += blockDim.x) {
    const int l = i % cw;
    const int kj = i / cw;  // k * p + j
    const size_t gi = (size_t)kj * ld + cc * cw + l;
    sm[i] = P.ca[gi];
    sm[per_plane + i] = P.cz[gi];
    sm[2 * per_plane + i] = P.cb[gi];
  }
  __syncthreads();
  const T* sa = sm;
  const T* sz = sm + per_plane;
  const T* sb = sm + 2 * per_plane;
  const int ntile = (nA + TR - 1) / TR;
  T w0[E];
  for (int tile = brank; tile < ntile; tile += bstride) {
    int arow[E];
#pragma unroll
    for (int e = 0; e < E; ++e) arow[e] = tile * TR + rthr + e * rows_per_pass;
    T hv[E][kHist];
#pragma unroll
    for (int e = 0; e < E; ++e)
#pragma unroll
      for (int k = 0; k < kHist; ++k)
        hv[e][k] = (k < nsteps && arow[e] < nA) ? P.hist[((size_t)k * nA + arow[e]) * ld + c] : T(0);
#pragma unroll
    for (int e = 0; e < E; ++e)
      w0[e] = (first && arow[e] < nA && c < P.R) ? (T)__ldg(P.W + (size_t)__ldg(P.active + arow[e]) * P.ldw + c)
                                                 : T(0);
    T xa[E], pa[E], xb[E], pb[E];
    bool ona = false, onb = false;
    auto load = [&](int j, T (&x)[E], T (&pv)[E], bool& on) {
      on = P.pflag[j * ld + c] != 0 && nsteps > 0;
      const bool need = first || final_pass || on;
#pragma unroll
      for (int e = 0; e < E; ++e) {
        const bool ok = need && arow[e] < nA;
        const size_t o = ((size_t)j * nA + arow[e]) * ld + c;
        x[e] = first ? T(0) : (ok ? P.Xb[o] : T(0));
        pv[e] = first ? w0[e] : ((ok && on) ? P.Pb[o] : T(0));
      }
    };
    auto apply = [&](int j, T (&x)[E], T (&pv)[E], bool on) {
      if (!first && !final_pass && !on) return;
      if (on) {
#pragma unroll
        for (int k = 0; k < kHist; ++k) {
          if (k < nsteps) {
            const int si = (k * p + j) * cw + cl;
            const T aj = sa[si], zn = sz[si], bj = sb[si];
            if (aj != T(0) || zn != T(0)) {
#pragma unroll
              for (int e = 0; e < E; ++e) {
                x[e] = fma(aj, pv[e], x[e]);
                pv[e] = fma(zn, hv[e][k], bj * pv[e]);
              }
            }
          }
        }
        if (!final_pass)
#pragma unroll
          for (int e = 0; e < E; ++e)
            if (arow[e] < nA) P.Pb[((size_t)j * nA + arow[e]) * ld + c] = pv[e];
      }
      if (final_pass) {
        if (c < P.R)
#pragma unroll
          for (int e = 0; e < E; ++e)
            if (arow[e] < nA) {
              const size_t o = ((size_t)j * nA + arow[e]) * P.ldx + c;
              if (P.x_f32) reinterpret_cast<float*>(P.Xout)[o] = (float)x[e];
              else reinterpret_cast<double*>(P.Xout)[o] = (double)x[e];
            }
      } else {
#pragma unroll
        for (int e = 0; e < E; ++e)
          if (arow[e] < nA) P.Xb[((size_t)j * nA + arow[e]) * ld + c] = x[e];
      }
    };
    load(0, xa, pa, ona);
    for (int j = 0; j < p; j += 2) {
      if (j + 1 < p) load(j + 1, xb, pb, onb);
      apply(j, xa, pa, ona);
      if (j + 2 < p) load(j + 2, xa, pa, ona);
      if (j + 1 < p) apply(j + 1, xb, pb, onb);
    }
  }
}

// Deferred update from the composed coefficients: for each pole j and element,
//   X <- X + alpha P + sum_k gamma_k h_k,   P <- beta P + sum_k delta_k h_k
// (2 + 2M fused multiply-adds, no per-step branches; unused steps have zero coefficients
// and the history is zeroed per solve).  CTA = 128-byte column chunk as above; the chunk's
// coefficients of all poles are staged in shared memory as T, one row per (pole, column).
//
// Shared-memory row of one (pole, column) in the composed flush: gamma_k, delta_k
// interleaved for k = 0..M-1, then alpha, beta; padded so that a lane's row starts 16-byte
// aligned and the rows of 8 consecutive lanes fall on distinct banks (36 floats, 34 doubles:
// 4-word lane stride mod 32), which makes every coefficient read one conflict-free 128-bit
// shared load of two (FP32) or one (FP64) history steps' pair.
template <typename T>
POLAR_HD constexpr int composed_row() {
  return sizeof(T) == 4 ? 36 : 34;
}

template <typename T>
POLAR_HD size_t composed_smem_bytes(int ld, int p) {
  return (size_t)p * flush_cw<T>(ld) * composed_row<T>() * sizeof(T);
}

#ifndef POLAR_FLUSH_F64
#define POLAR_FLUSH_F64 0  // 1: FP32 iterates are updated with FP64 arithmetic in the flush
#endif
template <typename T> struct FlushAcc { using type = T; };
#if POLAR_FLUSH_F64
template <> struct FlushAcc<float> { using type = double; };
#endif

template <typename T, int E>
POLAR_D void shifted_update_composed(const SolvePrm<T>& P, int nsteps, bool first, bool final_pass, T* sm) {
  // X, P and the history stream through once per pass: evict-first loads and stores keep
  // the CG vectors and the graph in L2 across the pass
  using C = typename FlushAcc<T>::type;
  const int ld = P.ld, nA = P.nA, p = P.p;
  const int cw = flush_cw<T>(ld);
  const int nch = ld / cw;
  const int cc = blockIdx.x % nch;
  const int bstride = gridDim.x / nch;
  const int brank = blockIdx.x / nch;
  const int cl = threadIdx.x % cw;
  const int rthr = threadIdx.x / cw;
  const int rows_per_pass = blockDim.x / cw;
  const int TR = rows_per_pass * E;
  const int c = cc * cw + cl;
  // composed coefficients of this CTA's columns, in the composed_row layout: source t = 0
  // alpha, 1 beta, 2 + k gamma_k, 2 + M + k delta_k
  constexpr int NR = composed_row<T>();
  const int total = p * kNC * cw;
  for (int i = threadIdx.x; i < total; i += blockDim.x) {
    const int t = i % kNC;
    const int jl = i / kNC;  // j * cw + l
    const int j = jl / cw, l = jl % cw;
    const int dst = t == 0 ? 2 * kHist : t == 1 ? 2 * kHist + 1
                  : t < 2 + kHist ? 2 * (t - 2) : 2 * (t - 2 - kHist) + 1;
    sm[(size_t)jl * NR + dst] = (T)P.cmp[((size_t)j * ld + cc * cw + l) * kNC + t];
  }
  __syncthreads();
  const int ntile = (nA + TR - 1) / TR;
  for (int tile = brank; tile < ntile; tile += bstride) {
    int arow[E];
#pragma unroll
    for (int e = 0; e < E; ++e) arow[e] = tile * TR + rthr + e * rows_per_pass;
    T hv[E][kHist];
#pragma unroll
    for (int e = 0; e < E; ++e)
#pragma unroll
      for (int k = 0; k < kHist; ++k)
        hv[e][k] = arow[e] < nA ? __ldcs(P.hist + ((size_t)k * nA + arow[e]) * ld + c) : T(0);
    T w0[E];
#pragma unroll
    for (int e = 0; e < E; ++e)
      w0[e] = (first && arow[e] < nA && c < P.R) ? (T)__ldg(P.W + (size_t)__ldg(P.active + arow[e]) * P.ldw + c)
                                                 : T(0);
    // poles double-buffered: the X/P loads of pole j+1 are in flight while pole j runs
    auto load = [&](int j, T (&x)[E], T (&pv)[E], bool& on) {
      on = nsteps > 0 && P.pflag[j * ld + c] != 0;
      const bool need = first || final_pass || on;
#pragma unroll
      for (int e = 0; e < E; ++e) {
        const bool ok = need && arow[e] < nA;
        const size_t o = ((size_t)j * nA + arow[e]) * ld + c;
        x[e] = first ? T(0) : (ok ? __ldcs(P.Xb + o) : T(0));
        pv[e] = first ? w0[e] : ((ok && on) ? __ldcs(P.Pb + o) : T(0));
      }
    };
    auto apply = [&](int j, T (&x)[E], T (&pv)[E], bool on) {
      if (!first && !final_pass && !on) return;
      if (on) {
        const T* cf = sm + ((size_t)j * cw + cl) * NR;
        constexpr int V = 16 / (int)sizeof(T);  // coefficients per 128-bit shared load
        VecU<T, 2> ab;
        ab.v = *reinterpret_cast<const typename VecType<T, 2>::type*>(cf + 2 * kHist);
        const C alpha = (C)ab.a[0], beta = (C)ab.a[1];
        C xc[E], pc[E];
#pragma unroll
        for (int e = 0; e < E; ++e) {
          const C p0 = (C)pv[e];
          xc[e] = fma(alpha, p0, (C)x[e]);
          pc[e] = beta * p0;
        }
#pragma unroll
        for (int k0 = 0; k0 < 2 * kHist; k0 += V) {
          VecU<T, V> q;
          q.v = *reinterpret_cast<const typename VecType<T, V>::type*>(cf + k0);
#pragma unroll
          for (int u = 0; u < V; u += 2) {
            const int k = (k0 + u) / 2;
            const C gk = (C)q.a[u], dk = (C)q.a[u + 1];
#pragma unroll
            for (int e = 0; e < E; ++e) {
              xc[e] = fma(gk, (C)hv[e][k], xc[e]);
              pc[e] = fma(dk, (C)hv[e][k], pc[e]);
            }
          }
        }
#pragma unroll
        for (int e = 0; e < E; ++e) {
          x[e] = (T)xc[e];
          pv[e] = (T)pc[e];
        }
        if (!final_pass)
#pragma unroll
          for (int e = 0; e < E; ++e)
            if (arow[e] < nA) __stcs(P.Pb + ((size_t)j * nA + arow[e]) * ld + c, pv[e]);
      }
      if (final_pass) {
        if (c < P.R)
#pragma unroll
          for (int e = 0; e < E; ++e)
            if (arow[e] < nA) {
              const size_t o = ((size_t)j * nA + arow[e]) * P.ldx + c;
              if (P.x_f32) reinterpret_cast<float*>(P.Xout)[o] = (float)x[e];
              else reinterpret_cast<double*>(P.Xout)[o] = (double)x[e];
            }
      } else {
#pragma unroll
        for (int e = 0; e < E; ++e)
          if (arow[e] < nA) __stcs(P.Xb + ((size_t)j * nA + arow[e]) * ld + c, x[e]);
      }
    };
    T xa[E], pa[E], xb[E], pb[E];
    bool ona = false, onb = false;
    load(0, xa, pa, ona);
    for (int j = 0; j < p; j += 2) {
      if (j + 1 < p) load(j + 1, xb, pb, onb);
      apply(j, xa, pa, ona);
      if (j + 2 < p) load(j + 2, xa, pa, ona);
      if (j + 1 < p) apply(j + 1, xb, pb, onb);
    }
  }
}

// One iteration of the zeta recurrence, the three-scalar norm tracker and pole freezing
// for item q = (pole j, column c) (realworld/polar_gpu.py:107-120); writes this step's
// deferred-update coefficients (identity when the pole or column is inactive).
template <typename T>
POLAR_D void pole_step(const SolvePrm<T>& P, long long q, int slot, double shift0) {
  const int ld = P.ld, p = P.p;
  const int j = (int)(q / ld), c = (int)(q % ld);
  const bool m = P.live[q] && P.upd[c];
  const size_t ci = ((size_t)slot * p + j) * ld + c;
  int pf = slot == 0 ? 0 : P.pflag[q];
  if (m) {
    const double theta = __ldg(P.tau + j) - shift0;
    const double a = P.ag[c], be = P.beg[c], chi = P.chig[c], rrn = P.rr[c];
    const double z = P.z[q], zp = P.zp[q];
    const double zn = z / (1.0 + a * theta + chi * (1.0 - z / zp));
    const double fac = zn / z;
    const double aj = a * fac;
    const double bj = be * fac * fac;
    P.ca[ci] = (T)aj;
    P.cz[ci] = (T)zn;
    P.cb[ci] = (T)bj;
    if (P.track) {
      const double ipv = P.ip[q], pnv = P.pn[q];
      P.hs[q] += 2.0 * aj * ipv + aj * aj * pnv;
      P.ip[q] = bj * (ipv + aj * pnv);
      P.pn[q] = zn * zn * rrn + bj * bj * pnv;
    }
    P.zp[q] = z;
    P.z[q] = zn;
    if (fabs(zn) * sqrt(rrn) <= P.stop[c]) P.live[q] = 0;
    pf = 1;
    if (P.cmp) {
      // compose this step into the block's closed form:
      //   X_{k+1} = X_k + aj P_k,  P_{k+1} = zn h_k + bj P_k
      double* cq = P.cmp + (size_t)q * kNC;
      if (slot == 0) {
        cq[0] = 0.0;
        cq[1] = 1.0;
        for (int i = 0; i < 2 * kHist; ++i) cq[2 + i] = 0.0;
      }
      double beta = cq[1];
      cq[0] += aj * beta;
      for (int i = 0; i < slot; ++i) {
        const double di = cq[2 + kHist + i];
        cq[2 + i] += aj * di;
        cq[2 + kHist + i] = bj * di;
      }
      cq[1] = bj * beta;
      cq[2 + kHist + slot] = zn;
    }
  } else {
    P.ca[ci] = T(0);
    P.cz[ci] = T(0);
    P.cb[ci] = T(1);
    if (P.cmp && slot == 0) {
      double* cq = P.cmp + (size_t)q * kNC;
      cq[0] = 0.0;
      cq[1] = 1.0;
      for (int i = 0; i < 2 * kHist; ++i) cq[2 + i] = 0.0;
    }
  }
  P.pflag[q] = pf;
}

// pole_step split over the kHist (= 16) lanes of a half-warp: lane i of the half-warp that
// holds item q forms the item's step scalars (the same arithmetic as pole_step) and
// updates only its own composed pair (gamma_i, delta_i); lane 0 also advances the item's
// recurrence state, this slot's bookkeeping and the coefficient planes, after every lane
// has read the state (half-warp sync on `hmask`).  Requires P.cmp and kHist == 16.
template <typename T>
POLAR_D void pole_step_unit(const SolvePrm<T>& P, long long q, int i, unsigned hmask, int slot, double shift0) {
  static_assert(kHist == 16, "one half-warp per pole item");
  const int ld = P.ld;
  const int j = (int)(q / ld), c = (int)(q % ld);
  const bool m = P.live[q] && P.upd[c];
  double* cq = P.cmp + (size_t)q * kNC;
  const size_t ci = ((size_t)slot * P.p + j) * ld + c;
  if (!m) {
    if (slot == 0) {
      cq[2 + i] = 0.0;
      cq[2 + kHist + i] = 0.0;
      if (i == 0) {
        cq[0] = 0.0;
        cq[1] = 1.0;
      }
    }
    if (i == 0) {
      P.ca[ci] = T(0);
      P.cz[ci] = T(0);
      P.cb[ci] = T(1);
      if (slot == 0) P.pflag[q] = 0;
    }
    return;
  }
  const double theta = __ldg(P.tau + j) - shift0;
  const double a = P.ag[c], be = P.beg[c], chi = P.chig[c];
  const double z = P.z[q], zp = P.zp[q];
  const double zn = z / (1.0 + a * theta + chi * (1.0 - z / zp));
  const double fac = zn / z;
  const double aj = a * fac;
  const double bj = be * fac * fac;
  if (i < slot) {
    const double di = cq[2 + kHist + i];
    cq[2 + i] += aj * di;
    cq[2 + kHist + i] = bj * di;
  } else if (slot == 0) {
    cq[2 + i] = 0.0;
    if (i > 0) cq[2 + kHist + i] = 0.0;
  }
  __syncwarp(hmask);
  if (i != 0) return;
  const double beta = slot == 0 ? 1.0 : cq[1];
  cq[0] = (slot == 0 ? 0.0 : cq[0]) + aj * beta;
  cq[1] = bj * beta;
  cq[2 + kHist + slot] = zn;
  const double rrn = P.rr[c];
  P.ca[ci] = (T)aj;
  P.cz[ci] = (T)zn;
  P.cb[ci] = (T)bj;
  if (P.track) {
    const double ipv = P.ip[q], pnv = P.pn[q];
    P.hs[q] += 2.0 * aj * ipv + aj * aj * pnv;
    P.ip[q] = bj * (ipv + aj * pnv);
    P.pn[q] = zn * zn * rrn + bj * bj * pnv;
  }
  P.zp[q] = z;
  P.z[q] = zn;
  if (fabs(zn) * sqrt(rrn) <= P.stop[c]) P.live[q] = 0;
  P.pflag[q] = 1;
}

// Column scalars after the r.r reduction (realworld/polar_gpu.py:103-106, 121-125):
// beta, chi, direction-update mask, convergence.  Run by one CTA.  Returns (uniformly
// over the CTA) whether any column is still active.
template <typename T>
POLAR_D bool column_step(const SolvePrm<T>& P, const double* rrn_s) {
  int anyv = 0;
  for (int c = threadIdx.x; c < P.ld; c += blockDim.x) {
    const int a_on = P.act[c];
    const double rrn = rrn_s[c];
    const double a = P.ag[c];
    const double rr = P.rr[c];
    const double be = a_on ? rrn / rr : 0.0;
    P.chig[c] = a_on ? a * P.bp[c] / P.ap[c] : 0.0;
    P.upd[c] = a_on;
    P.beg[c] = be;
    if (a_on) {
      if (!isfinite(rrn)) atomicCAS(P.ctl + 1, 0, (int)POLAR_ERR_NONFINITE);
      P.rr[c] = rrn;
      P.ap[c] = a;
      P.bp[c] = be;
      const bool done = sqrt(rrn) <= P.stop[c];
      P.act[c] = done ? 0 : 1;
      anyv |= done ? 0 : 1;
      if (c < P.R) P.iters_out[c] += 1;
    }
  }
  return __syncthreads_or(anyv) != 0;
}

// Initial scalars from r.r of the right-hand sides (realworld/polar_gpu.py:93-99).
template <typename T>
POLAR_D bool init_step(const SolvePrm<T>& P, const double* rr_s) {
  const int ld = P.ld, p = P.p;
  int anyv = 0;
  for (int c = threadIdx.x; c < ld; c += blockDim.x) {
    const double rr = rr_s[c];
    if (!isfinite(rr)) atomicCAS(P.ctl + 1, 0, (int)POLAR_ERR_NONFINITE);
    const int a = rr > 0.0 ? 1 : 0;
    P.rr[c] = rr;
    P.stop[c] = P.tol * sqrt(rr);
    P.act[c] = a;
    P.upd[c] = 0;
    P.ap[c] = 1.0;
    P.bp[c] = 0.0;
    P.ag[c] = 0.0;
    P.beg[c] = 0.0;
    P.chig[c] = 0.0;
    anyv |= a;
  }
  for (int it = threadIdx.x; it < p * ld; it += blockDim.x) {
    const double rr = rr_s[it % ld];
    P.z[it] = 1.0;
    P.zp[it] = 1.0;
    P.live[it] = rr > 0.0 ? 1 : 0;
    P.hs[it] = 0.0;
    P.ip[it] = 0.0;
    P.pn[it] = rr;
    P.pflag[it] = 0;
  }
  return __syncthreads_or(anyv) != 0;
}

}  // namespace polar
