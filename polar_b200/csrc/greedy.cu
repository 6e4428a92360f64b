// Greedy-round kernels of POLAR (sm_100a): incidence right-hand sides, bank caches,
// proxy score + stable top-B, re-rank, Sherman–Morrison maintenance and the F update.
// All are HBM-bound gathers/streams; they keep every selection on the device, so a
// round needs one small device->host read (the winner) and nothing else.
#include <cuda_runtime.h>

#include <cfloat>
#include <cmath>

#include "common.cuh"
#include "host_util.h"

namespace polar {

template <typename T>
POLAR_D double ldx(const void* p, size_t i) {
  return (double)reinterpret_cast<const T*>(p)[i];
}
POLAR_D double ldv(const void* p, int f32, size_t i) { return f32 ? ldx<float>(p, i) : ldx<double>(p, i); }

// ---------------------------------------------------------------------------------------
// W[:, c] = e_a - e_b with (a, b) = cand[sel[c]]; ia/ib = endpoint active positions.
__global__ void fill_incidence_kernel(int R, const int64_t* cand, const int64_t* sel, const int32_t* es,
                                      double* W, int ldw, int32_t* ia, int32_t* ib) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= R) return;
  const int64_t e = sel[c];
  W[(size_t)cand[2 * e] * ldw + c] = 1.0;
  W[(size_t)cand[2 * e + 1] * ldw + c] = -1.0;
  if (ia) ia[c] = es[2 * e];
  if (ib) ib[c] = es[2 * e + 1];
}

// ---------------------------------------------------------------------------------------
// out[j][e] = sum_c (X[j][ea][col0+c] - X[j][eb][col0+c])^2 ; 16 lanes per (j, e).
template <typename T>
__global__ void pair_norms_kernel(const T* X, int p, int nA, int ldx, int col0, int q, const int32_t* ea,
                                  const int32_t* eb, int N, double* out) {
  const int lanes = 16;
  const long long gidx = ((long long)blockIdx.x * blockDim.x + threadIdx.x) / lanes;
  const int lg = threadIdx.x & (lanes - 1);
  const unsigned mask = 0xffffu << (threadIdx.x & 16);
  const long long total = (long long)p * N;
  if (gidx >= total) return;
  const int j = (int)(gidx / N), e = (int)(gidx % N);
  const T* xa = X + ((size_t)j * nA + ea[e]) * ldx + col0;
  const T* xb = X + ((size_t)j * nA + eb[e]) * ldx + col0;
  double s = 0.0;
  for (int c = lg; c < q; c += lanes) {
    const double dlt = (double)xa[c] - (double)xb[c];
    s += dlt * dlt;
  }
  for (int o = 8; o > 0; o >>= 1) s += __shfl_xor_sync(mask, s, o);
  if (lg == 0) out[(size_t)j * N + e] = s;
}

// ---------------------------------------------------------------------------------------
// Stable top-B: key order (score descending, index ascending).
POLAR_D bool better(double s1, long long i1, double s2, long long i2) {
  return s1 > s2 || (s1 == s2 && i1 < i2);
}

constexpr int kTopBlock = 256;
constexpr int kTopPer = 2;  // elements per thread in the scoring and merge passes
constexpr int kMaxB = 64;

struct Cand {
  double s;
  long long i;
};

POLAR_D Cand warp_best(Cand c) {
  for (int o = 16; o > 0; o >>= 1) {
    const double s2 = __shfl_xor_sync(0xffffffffu, c.s, o);
    const long long i2 = __shfl_xor_sync(0xffffffffu, c.i, o);
    if (better(s2, i2, c.s, c.i)) {
      c.s = s2;
      c.i = i2;
    }
  }
  return c;
}

// Block-wide argmax by (score, index); all threads get the result.
POLAR_D Cand block_best(Cand c, Cand* sh) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  c = warp_best(c);
  if (lane == 0) sh[warp] = c;
  __syncthreads();
  if (warp == 0) {
    Cand d = lane < (int)(blockDim.x >> 5) ? sh[lane] : Cand{-INFINITY, LLONG_MAX};
    d = warp_best(d);
    if (lane == 0) sh[32] = d;
  }
  __syncthreads();
  Cand r = sh[32];
  __syncthreads();
  return r;
}

__global__ void __launch_bounds__(kTopBlock) score_block_topb_kernel(const double* h, const double* t,
                                                                     const double* tau, const double* om, double sigma,
                                                                     int p, int N, const uint8_t* live, int obj, int B,
                                                                     double* score_all, Cand* blk) {
  __shared__ Cand sh[33];
  const long long base = (long long)blockIdx.x * kTopBlock * kTopPer;
  double s[kTopPer];
  long long idx[kTopPer];
#pragma unroll
  for (int k = 0; k < kTopPer; ++k) {
    const long long e = base + (long long)k * kTopBlock + threadIdx.x;
    idx[k] = e;
    double v = -INFINITY;
    if (e < N) {
      if (obj == 1) {
        v = log1p(t[e] + sigma * h[e]);
      } else if (obj == 2) {
        double acc = 0.0;
        for (int j = 0; j < p; ++j) acc += om[j] * h[(size_t)j * N + e];
        v = acc;
      } else {
        double acc = 0.0;
        for (int j = 0; j < p; ++j) {
          const double hj = h[(size_t)j * N + e], tj = t[(size_t)j * N + e];
          acc += om[j] * hj / (1.0 + tj + (sigma + tau[j]) * hj);
        }
        v = acc;
      }
      if (score_all) score_all[e] = v;
      if (!live[e]) v = -INFINITY;
    } else {
      idx[k] = LLONG_MAX;
    }
    s[k] = v;
  }
  for (int b = 0; b < B; ++b) {
    Cand mine{-INFINITY, LLONG_MAX};
#pragma unroll
    for (int k = 0; k < kTopPer; ++k)
      if (idx[k] != LLONG_MAX && better(s[k], idx[k], mine.s, mine.i)) mine = Cand{s[k], idx[k]};
    const Cand w = block_best(mine, sh);
    if (threadIdx.x == 0) blk[(size_t)blockIdx.x * B + b] = w;
#pragma unroll
    for (int k = 0; k < kTopPer; ++k)
      if (idx[k] == w.i) idx[k] = LLONG_MAX;  // taken
  }
}

// One level of the candidate merge: each CTA keeps the B best of its 512 candidates.
__global__ void __launch_bounds__(kTopBlock) topb_level_kernel(const Cand* in, int n_in, int B, Cand* out) {
  __shared__ Cand sh[33];
  double s[kTopPer];
  long long idx[kTopPer];
#pragma unroll
  for (int k = 0; k < kTopPer; ++k) {
    const long long e = (long long)blockIdx.x * kTopBlock * kTopPer + (long long)k * kTopBlock + threadIdx.x;
    if (e < n_in) {
      const Cand c = in[e];
      s[k] = c.s;
      idx[k] = c.i;
    } else {
      s[k] = -INFINITY;
      idx[k] = LLONG_MAX;
    }
  }
  for (int b = 0; b < B; ++b) {
    Cand mine{-INFINITY, LLONG_MAX};
#pragma unroll
    for (int k = 0; k < kTopPer; ++k)
      if (idx[k] != LLONG_MAX && better(s[k], idx[k], mine.s, mine.i)) mine = Cand{s[k], idx[k]};
    const Cand w = block_best(mine, sh);
    if (threadIdx.x == 0) out[(size_t)blockIdx.x * B + b] = w;
#pragma unroll
    for (int k = 0; k < kTopPer; ++k)
      if (idx[k] == w.i) idx[k] = LLONG_MAX;
  }
}

__global__ void __launch_bounds__(1024) merge_topb_kernel(const Cand* blk, int ncand, int B, int64_t* out_idx,
                                                          double* out_score) {
  __shared__ Cand sh[33];
  extern __shared__ Cand pool[];
  for (int i = threadIdx.x; i < ncand; i += blockDim.x) pool[i] = blk[i];
  __syncthreads();
  for (int b = 0; b < B; ++b) {
    Cand mine{-INFINITY, LLONG_MAX};
    for (int i = threadIdx.x; i < ncand; i += blockDim.x)
      if (pool[i].i != LLONG_MAX && better(pool[i].s, pool[i].i, mine.s, mine.i)) mine = pool[i];
    const Cand w = block_best(mine, sh);
    if (threadIdx.x == 0) {
      out_idx[b] = w.i;
      if (out_score) out_score[b] = w.s;
    }
    for (int i = threadIdx.x; i < ncand; i += blockDim.x)
      if (pool[i].i == w.i) pool[i].i = LLONG_MAX;
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------------------
// gq[c] = sum_j om_j hh[j][c] / (1 + U[j][ia[c]][c] - U[j][ib[c]][c])   (obj 0)
//       = log1p(U[0][ia[c]][c] - U[0][ib[c]][c])                          (obj 1)
__global__ void rerank_kernel(const void* U, int u_f32, int p, int nA, int ldu, const int32_t* ia,
                              const int32_t* ib, int Br, const double* hh, const double* om, int obj, double* gq,
                              int32_t* best) {
  __shared__ double sg[1024];
  for (int c = threadIdx.x; c < Br; c += blockDim.x) {
    double g;
    if (obj == 1) {
      const double bu = ldv(U, u_f32, (size_t)ia[c] * ldu + c) - ldv(U, u_f32, (size_t)ib[c] * ldu + c);
      g = log1p(bu);
    } else {
      g = 0.0;
      for (int j = 0; j < p; ++j) {
        const double bu = ldv(U, u_f32, ((size_t)j * nA + ia[c]) * ldu + c) -
                          ldv(U, u_f32, ((size_t)j * nA + ib[c]) * ldu + c);
        g += om[j] * hh[(size_t)j * Br + c] / (1.0 + bu);
      }
    }
    gq[c] = g;
    if (c < 1024) sg[c] = g;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    int bi = 0;
    double bv = sg[0];
    for (int c = 1; c < Br && c < 1024; ++c)
      if (sg[c] > bv || (isnan(sg[c]) && !isnan(bv))) {
        bv = sg[c];
        bi = c;
      }
    *best = bi;
  }
}

// ---------------------------------------------------------------------------------------
// Maintenance (polar_gpu.py:242-249).
struct MaintTmp {
  double *xi, *eta, *D, *nxi, *neta, *wX, *wY, *xiD, *etaD;
};

POLAR_HD size_t al256(size_t x) { return (x + 255) & ~size_t(255); }

static MaintTmp maint_tmp(void* base, int p, int nA, int q) {
  char* b = (char*)base;
  MaintTmp m;
  size_t o = 0;
  m.xi = (double*)(b + o); o += al256((size_t)p * q * 8);
  m.eta = (double*)(b + o); o += al256((size_t)p * q * 8);
  m.D = (double*)(b + o); o += al256((size_t)p * 8);
  m.nxi = (double*)(b + o); o += al256((size_t)p * 8);
  m.neta = (double*)(b + o); o += al256((size_t)p * 8);
  m.wX = (double*)(b + o); o += al256((size_t)p * nA * 8);
  m.wY = (double*)(b + o); o += al256((size_t)p * nA * 8);
  m.xiD = (double*)(b + o); o += al256((size_t)p * q * 8);
  m.etaD = (double*)(b + o); o += al256((size_t)p * q * 8);
  return m;
}

static size_t maint_tmp_bytes(int p, int nA, int q) {
  return al256((size_t)p * q * 8) * 4 + al256((size_t)p * 8) * 3 + al256((size_t)p * nA * 8) * 2;
}

// one CTA per pole
__global__ void maint_setup_kernel(const void* X, int ldx, const void* Y, int ldy, int f32, int p, int nA, int q,
                                   const void* U, int u_f32, int ldu, const int32_t* win, const double* G,
                                   MaintTmp m) {
  const int j = blockIdx.x;
  const int uc = win[0], a = win[1], b = win[2];
  const int64_t e = *reinterpret_cast<const int64_t*>(win + 4);
  const double* gce = G + (size_t)e * q;
  __shared__ double s1[256], s2[256];
  double n1 = 0.0, n2 = 0.0;
  for (int c = threadIdx.x; c < q; c += blockDim.x) {
    const double xi = ldv(X, f32, ((size_t)j * nA + a) * ldx + c) - ldv(X, f32, ((size_t)j * nA + b) * ldx + c);
    const double eta = gce[c] - (ldv(Y, f32, ((size_t)j * nA + a) * ldy + c) - ldv(Y, f32, ((size_t)j * nA + b) * ldy + c));
    m.xi[(size_t)j * q + c] = xi;
    m.eta[(size_t)j * q + c] = eta;
    n1 += xi * xi;
    n2 += eta * eta;
  }
  s1[threadIdx.x] = n1;
  s2[threadIdx.x] = n2;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t1 = 0.0, t2 = 0.0;
    for (int i = 0; i < (int)blockDim.x; ++i) {
      t1 += s1[i];
      t2 += s2[i];
    }
    m.nxi[j] = t1;
    m.neta[j] = t2;
    s1[0] = 1.0 + ldv(U, u_f32, ((size_t)j * nA + a) * ldu + uc) - ldv(U, u_f32, ((size_t)j * nA + b) * ldu + uc);
    m.D[j] = s1[0];
  }
  __syncthreads();
  const double D = s1[0];
  for (int c = threadIdx.x; c < q; c += blockDim.x) {
    m.xiD[(size_t)j * q + c] = m.xi[(size_t)j * q + c] / D;
    m.etaD[(size_t)j * q + c] = m.eta[(size_t)j * q + c] / D;
  }
}

// One 16-lane group per (pole, active row): w = row . dir (before the update), then
// X_row -= u xi/D, Y_row += u eta/D.  Lanes own VEC consecutive columns (vector loads).
template <typename T, int VEC>
__global__ void maint_rows_kernel(T* X, int ldx, T* Y, int ldy, int p, int nA, int q, const void* U, int u_f32,
                                  int ldu, const int32_t* win, MaintTmp m) {
  const int lanes = 16;
  const long long gidx = ((long long)blockIdx.x * blockDim.x + threadIdx.x) / lanes;
  const int lg = threadIdx.x & (lanes - 1);
  const unsigned mask = 0xffffu << (threadIdx.x & 16);
  if (gidx >= (long long)p * nA) return;
  const int j = (int)(gidx / nA), a = (int)(gidx % nA);
  const int uc = win[0];
  const double u = ldv(U, u_f32, ((size_t)j * nA + a) * ldu + uc);
  T* xr = X + ((size_t)j * nA + a) * ldx;
  T* yr = Y + ((size_t)j * nA + a) * ldy;
  const double* xi = m.xi + (size_t)j * q;
  const double* eta = m.eta + (size_t)j * q;
  const double* xiD = m.xiD + (size_t)j * q;
  const double* etaD = m.etaD + (size_t)j * q;
  double wx = 0.0, wy = 0.0;
  for (int c = lg * VEC; c < q; c += lanes * VEC) {
    T xv[VEC], yv[VEC];
    vload<T, VEC>(xv, xr + c);
    vload<T, VEC>(yv, yr + c);
#pragma unroll
    for (int v = 0; v < VEC; ++v) {
      const double x = (double)xv[v], y = (double)yv[v];
      wx = fma(x, __ldg(xi + c + v), wx);
      wy = fma(y, __ldg(eta + c + v), wy);
      xv[v] = (T)fma(-u, __ldg(xiD + c + v), x);
      yv[v] = (T)fma(u, __ldg(etaD + c + v), y);
    }
    vstore<T, VEC>(xr + c, xv);
    vstore<T, VEC>(yr + c, yv);
  }
  for (int o = 8; o > 0; o >>= 1) {
    wx += __shfl_xor_sync(mask, wx, o);
    wy += __shfl_xor_sync(mask, wy, o);
  }
  if (lg == 0) {
    m.wX[gidx] = wx;
    m.wY[gidx] = wy;
  }
}

__global__ void maint_cache_kernel(int p, int nA, int N, const void* U, int u_f32, int ldu, const int32_t* win,
                                   const int32_t* es, MaintTmp m, double* h, double* t) {
  const long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= (long long)p * N) return;
  const int j = (int)(g / N), e = (int)(g % N);
  const int uc = win[0];
  const int32_t* ea = es;
  const int32_t* eb = es + 1;
  const int a = ea[2 * e], b = eb[2 * e];
  const double cc = (ldv(U, u_f32, ((size_t)j * nA + a) * ldu + uc) - ldv(U, u_f32, ((size_t)j * nA + b) * ldu + uc)) /
                    m.D[j];
  const double dx = m.wX[(size_t)j * nA + a] - m.wX[(size_t)j * nA + b];
  const double dy = m.wY[(size_t)j * nA + a] - m.wY[(size_t)j * nA + b];
  const size_t o = (size_t)j * N + e;
  h[o] = fmax(0.0, h[o] - 2.0 * cc * dx + cc * cc * m.nxi[j]);
  t[o] = fmax(0.0, t[o] + 2.0 * cc * dy + cc * cc * m.neta[j]);
}

// Column-split form (the sketch columns spread over several ranks): this rank's share of
// the cache change, summed over the ranks before cache_apply_kernel clamps it in.
__global__ void maint_delta_kernel(int p, int nA, int N, const void* U, int u_f32, int ldu, const int32_t* win,
                                   const int32_t* es, MaintTmp m, double* dh, double* dt) {
  const long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= (long long)p * N) return;
  const int j = (int)(g / N), e = (int)(g % N);
  const int uc = win[0];
  const int a = es[2 * e], b = es[2 * e + 1];
  const double cc = (ldv(U, u_f32, ((size_t)j * nA + a) * ldu + uc) - ldv(U, u_f32, ((size_t)j * nA + b) * ldu + uc)) /
                    m.D[j];
  const double dx = m.wX[(size_t)j * nA + a] - m.wX[(size_t)j * nA + b];
  const double dy = m.wY[(size_t)j * nA + a] - m.wY[(size_t)j * nA + b];
  const size_t o = (size_t)j * N + e;
  dh[o] = cc * cc * m.nxi[j] - 2.0 * cc * dx;
  dt[o] = cc * cc * m.neta[j] + 2.0 * cc * dy;
}

__global__ void cache_apply_kernel(double* h, const double* dh, double* t, const double* dt, long long count) {
  for (long long o = (long long)blockIdx.x * blockDim.x + threadIdx.x; o < count; o += (long long)gridDim.x * blockDim.x) {
    h[o] = fmax(0.0, h[o] + dh[o]);
    t[o] = fmax(0.0, t[o] + dt[o]);
  }
}

// Winner record: win[0] = shortlist position, win[1] = aa, win[2] = bb, win[4..5] = e.
__global__ void select_kernel(const int64_t* shortl, const int32_t* best, const int32_t* es, uint8_t* live,
                              int32_t* win) {
  if (threadIdx.x != 0) return;
  const int b = best ? *best : 0;
  const int64_t e = shortl[b];
  win[0] = b;
  win[1] = es[2 * e];
  win[2] = es[2 * e + 1];
  win[3] = 0;
  *reinterpret_cast<int64_t*>(win + 4) = e;
  if (live) live[e] = 0;
}

__global__ void rank1_rows_kernel(double* F, int ldf, int q, const double* G, const int64_t* cand, const int64_t* sel) {
  const int64_t e = *sel;  // sel may point at win[4..5]
  const int64_t a = cand[2 * e], b = cand[2 * e + 1];
  for (int c = threadIdx.x; c < q; c += blockDim.x) {
    const double g = G[(size_t)e * q + c];
    F[(size_t)a * ldf + c] += g;
    F[(size_t)b * ldf + c] -= g;
  }
}

static int check_launch(const char* what) {
  count_launch();
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return set_cuda_error(what, e);
  return POLAR_OK;
}

}  // namespace polar

using namespace polar;

extern "C" int polar_fill_incidence(int n, int R, const int64_t* d_cand, const int64_t* d_sel, const int32_t* d_es,
                                    double* d_W, int ldw, int32_t* d_ia, int32_t* d_ib, polar_stream_t stream) {
  clear_error();
  if (n < 1 || R < 1 || ldw < R || !d_cand || !d_sel || !d_W) return set_error(POLAR_ERR_BAD_ARG, "bad arguments");
  if ((d_ia || d_ib) && !d_es) return set_error(POLAR_ERR_BAD_ARG, "ia/ib need es");
  cudaStream_t st = (cudaStream_t)stream;
  cudaError_t e = cudaMemsetAsync(d_W, 0, sizeof(double) * (size_t)n * ldw, st);
  if (e != cudaSuccess) return set_cuda_error("cudaMemsetAsync", e);
  fill_incidence_kernel<<<(R + 127) / 128, 128, 0, st>>>(R, d_cand, d_sel, d_es, d_W, ldw, d_ia, d_ib);
  return check_launch("fill_incidence");
}

extern "C" int polar_pair_norms(const void* d_X, int x_f32, int p, int nA, int ldx, int col0, int q,
                                const int32_t* d_ea, const int32_t* d_eb, int N, double* d_out, polar_stream_t stream) {
  clear_error();
  if (!d_X || !d_ea || !d_eb || !d_out || p < 1 || nA < 1 || q < 1 || N < 0 || col0 + q > ldx)
    return set_error(POLAR_ERR_BAD_ARG, "bad arguments");
  if (N == 0) return POLAR_OK;
  const long long threads = (long long)p * N * 16;
  const int blocks = (int)((threads + 255) / 256);
  cudaStream_t st = (cudaStream_t)stream;
  if (x_f32)
    pair_norms_kernel<float><<<blocks, 256, 0, st>>>((const float*)d_X, p, nA, ldx, col0, q, d_ea, d_eb, N, d_out);
  else
    pair_norms_kernel<double><<<blocks, 256, 0, st>>>((const double*)d_X, p, nA, ldx, col0, q, d_ea, d_eb, N, d_out);
  return check_launch("pair_norms");
}

extern "C" size_t polar_topb_tmp_bytes(int N, int B) {
  const long long per = (long long)kTopBlock * kTopPer;
  const long long nb = (N + per - 1) / per;
  return 2 * (size_t)(nb > 0 ? nb : 1) * (B > 0 ? B : 1) * sizeof(Cand) + 256;
}

extern "C" int polar_score_topb(const double* d_h, const double* d_t, const double* d_tau, const double* d_om,
                                double sigma, int p, int N, const uint8_t* d_live, int obj, int B, int64_t* d_out_idx,
                                double* d_out_score, double* d_score_all, void* d_tmp, polar_stream_t stream) {
  clear_error();
  if (!d_h || !d_t || !d_tau || !d_om || !d_live || !d_out_idx || !d_tmp || p < 1 || N < 1)
    return set_error(POLAR_ERR_BAD_ARG, "bad arguments");
  if (B < 1 || B > kMaxB || B > N) return set_error(POLAR_ERR_BAD_ARG, "B out of range");
  if (obj < 0 || obj > 2) return set_error(POLAR_ERR_BAD_ARG, "obj must be 0, 1 or 2");
  const long long per = (long long)kTopBlock * kTopPer;
  const int nb = (int)((N + per - 1) / per);
  cudaStream_t st = (cudaStream_t)stream;
  score_block_topb_kernel<<<nb, kTopBlock, 0, st>>>(d_h, d_t, d_tau, d_om, sigma, p, N, d_live, obj, B, d_score_all,
                                                    (Cand*)d_tmp);
  int rc = check_launch("score_block_topb");
  if (rc) return rc;
  // merge levels until one CTA can take the rest
  const long long per_lvl = (long long)kTopBlock * kTopPer;
  Cand* a = (Cand*)d_tmp;
  Cand* b2 = a + (size_t)nb * B;
  long long ncand = (long long)nb * B;
  while (ncand > 4096) {
    const int nb2 = (int)((ncand + per_lvl - 1) / per_lvl);
    topb_level_kernel<<<nb2, kTopBlock, 0, st>>>(a, (int)ncand, B, b2);
    rc = check_launch("topb_level");
    if (rc) return rc;
    Cand* t = a;
    a = b2;
    b2 = t;
    ncand = (long long)nb2 * B;
  }
  const size_t smem = (size_t)ncand * sizeof(Cand);
  if (smem > 48 * 1024)
    cudaFuncSetAttribute(merge_topb_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  merge_topb_kernel<<<1, 1024, smem, st>>>(a, (int)ncand, B, d_out_idx, d_out_score);
  return check_launch("merge_topb");
}

extern "C" int polar_rerank(const void* d_U, int u_f32, int p, int nA, int ldu, const int32_t* d_ia,
                            const int32_t* d_ib, int Br, const double* d_hh, const double* d_om, int obj, double* d_gq,
                            int32_t* d_best, polar_stream_t stream) {
  clear_error();
  if (!d_U || !d_ia || !d_ib || !d_gq || !d_best || Br < 1 || Br > 1024 || ldu < Br || p < 1)
    return set_error(POLAR_ERR_BAD_ARG, "bad arguments");
  if (obj == 0 && (!d_hh || !d_om)) return set_error(POLAR_ERR_BAD_ARG, "frac re-rank needs hh and om");
  rerank_kernel<<<1, 256, 0, (cudaStream_t)stream>>>(d_U, u_f32, p, nA, ldu, d_ia, d_ib, Br, d_hh, d_om, obj, d_gq,
                                                     d_best);
  return check_launch("rerank");
}

extern "C" size_t polar_maintain_tmp_bytes(int p, int nA, int q) { return maint_tmp_bytes(p, nA, q); }

extern "C" int polar_select(const int64_t* d_short, const int32_t* d_best, const int32_t* d_es, uint8_t* d_live,
                            int32_t* d_win, polar_stream_t stream) {
  clear_error();
  if (!d_short || !d_es || !d_win) return set_error(POLAR_ERR_BAD_ARG, "bad arguments");
  select_kernel<<<1, 32, 0, (cudaStream_t)stream>>>(d_short, d_best, d_es, d_live, d_win);
  return check_launch("select");
}

// Both maintenance forms: delta == false updates h, t in place; delta == true writes this
// rank's cache change to h, t (as dh, dt).
static int maintain(void* d_X, int ldx, void* d_Y, int ldy, int xy_f32, int p, int nA, int q, const void* d_U,
                    int u_f32, int ldu, const int32_t* d_win, const double* d_G, const int32_t* d_es, int N,
                    double* d_h, double* d_t, void* d_tmp, polar_stream_t stream, bool delta) {
  clear_error();
  if (!d_X || !d_Y || !d_U || !d_win || !d_G || !d_es || !d_h || !d_t || !d_tmp || p < 1 || nA < 1 || q < 1 ||
      ldx < q || ldy < q)
    return set_error(POLAR_ERR_BAD_ARG, "bad arguments");
  cudaStream_t st = (cudaStream_t)stream;
  MaintTmp m = maint_tmp(d_tmp, p, nA, q);
  maint_setup_kernel<<<p, 128, 0, st>>>(d_X, ldx, d_Y, ldy, xy_f32, p, nA, q, d_U, u_f32, ldu, d_win, d_G, m);
  int rc = check_launch("maint_setup");
  if (rc) return rc;
  const long long thr = (long long)p * nA * 16;
  const int blocks = (int)((thr + 255) / 256);
  const uintptr_t al = (uintptr_t)d_X | (uintptr_t)d_Y;
  if (xy_f32) {
    if (q % 4 == 0 && ldx % 4 == 0 && ldy % 4 == 0 && al % 16 == 0)
      maint_rows_kernel<float, 4><<<blocks, 256, 0, st>>>((float*)d_X, ldx, (float*)d_Y, ldy, p, nA, q, d_U, u_f32,
                                                          ldu, d_win, m);
    else
      maint_rows_kernel<float, 1><<<blocks, 256, 0, st>>>((float*)d_X, ldx, (float*)d_Y, ldy, p, nA, q, d_U, u_f32,
                                                          ldu, d_win, m);
  } else {
    if (q % 2 == 0 && ldx % 2 == 0 && ldy % 2 == 0 && al % 16 == 0)
      maint_rows_kernel<double, 2><<<blocks, 256, 0, st>>>((double*)d_X, ldx, (double*)d_Y, ldy, p, nA, q, d_U,
                                                           u_f32, ldu, d_win, m);
    else
      maint_rows_kernel<double, 1><<<blocks, 256, 0, st>>>((double*)d_X, ldx, (double*)d_Y, ldy, p, nA, q, d_U,
                                                           u_f32, ldu, d_win, m);
  }
  rc = check_launch("maint_rows");
  if (rc) return rc;
  if (N > 0) {
    const long long t2 = (long long)p * N;
    if (delta)
      maint_delta_kernel<<<(int)((t2 + 255) / 256), 256, 0, st>>>(p, nA, N, d_U, u_f32, ldu, d_win, d_es, m, d_h, d_t);
    else
      maint_cache_kernel<<<(int)((t2 + 255) / 256), 256, 0, st>>>(p, nA, N, d_U, u_f32, ldu, d_win, d_es, m, d_h, d_t);
    rc = check_launch(delta ? "maint_delta" : "maint_cache");
  }
  return rc;
}

extern "C" int polar_maintain(void* d_X, int ldx, void* d_Y, int ldy, int xy_f32, int p, int nA, int q, const void* d_U,
                              int u_f32, int ldu, const int32_t* d_win, const double* d_G, const int32_t* d_es, int N,
                              double* d_h, double* d_t, void* d_tmp, polar_stream_t stream) {
  return maintain(d_X, ldx, d_Y, ldy, xy_f32, p, nA, q, d_U, u_f32, ldu, d_win, d_G, d_es, N, d_h, d_t, d_tmp, stream,
                  false);
}

extern "C" int polar_maintain_split(void* d_X, int ldx, void* d_Y, int ldy, int xy_f32, int p, int nA, int q,
                                    const void* d_U, int u_f32, int ldu, const int32_t* d_win, const double* d_G,
                                    const int32_t* d_es, int N, double* d_dh, double* d_dt, void* d_tmp,
                                    polar_stream_t stream) {
  return maintain(d_X, ldx, d_Y, ldy, xy_f32, p, nA, q, d_U, u_f32, ldu, d_win, d_G, d_es, N, d_dh, d_dt, d_tmp,
                  stream, true);
}

extern "C" int polar_cache_apply(double* d_h, const double* d_dh, double* d_t, const double* d_dt, int64_t count,
                                 polar_stream_t stream) {
  clear_error();
  if (!d_h || !d_dh || !d_t || !d_dt || count < 0) return set_error(POLAR_ERR_BAD_ARG, "bad arguments");
  if (count == 0) return POLAR_OK;
  const long long blocks = (count + 255) / 256;
  cache_apply_kernel<<<(int)(blocks < 148 * 16 ? blocks : 148 * 16), 256, 0, (cudaStream_t)stream>>>(d_h, d_dh, d_t,
                                                                                                     d_dt, count);
  return check_launch("cache_apply");
}

extern "C" int polar_rank1_rows(double* d_F, int ldf, int q, const double* d_G, const int64_t* d_cand,
                                const int64_t* d_sel, polar_stream_t stream) {
  clear_error();
  if (!d_F || !d_G || !d_cand || !d_sel || q < 1 || ldf < q) return set_error(POLAR_ERR_BAD_ARG, "bad arguments");
  rank1_rows_kernel<<<1, 128, 0, (cudaStream_t)stream>>>(d_F, ldf, q, d_G, d_cand, d_sel);
  return check_launch("rank1_rows");
}
