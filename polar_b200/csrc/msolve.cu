// Persistent multi-shift CG for POLAR (sm_100a).
//
// Replaces realworld/polar_gpu.py:88-133 (msolve).  One cooperative launch runs every
// iteration of the seed CG for all R columns, the zeta recurrences of all p poles and the
// three-scalar norm tracker, with bounded grid barriers between the phases:
//
//   P1  v = (M + tau_0 I) d  (CSR SpMM, heavy rows split)  + per-CTA partials of d.v
//   R1  last CTA: a = rr / d.v
//   P2  r <- r - a v ; partials of r.r ; r on the active rows -> history slot
//   R2  last CTA: beta, zeta recurrences, tracker, freezing, convergence; the
//       per-pole step coefficients (a_j, zeta_j, beta_j) of this iteration -> table
//   P3  d <- r + beta d
//   P4  every M iterations (and at exit): the deferred shifted update.  For each
//       active row / column / pole, M steps of  X += a_j P ; P = zeta_j r + beta_j P
//       are applied from the history in registers: X and P cross HBM once per M
//       iterations instead of once per iteration.  The arithmetic per element is the
//       same sequence of operations as the per-iteration update.
//
// Poles whose iterates are frozen for a whole block of M steps are skipped.
#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "common.cuh"
#include "graph_ops.cuh"
#include "host_util.h"
#include "solver_core.cuh"
#include "msolve_mk.h"
#include "batch_split.h"

namespace polar {

// ---------------------------------------------------------------------------------------
// The whole solve for one problem on `vnb` co-resident CTAs; this CTA is number `vb` of
// them.  The CTAs of a problem synchronise only among themselves (barrier words in the
// problem's own control block).
template <typename T, int VEC, bool WEIGHTED, int E>
POLAR_D void msolve_run(const SolvePrm<T>& P, const int vb, const int vnb) {
  __shared__ double red[kWarps * kMaxLd];
  __shared__ double s_col[2][kMaxLd];

  GridSync gs;
  gs.count = reinterpret_cast<unsigned*>(P.ctl + 4);
  gs.gen = reinterpret_cast<unsigned*>(P.ctl + 5);
  gs.err = P.ctl + 1;
  gs.where = P.ctl + 2;
  gs.timeout_ns = P.timeout_ns;
  gs.nblk = (unsigned)vnb;

  const int ld = P.ld, p = P.p, n = P.n, nA = P.nA;
  const RowGroup rg = make_row_group<VEC>(ld);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int gpw = 32 / rg.G;
  const long long tid = (long long)vb * blockDim.x + threadIdx.x;
  const long long nth = (long long)vnb * blockDim.x;
  const long long nvec = (long long)n * rg.G;  // VEC-vectors in an n x ld block
  double* my_part = P.part + (size_t)vb * ld;

  // ---- P0: r = d = W, partial r.r ----
  {
    double acc[VEC];
#pragma unroll
    for (int v = 0; v < VEC; ++v) acc[v] = 0.0;
    for (long long e = tid; e < nvec; e += nth) {
      const long long i = e / rg.G;
      double wd[VEC];
#pragma unroll
      for (int v = 0; v < VEC; ++v) {
        const int c = rg.col + v;
        wd[v] = (c < P.R) ? __ldg(P.W + (size_t)i * P.ldw + c) : 0.0;
        acc[v] += wd[v] * wd[v];
      }
      vstore<double, VEC>(P.r + (size_t)i * ld + rg.col, wd);
      store_dir<T, VEC>(P, wd, (size_t)i * ld + rg.col);
    }
    reduce_cols_to_part<VEC>(acc, rg.G, ld, red, my_part);
  }
  {
    unsigned g0;
    if (grid_arrive(gs, g0)) {
      reduce_partials(P.part, vnb, ld, red, s_col[0]);
      int anyv = 0;
      for (int c = threadIdx.x; c < ld; c += blockDim.x) {
        const double rr = s_col[0][c];
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
        const int c = it % ld;
        const double rr = s_col[0][c];
        P.z[it] = 1.0;
        P.zp[it] = 1.0;
        P.live[it] = rr > 0.0 ? 1 : 0;
        P.hs[it] = 0.0;
        P.ip[it] = 0.0;
        P.pn[it] = rr;
        P.pflag[it] = 0;
      }
      anyv = __syncthreads_or(anyv);
      if (threadIdx.x == 0) {
        P.ctl[3] = anyv;
        P.stats[0] = 0;
        P.stats[1] = 0;
      }
      if (!grid_release(gs, g0)) return;
    } else if (!grid_wait(gs, g0, 1)) {
      return;
    }
  }

  const double shift0 = __ldg(P.tau);
  const int lgG = __ffs(rg.G) - 1;
  int pending = 0;
  bool first = true;
  bool flush_pending = false;
  long long it = 0;
  bool capped = false;
  bool more = ld_volatile_i32(P.ctl + 3) != 0 && P.maxit > 0;
  if (ld_volatile_i32(P.ctl + 3) != 0 && P.maxit <= 0) capped = true;
  const bool timer = vb == 0 && threadIdx.x == 0;
  uint64_t tmark = timer ? globaltimer_ns() : 0;
  auto lap = [&](int slot) {
    if (timer) {
      const uint64_t t = globaltimer_ns();
      P.stats[2 + slot] += (long long)(t - tmark);
      tmark = t;
    }
  };
  lap(5);  // init (P0 + R0)
  while (more) {
    // ---- P4 (deferred shifted update of the previous M iterations) ----
    if (flush_pending) {
      shifted_update<T, E>(P, pending, first, false, tid, nth);
      first = false;
      pending = 0;
      flush_pending = false;
      if (vb == 0 && threadIdx.x == 0) P.stats[1] += 1;
    }
    lap(0);
    // ---- P1 ----
    spmm_phase<T, VEC, WEIGHTED, true>(P.g, ld, shift0, P.d, P.v, ld, P.chunk_part, P.hcount, red, P.act, vb,
                                       vnb);
    reduce_red_to_part(red, ld, my_part);
    // ---- R1 ----
    {
      unsigned g1;
      if (grid_arrive(gs, g1)) {
        reduce_partials(P.part, vnb, ld, red, s_col[0]);
        for (int c = threadIdx.x; c < ld; c += blockDim.x) {
          const int a_on = P.act[c];
          const double dv = s_col[0][c];
          const double a = a_on ? P.rr[c] / dv : 0.0;
          if (a_on && !isfinite(a)) atomicCAS(P.ctl + 1, 0, (int)POLAR_ERR_NONFINITE);
          P.ag[c] = a;
        }
        if (!grid_release(gs, g1)) return;
      } else if (!grid_wait(gs, g1, 2)) {
        return;
      }
    }
    lap(1);
    // ---- P2 ----
    {
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
        T* hslot = P.hist + (size_t)pending * nA * ld;
        constexpr int U = 2;
        for (long long e0 = tid; e0 < nvec; e0 += U * nth) {
          double rv[U][VEC];
          T vv[U][VEC];
          long long ii[U];
#pragma unroll
          for (int u = 0; u < U; ++u) {
            const long long e = e0 + u * nth;
            ii[u] = e < nvec ? (e >> lgG) : -1;
            if (ii[u] >= 0) {
              vload<double, VEC>(rv[u], P.r + (size_t)ii[u] * ld + rg.col);
              vload<T, VEC>(vv[u], P.v + (size_t)ii[u] * ld + rg.col);
            }
          }
#pragma unroll
          for (int u = 0; u < U; ++u) {
            if (ii[u] < 0) continue;
            T rt[VEC];
#pragma unroll
            for (int v = 0; v < VEC; ++v) {
              if (on[v]) rv[u][v] = rv[u][v] - a_c[v] * (double)vv[u][v];
              racc[v] += rv[u][v] * rv[u][v];
              rt[v] = (T)rv[u][v];
            }
            vstore<double, VEC>(P.r + (size_t)ii[u] * ld + rg.col, rv[u]);
            const int ai = __ldg(P.active_pos + ii[u]);
            if (ai >= 0) vstore<T, VEC>(hslot + (size_t)ai * ld + rg.col, rt);
          }
        }
      }
      reduce_cols_to_part<VEC>(racc, rg.G, ld, red, my_part);
    }
    // ---- R2: column scalars (serial, last CTA) ----
    {
      unsigned g2;
      if (grid_arrive(gs, g2)) {
        double* s_rrn = s_col[0];
        reduce_partials(P.part, vnb, ld, red, s_rrn);
        int anyv2 = 0;
        for (int c = threadIdx.x; c < ld; c += blockDim.x) {
          const int a_on = P.act[c];
          const double rrn = s_rrn[c];
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
            anyv2 |= done ? 0 : 1;
            if (c < P.R) P.iters_out[c] += 1;
          }
        }
        anyv2 = __syncthreads_or(anyv2);
        if (threadIdx.x == 0) {
          P.ctl[3] = anyv2;
          P.stats[0] = it + 1;
        }
        if (!grid_release(gs, g2)) return;
      } else if (!grid_wait(gs, g2, 3)) {
        return;
      }
    }
    lap(2);
    const int any_after = ld_volatile_i32(P.ctl + 3);
    more = any_after && it + 1 < P.maxit;
    capped = any_after && !more;
    // ---- pole recurrences (distributed: each thread owns fixed (pole, column) items) ----
    for (long long q = tid; q < (long long)p * ld; q += nth) {
      const int j = (int)(q / ld), c = (int)(q % ld);
      const bool m = P.live[q] && P.upd[c];
      const size_t ci = ((size_t)pending * p + j) * ld + c;
      int pf = pending == 0 ? 0 : P.pflag[q];
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
      } else {
        P.ca[ci] = T(0);
        P.cz[ci] = T(0);
        P.cb[ci] = T(1);
      }
      P.pflag[q] = pf;
    }
    // ---- P3 ----
    if (more) {
      double be_c[VEC];
      bool on[VEC], any_on = false;
#pragma unroll
      for (int v = 0; v < VEC; ++v) {
        be_c[v] = P.beg[rg.col + v];
        on[v] = P.upd[rg.col + v] != 0;
        any_on |= on[v];
      }
      if (any_on) {
        constexpr int U = 2;
        for (long long e0 = tid; e0 < nvec; e0 += U * nth) {
          double rv[U][VEC], dv[U][VEC];
          long long ii[U];
#pragma unroll
          for (int u = 0; u < U; ++u) {
            const long long e = e0 + u * nth;
            ii[u] = e < nvec ? (e >> lgG) : -1;
            if (ii[u] >= 0) {
              vload<double, VEC>(rv[u], P.r + (size_t)ii[u] * ld + rg.col);
              load_dir<T, VEC>(P, dv[u], (size_t)ii[u] * ld + rg.col);
            }
          }
#pragma unroll
          for (int u = 0; u < U; ++u) {
            if (ii[u] < 0) continue;
#pragma unroll
            for (int v = 0; v < VEC; ++v)
              if (on[v]) dv[u][v] = rv[u][v] + be_c[v] * dv[u][v];
            store_dir<T, VEC>(P, dv[u], (size_t)ii[u] * ld + rg.col);
          }
        }
      }
    }
    ++pending;
    ++it;
    flush_pending = pending == kHist;
    if (!grid_sync(gs, 4)) return;
    lap(3);
  }
  // ---- final pass: remaining steps, X -> output ----
  shifted_update<T, E>(P, pending, first, true, tid, nth);
  lap(4);
  if (vb == 0) {
    if (P.track && P.h_out)
      for (int q = threadIdx.x; q < p * ld; q += blockDim.x) {
        const int j = q / ld, c = q % ld;
        if (c < P.R) P.h_out[(size_t)j * P.R + c] = P.hs[q];
      }
    if (threadIdx.x == 0) {
      P.stats[1] += 1;
      P.ctl[0] = capped ? (int)POLAR_ERR_ITER_CAP : 0;
    }
  }
}

template <typename T, int VEC, bool WEIGHTED, int E>
__global__ void __launch_bounds__(kBlock, 1) msolve_kernel(const __grid_constant__ SolvePrm<T> P) {
  msolve_run<T, VEC, WEIGHTED, E>(P, (int)blockIdx.x, (int)gridDim.x);
}

// Many independent solves in one cooperative launch.  Problem b owns CTAs
// [cta_off[b], cta_off[b+1]); its parameter block lives in its own workspace and is staged
// in shared memory.  Problems never wait on one another: each share of CTAs runs its own
// solve to convergence and leaves.
constexpr int kMaxBatch = 64;
struct BatchPrm {
  int nprob;
  int cta_off[kMaxBatch + 1];
  const void* prm[kMaxBatch];
};

template <typename T, int VEC, bool WEIGHTED, int E>
__global__ void __launch_bounds__(kBlock, 1) msolve_batch_kernel(const __grid_constant__ BatchPrm B) {
  __shared__ __align__(16) int s_prm[(sizeof(SolvePrm<T>) + 3) / 4];
  int b = 0;
  while (b + 1 < B.nprob && (int)blockIdx.x >= B.cta_off[b + 1]) ++b;
  const int* src = reinterpret_cast<const int*>(B.prm[b]);
  for (int i = threadIdx.x; i < (int)(sizeof(SolvePrm<T>) / 4); i += blockDim.x) s_prm[i] = src[i];
  __syncthreads();
  const SolvePrm<T>& P = *reinterpret_cast<const SolvePrm<T>*>(s_prm);
  msolve_run<T, VEC, WEIGHTED, E>(P, (int)blockIdx.x - B.cta_off[b], B.cta_off[b + 1] - B.cta_off[b]);
}

// ---------------------------------------------------------------------------------------
struct SolveLayout {
  size_t off[48];
  size_t total;
  int ld, vec;
};

static int choose_vec(int precision, int ld) {
  if (precision == POLAR_MIXED) return ld >= 4 ? 4 : ld;
  return ld >= 2 ? 2 : 1;
}

static int choose_ld(int precision, int R) {
  int ld = next_pow2(R < 1 ? 1 : R);
  const int vec = choose_vec(precision, ld);
  if (ld < vec) ld = vec;
  return ld;
}

static int max_ld(int precision) { return precision == POLAR_MIXED ? 128 : 64; }

static size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

static int max_grid_for(int precision, int vec, bool weighted);

static void solve_layout(const polar_graph* g, int precision, int R, int p, int nA, int grid, SolveLayout* L) {
  const int ld = choose_ld(precision, R);
  const size_t ts = precision == POLAR_MIXED ? 4 : 8;
  const size_t n = g->n;
  size_t o = 0;
  int k = 0;
  auto add = [&](size_t bytes) {
    L->off[k++] = o;
    o += align256(bytes);
  };
  add(n * ld * 8);                                 // 0 r (FP64 in every precision)
  add(n * ld * ts);                                // 1 d
  add(n * ld * ts);                                // 2 v
  add((size_t)kHist * nA * ld * ts);               // 3 hist
  add((size_t)p * nA * ld * ts);                   // 4 P
  add((size_t)p * nA * ld * ts);                   // 5 X
  add((size_t)(g->nchunks > 0 ? g->nchunks : 1) * ld * 8);   // 6 chunk partials (FP64 sums)
  add((size_t)(g->nheavy > 0 ? g->nheavy : 1) * 4 * (ld > 16 ? ld / 16 : 1));  // 7 heavy counters per panel
  add((size_t)grid * ld * 8);                      // 8 CTA partials
  for (int i = 0; i < 6; ++i) add((size_t)ld * 8);  // 9..14 rr stop ap bp a be
  add((size_t)ld * 4);                             // 15 act
  add((size_t)ld * 4);                             // 16 upd
  for (int i = 0; i < 5; ++i) add((size_t)p * ld * 8);  // 17..21 z zp h ip pn
  add((size_t)p * ld * 4);                         // 22 live
  add((size_t)p * ld * 4);                         // 23 pflag
  for (int i = 0; i < 3; ++i) add((size_t)kHist * p * ld * ts);  // 24..26 coef planes
  add(64);                                         // 27 ctl
  add(64);                                         // 28 stats
  add((size_t)ld * 8);                             // 29 chi
  add(4096);                                       // 30 device copy of the parameter block
  add((size_t)p * ld * kNC * 8);                   // 31 composed deferred-update coefficients
  add((size_t)kMaxHeavyCtas * ld * 8);             // 32 heavy-row d.v partials
  add(precision == POLAR_MIXED ? n * ld * 4 : 0);  // 33 direction remainder (mixed precision)
  L->total = o;
  L->ld = ld;
  L->vec = choose_vec(precision, ld);
}

template <typename T, int VEC, bool WEIGHTED, int E>
static int launch_solve(const SolvePrm<T>& prm, int grid, cudaStream_t st) {
  void* args[] = {(void*)&prm};
  cudaError_t e = cudaLaunchCooperativeKernel((const void*)msolve_kernel<T, VEC, WEIGHTED, E>, dim3(grid),
                                              dim3(kBlock), args, 0, st);
  count_launch();
  if (e != cudaSuccess) return set_cuda_error("cudaLaunchCooperativeKernel(msolve)", e);
  return POLAR_OK;
}

template <typename T, int VEC, bool WEIGHTED, int E>
static int occupancy_of() {
  int nb = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, msolve_kernel<T, VEC, WEIGHTED, E>, kBlock, 0);
  return nb;
}

static int max_grid_for(int precision, int vec, bool weighted) {
  int dev = 0, sms = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  int nb = 0;
  if (precision == POLAR_MIXED) {
    if (vec == 4) nb = weighted ? occupancy_of<float, 4, true, POLAR_E32>() : occupancy_of<float, 4, false, POLAR_E32>();
    else if (vec == 2) nb = weighted ? occupancy_of<float, 2, true, POLAR_E32>() : occupancy_of<float, 2, false, POLAR_E32>();
    else nb = weighted ? occupancy_of<float, 1, true, POLAR_E32>() : occupancy_of<float, 1, false, POLAR_E32>();
  } else {
    if (vec == 2) nb = weighted ? occupancy_of<double, 2, true, POLAR_E64>() : occupancy_of<double, 2, false, POLAR_E64>();
    else nb = weighted ? occupancy_of<double, 1, true, POLAR_E64>() : occupancy_of<double, 1, false, POLAR_E64>();
  }
  if (nb < 1) nb = 1;
  return nb * sms;
}

static uint64_t g_timeout_ns = 4000000000ull;  // 4 s per barrier wait
static int g_solver_mode = 0;                      // 0: kernel-per-phase graph, 1: persistent

template <typename T, int VEC, bool W, int E>
static int mk_grid_for() { return mk_grid_max<T, VEC, W, E>(); }

static int grid_for_mode(int precision, int vec, bool weighted) {
  if (g_solver_mode == 1) return max_grid_for(precision, vec, weighted);
  if (precision == POLAR_MIXED) {
    if (vec == 4) return weighted ? mk_grid_for<float, 4, true, POLAR_E32>() : mk_grid_for<float, 4, false, POLAR_E32>();
    if (vec == 2) return weighted ? mk_grid_for<float, 2, true, POLAR_E32>() : mk_grid_for<float, 2, false, POLAR_E32>();
    return weighted ? mk_grid_for<float, 1, true, POLAR_E32>() : mk_grid_for<float, 1, false, POLAR_E32>();
  }
  if (vec == 2) return weighted ? mk_grid_for<double, 2, true, POLAR_E64>() : mk_grid_for<double, 2, false, POLAR_E64>();
  return weighted ? mk_grid_for<double, 1, true, POLAR_E64>() : mk_grid_for<double, 1, false, POLAR_E64>();
}

}  // namespace polar

using namespace polar;

extern "C" void polar_set_barrier_timeout_ns(uint64_t ns) { g_timeout_ns = ns ? ns : 1; }

// Residual storage of the mixed-precision kernel-per-phase driver: 64 (FP64) or 32.
static int g_mixed_residual_bits = 64;

extern "C" int polar_set_mixed_residual(int bits) {
  clear_error();
  if (bits != 32 && bits != 64) return set_error(POLAR_ERR_BAD_ARG, "residual bits must be 32 or 64");
  g_mixed_residual_bits = bits;
  return POLAR_OK;
}

// L2 policy of the kernel-per-phase driver (SolvePrm::l2_mode / hot_rows).  Default mode 2
// (hot 32 MB evict_last, other gathers and streams evict_first): 5-7 % faster SpMM launches
// on the 4M-vertex graph at R = 16 and 128 in both precisions than no hints, and 1.5 %
// faster at R = 16 than a 64 MB hot prefix.
static int g_l2_mode = 2;
static size_t g_l2_hot_bytes = size_t(32) << 20;

namespace polar {
int l2_mode_setting() { return g_l2_mode; }
size_t l2_hot_bytes_setting() { return g_l2_hot_bytes; }
}  // namespace polar

extern "C" int polar_set_l2_policy(int mode, size_t hot_bytes) {
  clear_error();
  if (mode < 0 || mode > 2) return set_error(POLAR_ERR_BAD_ARG, "l2 mode must be 0, 1 or 2");
  g_l2_mode = mode;
  g_l2_hot_bytes = hot_bytes;
  return POLAR_OK;
}

namespace polar {
int mk_spmm_lanes(int precision, int ld);
int mk_sell_rows(int precision, int ld);
}

extern "C" int polar_sell_rows(int precision, int R) {
  if (g_solver_mode != 0) return 0;
  return mk_sell_rows(precision, choose_ld(precision, R < 1 ? 1 : R));
}

extern "C" int polar_heavy_threshold(int precision, int R) {
  const int ld = choose_ld(precision, R < 1 ? 1 : R);
  const int G = g_solver_mode == 0 ? mk_spmm_lanes(precision, ld) : ld / choose_vec(precision, ld);
  return 8 * G > 16 ? 8 * G : 16;
}

extern "C" int polar_set_solver_mode(int mode) {
  if (mode != 0 && mode != 1) return POLAR_ERR_BAD_ARG;
  g_solver_mode = mode;
  return POLAR_OK;
}

extern "C" size_t polar_msolve_workspace_bytes(const polar_graph* g, int precision, int R, int p, int nA) {
  if (!g || R < 1 || p < 1 || nA < 0) return 0;
  const int ld = choose_ld(precision, R);
  SolveLayout L;
  solve_layout(g, precision, R, p, nA, grid_for_mode(precision, choose_vec(precision, ld), g->d_wts != nullptr), &L);
  return L.total;
}

// Parameter block of one solve: arguments as polar_msolve takes them, workspace regions
// from the layout.  `composed`: deferred updates from composed coefficients (the
// kernel-per-phase driver); the persistent kernels apply the per-step coefficients.
template <typename TT>
static void fill_prm(SolvePrm<TT>& prm, const polar_graph* g, int R, int ld, int p, int nA, double tol,
                     int64_t maxit, int track, const double* d_W, int ldw, const double* d_tau,
                     const int32_t* d_active, const int32_t* d_active_pos, void* d_X_out, int x_f32, int ldx,
                     double* d_h_out, int64_t* d_iters_out, char* ws, const SolveLayout& L, bool composed) {
  prm.g = *g;
  prm.n = g->n;
  prm.R = R;
  prm.ld = ld;
  prm.p = p;
  prm.nA = nA;
  prm.tol = tol;
  prm.maxit = maxit;
  prm.track = track;
  prm.W = d_W;
  prm.ldw = ldw;
  prm.tau = d_tau;
  prm.active = d_active;
  prm.active_pos = d_active_pos;
  prm.Xout = d_X_out;
  prm.x_f32 = x_f32;
  prm.ldx = ldx;
  prm.h_out = d_h_out;
  prm.iters_out = (long long*)d_iters_out;
  prm.r = (double*)(ws + L.off[0]);
  // the FP32 residual (when chosen) takes the first half of the FP64 residual's region
  prm.r32 = (composed && sizeof(TT) == 4 && g_mixed_residual_bits == 32) ? (float*)(ws + L.off[0]) : nullptr;
  prm.d = (TT*)(ws + L.off[1]);
  prm.v = (TT*)(ws + L.off[2]);
  prm.hist = (TT*)(ws + L.off[3]);
  prm.Pb = (TT*)(ws + L.off[4]);
  prm.Xb = (TT*)(ws + L.off[5]);
  prm.chunk_part = (TT*)(ws + L.off[6]);
  prm.hcount = (int*)(ws + L.off[7]);
  prm.part = (double*)(ws + L.off[8]);
  prm.rr = (double*)(ws + L.off[9]);
  prm.stop = (double*)(ws + L.off[10]);
  prm.ap = (double*)(ws + L.off[11]);
  prm.bp = (double*)(ws + L.off[12]);
  prm.ag = (double*)(ws + L.off[13]);
  prm.beg = (double*)(ws + L.off[14]);
  prm.act = (int*)(ws + L.off[15]);
  prm.upd = (int*)(ws + L.off[16]);
  prm.z = (double*)(ws + L.off[17]);
  prm.zp = (double*)(ws + L.off[18]);
  prm.hs = (double*)(ws + L.off[19]);
  prm.ip = (double*)(ws + L.off[20]);
  prm.pn = (double*)(ws + L.off[21]);
  prm.live = (int*)(ws + L.off[22]);
  prm.pflag = (int*)(ws + L.off[23]);
  prm.ca = (TT*)(ws + L.off[24]);
  prm.cz = (TT*)(ws + L.off[25]);
  prm.cb = (TT*)(ws + L.off[26]);
  prm.ctl = (int*)(ws + L.off[27]);
  prm.stats = (long long*)(ws + L.off[28]);
  prm.chig = (double*)(ws + L.off[29]);
  prm.cmp = composed ? (double*)(ws + L.off[31]) : nullptr;
  prm.part_h = (double*)(ws + L.off[32]);
  prm.dlo = sizeof(TT) == 4 ? (float*)(ws + L.off[33]) : nullptr;
  prm.nbh = 0;
  prm.timeout_ns = g_timeout_ns;
  // the hint path lives in the kernel-per-phase kernels only
  prm.l2_mode = composed ? g_l2_mode : 0;
  const long long hot = (long long)(g_l2_hot_bytes / ((size_t)ld * sizeof(TT)));
  prm.hot_rows = (int)(hot < g->n ? hot : g->n);
}

extern "C" int polar_msolve(const polar_graph* g, int precision, const double* d_W, int ldw, int R,
                            const double* d_tau, int p, const int32_t* d_active, const int32_t* d_active_pos,
                            int nA, double tol, int64_t maxit, int track, void* d_X_out, int x_f32, int ldx,
                            double* d_h_out, int64_t* d_iters_out, void* d_workspace, size_t workspace_bytes,
                            polar_stream_t stream) {
  clear_error();
  if (!g || !d_W || !d_tau || !d_X_out || !d_iters_out || !d_workspace) return set_error(POLAR_ERR_BAD_ARG, "null pointer");
  if (precision != POLAR_FP64 && precision != POLAR_MIXED) return set_error(POLAR_ERR_BAD_ARG, "precision");
  if (R < 1 || R > max_ld(precision)) return set_error(POLAR_ERR_BAD_ARG, "R out of range for this precision");
  if (p < 1 || nA < 1 || ldw < R || ldx < R || g->n < 1) return set_error(POLAR_ERR_BAD_ARG, "bad sizes");
  if (track && !d_h_out) return set_error(POLAR_ERR_BAD_ARG, "track needs h_out");
  if ((g->d_wts == nullptr) != (g->d_diag == nullptr)) return set_error(POLAR_ERR_BAD_ARG, "weights and diag go together");
  const int ld = choose_ld(precision, R);
  const int vec = choose_vec(precision, ld);
  const bool weighted = g->d_wts != nullptr;
  const int grid = grid_for_mode(precision, vec, weighted);
  SolveLayout L;
  solve_layout(g, precision, R, p, nA, grid, &L);
  if (workspace_bytes < L.total) return set_error(POLAR_ERR_WORKSPACE, "workspace too small");
  cudaStream_t st = (cudaStream_t)stream;
  char* ws = (char*)d_workspace;
  // zero the small control/state regions the kernel expects cleared
  cudaError_t e;
  e = cudaMemsetAsync(ws + L.off[27], 0, 64, st);
  if (e == cudaSuccess) e = cudaMemsetAsync(ws + L.off[28], 0, 64, st);
  if (e == cudaSuccess) e = cudaMemsetAsync(ws + L.off[7], 0, L.off[8] - L.off[7], st);
  if (e == cudaSuccess) e = cudaMemsetAsync(d_iters_out, 0, sizeof(int64_t) * R, st);
  if (e != cudaSuccess) return set_cuda_error("cudaMemsetAsync", e);

  auto fill = [&](auto* prm_ptr) {
    fill_prm(*prm_ptr, g, R, ld, p, nA, tol, maxit, track, d_W, ldw, d_tau, d_active, d_active_pos, d_X_out, x_f32,
             ldx, d_h_out, d_iters_out, ws, L, g_solver_mode == 0);
  };
  int rc;
  if (g_solver_mode == 0) {
    MkResult res{};
    if (precision == POLAR_MIXED) {
      SolvePrm<float> prm;
      fill(&prm);
      SolvePrm<float>* dp = (SolvePrm<float>*)(ws + L.off[30]);
      if (vec == 4) rc = weighted ? mk_solve<float, 4, true, POLAR_E32>(prm, dp, st, &res) : mk_solve<float, 4, false, POLAR_E32>(prm, dp, st, &res);
      else if (vec == 2) rc = weighted ? mk_solve<float, 2, true, POLAR_E32>(prm, dp, st, &res) : mk_solve<float, 2, false, POLAR_E32>(prm, dp, st, &res);
      else rc = weighted ? mk_solve<float, 1, true, POLAR_E32>(prm, dp, st, &res) : mk_solve<float, 1, false, POLAR_E32>(prm, dp, st, &res);
    } else {
      SolvePrm<double> prm;
      fill(&prm);
      SolvePrm<double>* dp = (SolvePrm<double>*)(ws + L.off[30]);
      if (vec == 2) rc = weighted ? mk_solve<double, 2, true, POLAR_E64>(prm, dp, st, &res) : mk_solve<double, 2, false, POLAR_E64>(prm, dp, st, &res);
      else rc = weighted ? mk_solve<double, 1, true, POLAR_E64>(prm, dp, st, &res) : mk_solve<double, 1, false, POLAR_E64>(prm, dp, st, &res);
    }
    if (rc != POLAR_OK) return rc;
    const int status = res.err ? res.err : (res.capped ? (int)POLAR_ERR_ITER_CAP : 0);
    remember_solve_done(d_workspace, status, res.iterations, res.flushes, ld, res.grid, kBlock);
    return POLAR_OK;
  }
  if (precision == POLAR_MIXED) {
    SolvePrm<float> prm;
    fill(&prm);
    if (vec == 4) rc = weighted ? launch_solve<float, 4, true, POLAR_E32>(prm, grid, st) : launch_solve<float, 4, false, POLAR_E32>(prm, grid, st);
    else if (vec == 2) rc = weighted ? launch_solve<float, 2, true, POLAR_E32>(prm, grid, st) : launch_solve<float, 2, false, POLAR_E32>(prm, grid, st);
    else rc = weighted ? launch_solve<float, 1, true, POLAR_E32>(prm, grid, st) : launch_solve<float, 1, false, POLAR_E32>(prm, grid, st);
  } else {
    SolvePrm<double> prm;
    fill(&prm);
    if (vec == 2) rc = weighted ? launch_solve<double, 2, true, POLAR_E64>(prm, grid, st) : launch_solve<double, 2, false, POLAR_E64>(prm, grid, st);
    else rc = weighted ? launch_solve<double, 1, true, POLAR_E64>(prm, grid, st) : launch_solve<double, 1, false, POLAR_E64>(prm, grid, st);
  }
  if (rc != POLAR_OK) return rc;
  // remember the control block location for polar_msolve_finish
  remember_solve(d_workspace, (int*)(ws + L.off[27]), (long long*)(ws + L.off[28]), ld, grid, kBlock);
  return POLAR_OK;
}

extern "C" int polar_msolve_finish(void* d_workspace, polar_stream_t stream, polar_msolve_info* info) {
  clear_error();
  SolveRecord rec;
  if (!lookup_solve(d_workspace, &rec)) return set_error(POLAR_ERR_BAD_ARG, "no solve launched on this workspace");
  if (rec.done) {
    if (info) {
      memset(info, 0, sizeof(*info));
      info->status = rec.status;
      info->ld = rec.ld;
      info->grid = rec.grid;
      info->block = rec.block;
      info->iterations = rec.iterations;
      info->flushes = rec.flushes;
    }
    if (rec.status == POLAR_ERR_ITER_CAP) return set_error(rec.status, "multi-shift CG iteration cap");
    if (rec.status == POLAR_ERR_NONFINITE) return set_error(rec.status, "non-finite value in CG");
    return rec.status;
  }
  int ctl[4];
  long long stats[8];
  cudaStream_t st = (cudaStream_t)stream;
  cudaError_t e = cudaMemcpyAsync(ctl, rec.ctl, sizeof(ctl), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(stats, rec.stats, sizeof(stats), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return set_cuda_error("msolve finish", e);
  int status = ctl[1] != 0 ? ctl[1] : ctl[0];
  if (info) {
    info->status = status;
    info->ld = rec.ld;
    info->grid = rec.grid;
    info->block = rec.block;
    info->iterations = stats[0];
    info->flushes = stats[1];
    info->error_where = ctl[2];
    info->pad = 0;
    for (int i = 0; i < 6; ++i) info->phase_ns[i] = stats[2 + i];
  }
  if (status == POLAR_ERR_ITER_CAP) return set_error(status, "multi-shift CG iteration cap");
  if (status == POLAR_ERR_NONFINITE) return set_error(status, "non-finite value in CG");
  if (status == POLAR_ERR_TIMEOUT) return set_error(status, "grid barrier wait timed out");
  return status;
}

// ---------------------------------------------------------------------------------------
// Batched solves: many graphs (or many right-hand-side blocks) in one cooperative launch
// of the persistent kernel, the CTAs split between the problems in proportion to their
// work.
namespace polar {

static_assert(sizeof(SolvePrm<double>) <= 4096 && sizeof(SolvePrm<float>) <= 4096,
              "parameter block must fit its workspace region");

template <typename T, int VEC, bool WEIGHTED, int E>
static int batch_occupancy() {
  int nb = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, msolve_batch_kernel<T, VEC, WEIGHTED, E>, kBlock, 0);
  return nb;
}

static int batch_grid_max(int precision, int vec, bool weighted) {
  int dev = 0, sms = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  int nb = 0;
  if (precision == POLAR_MIXED) {
    if (vec == 4) nb = weighted ? batch_occupancy<float, 4, true, POLAR_E32>() : batch_occupancy<float, 4, false, POLAR_E32>();
    else if (vec == 2) nb = weighted ? batch_occupancy<float, 2, true, POLAR_E32>() : batch_occupancy<float, 2, false, POLAR_E32>();
    else nb = weighted ? batch_occupancy<float, 1, true, POLAR_E32>() : batch_occupancy<float, 1, false, POLAR_E32>();
  } else {
    if (vec == 2) nb = weighted ? batch_occupancy<double, 2, true, POLAR_E64>() : batch_occupancy<double, 2, false, POLAR_E64>();
    else nb = weighted ? batch_occupancy<double, 1, true, POLAR_E64>() : batch_occupancy<double, 1, false, POLAR_E64>();
  }
  if (nb < 1) nb = 1;
  return nb * sms;
}

template <typename T, int VEC, bool WEIGHTED, int E>
static int launch_batch(const BatchPrm& B, int grid, cudaStream_t st) {
  void* args[] = {(void*)&B};
  cudaError_t e = cudaLaunchCooperativeKernel((const void*)msolve_batch_kernel<T, VEC, WEIGHTED, E>, dim3(grid),
                                              dim3(kBlock), args, 0, st);
  count_launch();
  if (e != cudaSuccess) return set_cuda_error("cudaLaunchCooperativeKernel(msolve batch)", e);
  return POLAR_OK;
}

}  // namespace polar

// Kernel-per-phase driver for a batch: every problem's solve on its own stream with its
// grids scaled to its rows (a problem too small to fill the GPU takes a share of it), the
// host relaunching each solve's iteration block as soon as the previous one drains.
template <typename T, int VEC, bool W, int E>
static int batch_graph_run(const polar_msolve_problem* probs, int nprob, int ld, const std::vector<SolveLayout>& L,
                           cudaStream_t st) {
  std::vector<SolvePrm<T>> prm(nprob);
  std::vector<double> frac(nprob);
  const int full = mk_grid_max<T, VEC, W, E>();
  for (int b = 0; b < nprob; ++b) {
    const polar_msolve_problem& q = probs[b];
    char* ws = (char*)q.d_workspace;
    cudaError_t e = cudaMemsetAsync(ws + L[b].off[27], 0, 64, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(ws + L[b].off[28], 0, 64, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(ws + L[b].off[7], 0, L[b].off[8] - L[b].off[7], st);
    if (e == cudaSuccess) e = cudaMemsetAsync(q.d_iters_out, 0, sizeof(int64_t) * q.R, st);
    if (e != cudaSuccess) return set_cuda_error("cudaMemsetAsync (batch)", e);
    fill_prm(prm[b], q.g, q.R, ld, q.p, q.nA, q.tol, q.maxit, q.track, q.d_W, q.ldw, q.d_tau, q.d_active,
             q.d_active_pos, q.d_X_out, q.x_f32, q.ldx, q.d_h_out, q.d_iters_out, ws, L[b], true);
    prm[b].hot_rows /= nprob;  // concurrent solves share the L2
    // two row items per thread of the full grid count as a full share
    const double items = (double)q.g->n * (ld / VEC);
    const double f = items / ((double)full * kBlock * 2.0);
    frac[b] = f < 1.0 ? f : 1.0;
  }
  std::vector<MkResult> res;
  const int rc = mk_solve_batch<T, VEC, W, E>(prm, frac, st, res);
  if (rc != POLAR_OK) return rc;
  for (int b = 0; b < nprob; ++b) {
    const int status = res[b].err ? res[b].err : (res[b].capped ? (int)POLAR_ERR_ITER_CAP : 0);
    remember_solve_done(probs[b].d_workspace, status, res[b].iterations, res[b].flushes, ld, res[b].grid, kBlock);
  }
  return POLAR_OK;
}

static int batch_graph_driver(const polar_msolve_problem* probs, int nprob, int precision, int ld, int vec,
                              bool weighted, const std::vector<SolveLayout>& L, cudaStream_t st) {
  if (precision == POLAR_MIXED) {
    if (vec == 4) return weighted ? batch_graph_run<float, 4, true, POLAR_E32>(probs, nprob, ld, L, st)
                                  : batch_graph_run<float, 4, false, POLAR_E32>(probs, nprob, ld, L, st);
    if (vec == 2) return weighted ? batch_graph_run<float, 2, true, POLAR_E32>(probs, nprob, ld, L, st)
                                  : batch_graph_run<float, 2, false, POLAR_E32>(probs, nprob, ld, L, st);
    return weighted ? batch_graph_run<float, 1, true, POLAR_E32>(probs, nprob, ld, L, st)
                    : batch_graph_run<float, 1, false, POLAR_E32>(probs, nprob, ld, L, st);
  }
  if (vec == 2) return weighted ? batch_graph_run<double, 2, true, POLAR_E64>(probs, nprob, ld, L, st)
                                : batch_graph_run<double, 2, false, POLAR_E64>(probs, nprob, ld, L, st);
  return weighted ? batch_graph_run<double, 1, true, POLAR_E64>(probs, nprob, ld, L, st)
                  : batch_graph_run<double, 1, false, POLAR_E64>(probs, nprob, ld, L, st);
}

static int batch_layout_grid(int precision, int vec, bool weighted) {
  return g_solver_mode == 0 ? grid_for_mode(precision, vec, weighted) : batch_grid_max(precision, vec, weighted);
}

extern "C" size_t polar_msolve_batch_workspace_bytes(const polar_graph* g, int precision, int R, int p, int nA) {
  if (!g || R < 1 || p < 1 || nA < 0) return 0;
  const int ld = choose_ld(precision, R);
  SolveLayout L;
  solve_layout(g, precision, R, p, nA, batch_layout_grid(precision, choose_vec(precision, ld), g->d_wts != nullptr),
               &L);
  return L.total;
}

extern "C" int polar_msolve_batch(const polar_msolve_problem* probs, int nprob, int precision,
                                  polar_stream_t stream) {
  clear_error();
  if (!probs || nprob < 1) return set_error(POLAR_ERR_BAD_ARG, "no problems");
  if (nprob > kMaxBatch) return set_error(POLAR_ERR_BAD_ARG, "at most 64 problems per batch");
  if (precision != POLAR_FP64 && precision != POLAR_MIXED) return set_error(POLAR_ERR_BAD_ARG, "precision");
  const int ld = choose_ld(precision, probs[0].R);
  const bool weighted = probs[0].g && probs[0].g->d_wts != nullptr;
  for (int b = 0; b < nprob; ++b) {
    const polar_msolve_problem& q = probs[b];
    const polar_graph* g = q.g;
    if (!g || !q.d_W || !q.d_tau || !q.d_active || !q.d_active_pos || !q.d_X_out || !q.d_iters_out || !q.d_workspace)
      return set_error(POLAR_ERR_BAD_ARG, "null pointer in a batch problem");
    if (q.R < 1 || q.R > max_ld(precision)) return set_error(POLAR_ERR_BAD_ARG, "R out of range for this precision");
    if (q.p < 1 || q.nA < 1 || q.ldw < q.R || q.ldx < q.R || g->n < 1)
      return set_error(POLAR_ERR_BAD_ARG, "bad sizes in a batch problem");
    if (q.track && !q.d_h_out) return set_error(POLAR_ERR_BAD_ARG, "track needs h_out");
    if ((g->d_wts == nullptr) != (g->d_diag == nullptr)) return set_error(POLAR_ERR_BAD_ARG, "weights and diag go together");
    if (choose_ld(precision, q.R) != ld) return set_error(POLAR_ERR_BAD_ARG, "batch problems must share the padded width");
    if ((g->d_wts != nullptr) != weighted) return set_error(POLAR_ERR_BAD_ARG, "batch problems must all be weighted or all unweighted");
  }
  const int vec = choose_vec(precision, ld);
  const int gmax = batch_layout_grid(precision, vec, weighted);
  if (g_solver_mode != 0 && nprob > gmax) return set_error(POLAR_ERR_BAD_ARG, "more problems than co-resident CTAs");
  std::vector<SolveLayout> L(nprob);
  std::vector<double> cost(nprob);
  std::vector<int> cap(nprob), ctas;
  for (int b = 0; b < nprob; ++b) {
    const polar_msolve_problem& q = probs[b];
    solve_layout(q.g, precision, q.R, q.p, q.nA, gmax, &L[b]);
    if (q.workspace_bytes < L[b].total) return set_error(POLAR_ERR_WORKSPACE, "workspace too small (batch problem)");
    const double n = q.g->n, nnz = q.g->nnz;
    cost[b] = q.cost > 0.0 ? q.cost : (nnz + 2.0 * n) * ld / sqrt(q.g->sigma > 0.0 ? q.g->sigma : 1.0);
    const long long items = (long long)q.g->n * (ld / vec);
    long long c = (items + 2LL * kBlock - 1) / (2LL * kBlock);
    cap[b] = (int)(c < 1 ? 1 : (c > gmax ? gmax : c));
  }
  // each problem's barrier words and scratch live in its own workspace: no sharing
  for (int b = 0; b < nprob; ++b)
    for (int c = b + 1; c < nprob; ++c) {
      const char* b0 = (const char*)probs[b].d_workspace;
      const char* c0 = (const char*)probs[c].d_workspace;
      if (b0 < c0 + L[c].total && c0 < b0 + L[b].total)
        return set_error(POLAR_ERR_BAD_ARG, "batch problems must not share workspace memory");
    }
  cudaStream_t st = (cudaStream_t)stream;
  if (g_solver_mode == 0) return batch_graph_driver(probs, nprob, precision, ld, vec, weighted, L, st);
  split_ctas(cost, cap, gmax, ctas);
  BatchPrm B;
  memset(&B, 0, sizeof(B));
  B.nprob = nprob;
  B.cta_off[0] = 0;
  for (int b = 0; b < nprob; ++b) B.cta_off[b + 1] = B.cta_off[b] + ctas[b];
  const int grid = B.cta_off[nprob];
  for (int b = 0; b < nprob; ++b) {
    const polar_msolve_problem& q = probs[b];
    char* ws = (char*)q.d_workspace;
    cudaError_t e = cudaMemsetAsync(ws + L[b].off[27], 0, 64, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(ws + L[b].off[28], 0, 64, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(ws + L[b].off[7], 0, L[b].off[8] - L[b].off[7], st);
    if (e == cudaSuccess) e = cudaMemsetAsync(q.d_iters_out, 0, sizeof(int64_t) * q.R, st);
    if (e != cudaSuccess) return set_cuda_error("cudaMemsetAsync (batch)", e);
    if (precision == POLAR_MIXED) {
      SolvePrm<float> prm;
      fill_prm(prm, q.g, q.R, ld, q.p, q.nA, q.tol, q.maxit, q.track, q.d_W, q.ldw, q.d_tau, q.d_active,
               q.d_active_pos, q.d_X_out, q.x_f32, q.ldx, q.d_h_out, q.d_iters_out, ws, L[b], false);
      e = cudaMemcpyAsync(ws + L[b].off[30], &prm, sizeof(prm), cudaMemcpyHostToDevice, st);
    } else {
      SolvePrm<double> prm;
      fill_prm(prm, q.g, q.R, ld, q.p, q.nA, q.tol, q.maxit, q.track, q.d_W, q.ldw, q.d_tau, q.d_active,
               q.d_active_pos, q.d_X_out, q.x_f32, q.ldx, q.d_h_out, q.d_iters_out, ws, L[b], false);
      e = cudaMemcpyAsync(ws + L[b].off[30], &prm, sizeof(prm), cudaMemcpyHostToDevice, st);
    }
    if (e != cudaSuccess) return set_cuda_error("parameter block upload (batch)", e);
    B.prm[b] = ws + L[b].off[30];
  }
  int rc;
  if (precision == POLAR_MIXED) {
    if (vec == 4) rc = weighted ? launch_batch<float, 4, true, POLAR_E32>(B, grid, st) : launch_batch<float, 4, false, POLAR_E32>(B, grid, st);
    else if (vec == 2) rc = weighted ? launch_batch<float, 2, true, POLAR_E32>(B, grid, st) : launch_batch<float, 2, false, POLAR_E32>(B, grid, st);
    else rc = weighted ? launch_batch<float, 1, true, POLAR_E32>(B, grid, st) : launch_batch<float, 1, false, POLAR_E32>(B, grid, st);
  } else {
    if (vec == 2) rc = weighted ? launch_batch<double, 2, true, POLAR_E64>(B, grid, st) : launch_batch<double, 2, false, POLAR_E64>(B, grid, st);
    else rc = weighted ? launch_batch<double, 1, true, POLAR_E64>(B, grid, st) : launch_batch<double, 1, false, POLAR_E64>(B, grid, st);
  }
  if (rc != POLAR_OK) return rc;
  for (int b = 0; b < nprob; ++b) {
    char* ws = (char*)probs[b].d_workspace;
    remember_solve(probs[b].d_workspace, (int*)(ws + L[b].off[27]), (long long*)(ws + L[b].off[28]), ld, ctas[b], kBlock);
  }
  return POLAR_OK;
}
