/* polar.h — C ABI of libpolar.so, the sm_100a kernels behind polar_b200.
 *
 * All pointers named d_* are device pointers (any allocator; the Python host passes
 * torch tensors' data_ptr()).  Host structs are passed by pointer.  Every entry point
 * returns a status code (POLAR_OK == 0).  Launches are asynchronous on `stream`
 * unless stated otherwise; nothing here allocates device memory except where a
 * function says so; scratch memory comes from a caller-provided workspace whose size
 * is queried first.
 *
 * Reference interfaces replaced (chenty2333/POLAR):
 *   polar_spmm            <- realworld/spmm.py:4-25 (csr_spmm + spmm wrapper) and
 *                            realworld/polar_gpu.py:71-80 (Op.__call__: shift + added edges)
 *   polar_msolve          <- realworld/polar_gpu.py:88-133 (msolve)
 *   polar_pair_norms      <- realworld/polar_gpu.py:205 (bank caches h, t)
 *   polar_score_topb      <- realworld/polar_gpu.py:208-211, 219-221 (proxy, argsort top-B)
 *   polar_rerank          <- realworld/polar_gpu.py:229-237, 284-288 (G_q re-rank / marginal)
 *   polar_maintain        <- realworld/polar_gpu.py:242-249 (Sherman–Morrison maintenance)
 *   polar_fill_incidence  <- realworld/polar_gpu.py:225-226, 282 (incidence right-hand sides)
 *   polar_select          <- realworld/polar_gpu.py:221-223, 236-237, 240 (winner, live mask)
 *   polar_rank1_rows      <- realworld/polar_gpu.py:250 (F[a] += Gc[e]; F[b] -= Gc[e])
 */
#ifndef POLAR_H
#define POLAR_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef void* polar_stream_t; /* a cudaStream_t */

enum polar_status {
  POLAR_OK = 0,
  POLAR_ERR_ITER_CAP = 1,   /* CG reached maxit with a column unconverged (polar_gpu.py:129) */
  POLAR_ERR_NONFINITE = 2,  /* NaN/Inf in a right-hand side or a CG scalar */
  POLAR_ERR_BAD_ARG = 3,    /* rejected before launch */
  POLAR_ERR_WORKSPACE = 4,  /* workspace too small */
  POLAR_ERR_TIMEOUT = 5,    /* a grid barrier wait exceeded its time limit */
  POLAR_ERR_CUDA = 6,       /* a CUDA runtime call failed (see polar_last_error) */
  POLAR_ERR_UNSUPPORTED = 7
};

enum polar_precision {
  POLAR_FP64 = 0,  /* every vector and scalar in FP64 (the parity path) */
  POLAR_MIXED = 1  /* FP32 vectors / SpMM / shifted iterates, FP64 scalars and dot products */
};

/* Graph operator M = L + sigma I + sum_S w_e b_e b_e^T (+ shift I at apply time).
 * The CSR holds only the off-diagonal neighbour lists of L (no diagonal entries).
 * Unweighted graphs pass d_wts = d_diag = NULL: every neighbour weight is 1 and the
 * diagonal is (indptr[i+1]-indptr[i]) + sigma.  Added edges (Op.add) are a sorted list
 * of rows that carry extra neighbours (x_*), flagged in the bitset d_xbits.  Rows with
 * more than heavy_thresh neighbours are split into chunks (h_*), combined in a fixed
 * order so results are deterministic.  All other rows are covered by row blocks
 * (d_rowblk): contiguous row ranges of bounded work that the SpMM streams through. */
typedef struct polar_graph {
  int32_t n;
  int32_t nnz;
  const int32_t* d_indptr;   /* n+1 */
  const int32_t* d_indices;  /* nnz */
  const double* d_wts;       /* nnz or NULL */
  const double* d_diag;      /* n or NULL (weighted degree + sigma) */
  double sigma;
  /* added edges */
  int32_t nx;                /* rows with added neighbours */
  const uint32_t* d_xbits;   /* (n+31)/32 words, or NULL when nx == 0 */
  const int32_t* d_xrow;     /* nx, ascending */
  const int32_t* d_xoff;     /* nx+1 */
  const int32_t* d_xnbr;     /* xoff[nx] */
  const double* d_xwt;       /* xoff[nx] or NULL (weight 1) */
  /* heavy-row split */
  int32_t heavy_thresh;
  int32_t nheavy;
  int32_t nchunks;
  const int32_t* d_hrow;       /* nheavy: row id */
  const int32_t* d_hchunk_off; /* nheavy+1: chunk range of each heavy row */
  const int32_t* d_chunk_row;  /* nchunks: heavy index */
  const int32_t* d_chunk_lo;   /* nchunks: first nnz position */
  const int32_t* d_chunk_hi;   /* nchunks: one past last */
  /* light rows in contiguous blocks of roughly equal work (heavy rows excluded) */
  int32_t nrb;
  const int32_t* d_rowblk;     /* 2*nrb: [first row, one past last row] */
  /* optional sliced ELL of the light rows (unweighted graphs): slices of sell_s rows,
   * sorted by degree; neighbour k of slice row r at sl_idx[sl_off[s] + k*sell_s + r],
   * -1 pads; sl_rows[s*sell_s + r] = row id or -1.  nsl == 0: not provided. */
  int32_t nsl;
  int32_t sell_s;
  const int32_t* d_sl_off;     /* nsl+1 */
  const int32_t* d_sl_rows;    /* nsl*sell_s */
  const int32_t* d_sl_idx;
} polar_graph;

/* Statistics of the last solve (filled by polar_msolve_finish). */
typedef struct polar_msolve_info {
  int32_t status;
  int32_t ld;            /* padded column count used internally */
  int32_t grid;          /* CTAs of the persistent launch */
  int32_t block;         /* threads per CTA */
  int64_t iterations;    /* seed iterations executed (max over columns) */
  int64_t flushes;       /* deferred shifted-update passes */
  int32_t error_where;   /* phase code where a barrier wait timed out (0 = none) */
  int32_t pad;
  /* wall time per phase seen by CTA 0, barriers included (ns): [0] deferred shifted
   * updates, [1] SpMM + d.v reduction, [2] residual update + r.r reduction,
   * [3] pole recurrences + direction update, [4] final pass, [5] initialisation */
  int64_t phase_ns[6];
} polar_msolve_info;

/* ---- error text of the last failing call on this host thread ---- */
const char* polar_last_error(void);
int polar_version(void);

/* ---- instrumentation ----
 * polar_launch_count: kernels launched by this library so far (all entry points).
 * polar_set_kernel_timing(1) resets and enables per-class device timing of the
 * solver's kernels (CUDA events around each launch); polar_kernel_timing returns, for
 * class 0 SpMM (light rows), 6 SpMM heavy-row launch, 1 residual update,
 * 2 direction/pole update, 3 deferred update, 4 init, the number of timed launches, their
 * summed device time (ms) and summed algorithmic bytes (SpMM, both launches together,
 * counted on class 0: 4(n+1) + 4 nnz + 2 s n R; residual, r in FP64: (16 + s) n R + s nA R;
 * direction: 24 n R (r and the direction in, the direction out; in mixed precision the
 * direction is an FP32 value plus its FP32 remainder); deferred update: (4p + M) s nA R). */
long long polar_launch_count(void);
void polar_set_kernel_timing(int on);
int polar_kernel_timing(int cls, long long* launches, double* ms, double* bytes);

/* ---- SpMM: Y = (M + shift I) X for an R-column row-major block ----
 * Replaces realworld/spmm.py:4-25 and polar_gpu.py:71-80.  dtype: POLAR_FP64 -> double
 * X/Y, POLAR_MIXED -> float X/Y.  ldx, ldy in elements.  d_scratch: chunk partials
 * (nchunks * ld accumulators) and nheavy counters; size from polar_spmm_scratch_bytes.
 * The counters must be zero before the first call (polar_spmm_scratch_init). */
size_t polar_spmm_scratch_bytes(const polar_graph* g, int precision, int R);
int polar_spmm_scratch_init(const polar_graph* g, int precision, int R, void* d_scratch,
                            polar_stream_t stream);
int polar_spmm(const polar_graph* g, int precision, int R, double shift, const void* d_X, int ldx,
               void* d_Y, int ldy, void* d_scratch, polar_stream_t stream);
/* Same apply as polar_spmm with the heavy-row scratch in a fixed 8 MiB device array inside
 * the library, so the call allocates nothing.  No counterpart in the reference: it serves
 * callers that may not allocate device memory when they apply the operator.  Arguments are
 * checked as polar_spmm checks them before anything is queued (POLAR_ERR_BAD_ARG leaves
 * the stream untouched); POLAR_ERR_WORKSPACE when polar_spmm_scratch_bytes(g, precision, R)
 * exceeds 8 MiB.  The first call on each device, and the first call in a new context (for
 * instance after cudaDeviceReset), resolves the array's address (cudaGetSymbolAddress)
 * and should come before any stream capture.  All calls on a device share the array: calls
 * that overlap in time race and must be serialised by the caller. */
int polar_spmm_noalloc(const polar_graph* g, int precision, int R, double shift, const void* d_X, int ldx,
                       void* d_Y, int ldy, polar_stream_t stream);

/* ---- multi-shift CG (polar_gpu.py:88-133) ----
 * Solves (M + tau_j I) U_j = W for all p poles and R columns.  W: n x R FP64 row-major
 * (ldw).  Pole iterates are kept on the nA active rows (d_active: ids ascending;
 * d_active_pos: n entries, row -> active index or -1).  Outputs: X_out[p][nA][ldx]
 * (x_f32 ? float : double) written at column offset 0..R-1, h_out[p][R] (tracked
 * ||U_j[:,c]||^2, only when track), iters_out[R].  maxit: iteration cap (status
 * POLAR_ERR_ITER_CAP when hit).
 * BLOCKING with the default driver (polar_set_solver_mode(0)): the call queues blocks of
 * 16 iterations on `stream` as CUDA-graph launches and synchronises `stream` after each
 * block to read the convergence flags, so it returns only when the solve has ended (the
 * host loop stands in for the reference's host-side convergence check every 8 iterations,
 * polar_gpu.py:126).  It therefore cannot be captured into a caller's CUDA graph.  With
 * driver 1 the call returns after one cooperative launch.  In both cases
 * polar_msolve_finish synchronises the stream and returns the solve status. */
size_t polar_msolve_workspace_bytes(const polar_graph* g, int precision, int R, int p, int nA);
int polar_msolve(const polar_graph* g, int precision, const double* d_W, int ldw, int R,
                 const double* d_tau, int p, const int32_t* d_active, const int32_t* d_active_pos,
                 int nA, double tol, int64_t maxit, int track, void* d_X_out, int x_f32, int ldx,
                 double* d_h_out, int64_t* d_iters_out, void* d_workspace, size_t workspace_bytes,
                 polar_stream_t stream);
int polar_msolve_finish(void* d_workspace, polar_stream_t stream, polar_msolve_info* info);
/* Host-side limit for each grid-barrier wait inside polar_msolve (nanoseconds). */
void polar_set_barrier_timeout_ns(uint64_t ns);
/* Solver driver: 0 (default) one high-occupancy kernel per phase, M iterations per
 * CUDA-graph launch, host checks convergence once per launch (polar_msolve then returns
 * after the solve); 1: one persistent cooperative kernel with bounded grid barriers. */
int polar_set_solver_mode(int mode);
/* Degree above which polar_msolve expects a row to be chunked for an R-column solve in
 * this precision: 8 x (lanes per row).  Heavy rows are split into chunks of at most 256
 * neighbours (polar_graph h_* fields), each processed by one warp. */
int polar_heavy_threshold(int precision, int R);
/* Rows per warp of the sliced-ELL layout polar_msolve uses for an R-column solve in this
 * precision (0: it uses the CSR row loop). */
int polar_sell_rows(int precision, int R);
/* Bytes of each row that one lane of the solver's SpMM owns (16, 32 or 64; 0 = default 64).
 * A row is processed by ld * element_size / bytes lanes. */
void polar_set_spmm_lane_bytes(int bytes);
/* 1 (default): polar_sell_rows reports the sliced-ELL height the solver uses; 0: CSR rows. */
void polar_set_sell(int on);
/* L2 eviction priorities of the solver's SpMM and direction update (default driver only):
 * mode 0 none; 1: the first hot_bytes / (row bytes) rows of the direction (the most
 * gathered rows of a degree-ordered graph) are gathered and stored with evict_last, the
 * neighbour indices and the SpMM output with evict_first; 2 (default, 32 MB): as 1, with
 * gathers of the other rows evict_first too.  Caching only: results are identical in
 * every mode. */
int polar_set_l2_policy(int mode, size_t hot_bytes);
/* Residual storage of the mixed-precision solve (default driver): 64 (default) keeps r in
 * FP64; 32 stores r in FP32 (rounded after every update, norms taken of the stored value),
 * with the direction still held to FP64 accuracy as an FP32 value plus FP32 remainder. */
int polar_set_mixed_residual(int bits);

/* ---- batched multi-shift solves (many graphs at once) ----
 * Replaces a loop of realworld/polar_gpu.py:88-133 (msolve) calls, one per graph: the
 * reference solves one graph per call.  Each problem carries exactly the arguments of
 * polar_msolve (its own graph, right-hand sides, poles, active rows, tolerance and
 * outputs) and its own workspace of polar_msolve_batch_workspace_bytes.  All problems of a
 * batch share the precision, the padded width (next power of two of R) and weighted-ness;
 * each graph's partition uses polar_heavy_threshold / polar_sell_rows as for polar_msolve.
 * Driver 0 (default): every problem's solve runs on its own stream (ordered after
 * `stream`), with its grids scaled to its rows, and the host relaunches each solve's
 * iteration block as soon as the previous one drains; the call returns when all are done.
 * Driver 1 (polar_set_solver_mode(1)): one cooperative launch of the persistent solver;
 * problem b gets a share of the co-resident CTAs in proportion to `cost` (<= 0:
 * (nnz + 2n) * width / sqrt(sigma)), and its CTAs synchronise only among themselves, with
 * the same bounded waits as polar_msolve; at most as many problems as co-resident CTAs.
 * At most 64 problems.  polar_msolve_finish(d_workspace of problem b) returns problem b's
 * status and statistics. */
typedef struct polar_msolve_problem {
  const polar_graph* g;     /* host pointer, read during the call */
  const double* d_W;        /* n x R FP64, ldw */
  const double* d_tau;      /* p */
  const int32_t* d_active;  /* nA, ascending */
  const int32_t* d_active_pos; /* n: row -> active index or -1 */
  void* d_X_out;            /* [p][nA][ldx], float when x_f32 else double */
  double* d_h_out;          /* [p][R] when track, else NULL */
  int64_t* d_iters_out;     /* R */
  void* d_workspace;
  size_t workspace_bytes;
  double tol;
  int64_t maxit;
  double cost;              /* relative work for the CTA split; <= 0: estimated */
  int32_t ldw, R, p, nA, track, x_f32, ldx, pad;
} polar_msolve_problem;
size_t polar_msolve_batch_workspace_bytes(const polar_graph* g, int precision, int R, int p, int nA);
int polar_msolve_batch(const polar_msolve_problem* probs, int nprob, int precision, polar_stream_t stream);

/* ---- sketch construction (realworld/polar_gpu.py:137-165: _block_rows, sketches) ----
 * polar_block_orth: d_G holds ceil(rows/q) Gaussian q x q blocks, row-major
 * (G[b][r][j]), in the order the reference draws them.  Each block's columns are
 * orthonormalised in order (QR with a positive diagonal of R, as the reference's
 * sign-fixed numpy QR); row b*q + i of W (rows x q, ldw) receives column i of block b's
 * Q, times d_scale[b*q + i] when d_scale is given (the reference's U *= sqrt(w)).  q <= 128.
 * polar_center_columns: W (rows x q) -= its column means (the reference's W - W.mean(0)),
 * with a caller scratch of polar_center_columns_tmp_bytes(q).
 * polar_incidence_apply: F[i] += sum_k sign[k] * U[eidx[k]] over the CSR row i
 * (indptr n+1, eidx and int8 sign per entry): F += C^T U for one edge chunk of the
 * reference's F = C_0^T U. */
int polar_block_orth(const double* d_G, int64_t rows, int q, const double* d_scale, double* d_W, int ldw,
                     polar_stream_t stream);
size_t polar_center_columns_tmp_bytes(int q);
int polar_center_columns(double* d_W, int64_t rows, int q, int ldw, void* d_tmp, size_t tmp_bytes,
                         polar_stream_t stream);
int polar_incidence_apply(int n, const int32_t* d_indptr, const int32_t* d_eidx, const int8_t* d_sign,
                          const double* d_U, int ldu, int q, double* d_F, int ldf, polar_stream_t stream);

/* ---- incidence right-hand sides (polar_gpu.py:225-226, 282) ----
 * For c < R with e = sel[c] and (a, b) = cand[e] (cand: int64 [N][2]):
 * W[:, c] = e_a - e_b (n x R FP64, ldw; zeroed first).  When d_es (int32 [N][2], the
 * endpoints' active positions) is given, ia[c] = es[e][0] and ib[c] = es[e][1]. */
int polar_fill_incidence(int n, int R, const int64_t* d_cand, const int64_t* d_sel, const int32_t* d_es,
                         double* d_W, int ldw, int32_t* d_ia, int32_t* d_ib, polar_stream_t stream);

/* ---- bank caches (polar_gpu.py:205) ----
 * out[j][e] = sum_c (X[j][ea[e]][c] - X[j][eb[e]][c])^2 over q columns, FP64 out.
 * X is [p][nA][ldx] starting at column col0, float or double. */
int polar_pair_norms(const void* d_X, int x_f32, int p, int nA, int ldx, int col0, int q,
                     const int32_t* d_ea, const int32_t* d_eb, int N, double* d_out,
                     polar_stream_t stream);

/* ---- proxy score + stable top-B (polar_gpu.py:208-211, 219-221) ----
 * score[e] = sum_j om_j h_je / (1 + t_je + (sigma + tau_j) h_je)   (obj 0, 'frac'/'er')
 *          = log1p(t_0e + sigma h_0e)                                (obj 1, 'logdet')
 *          = sum_j om_j h_je                                         (obj 2: the sketched
 *            adjoint d f_s / d w_e at w = 0, the candidate screen; no reference counterpart)
 * Dead candidates (live[e] == 0) score -inf.  The B best by (score desc, index asc) —
 * the order of a stable argsort of -score — go to out_idx / out_score (device).
 * d_score_all (optional, N doubles) receives every candidate's score before the live
 * mask, dead candidates included.
 * d_tmp: polar_topb_tmp_bytes(N, B) bytes. */
size_t polar_topb_tmp_bytes(int N, int B);
int polar_score_topb(const double* d_h, const double* d_t, const double* d_tau, const double* d_om,
                     double sigma, int p, int N, const uint8_t* d_live, int obj, int B,
                     int64_t* d_out_idx, double* d_out_score, double* d_score_all, void* d_tmp,
                     polar_stream_t stream);

/* ---- re-rank (polar_gpu.py:229-237) ----
 * For shortlist column j: bu_j[pole] = U[pole][ia[j]][j] - U[pole][ib[j]][j];
 * gq[j] = sum_pole om hh[pole][j] / (1 + bu_j[pole])  (obj 0)  or log1p(bu_j[0]) (obj 1).
 * Writes gq (Br) and the winner position (first maximum) to d_best. */
int polar_rerank(const void* d_U, int u_f32, int p, int nA, int ldu, const int32_t* d_ia,
                 const int32_t* d_ib, int Br, const double* d_hh, const double* d_om, int obj,
                 double* d_gq, int32_t* d_best, polar_stream_t stream);

/* ---- winner selection (polar_gpu.py:221-223, 236-237, 240) ----
 * e = short[best ? *best : 0]; writes the winner record d_win (int32[6]):
 * win[0] = shortlist position, win[1] = es[e][0], win[2] = es[e][1], win[4..5] = e (int64),
 * and clears live[e] when d_live is given. */
int polar_select(const int64_t* d_short, const int32_t* d_best, const int32_t* d_es, uint8_t* d_live,
                 int32_t* d_win, polar_stream_t stream);

/* ---- maintenance (polar_gpu.py:242-249) ----
 * With the winner record d_win (see polar_select), its solve column U[:, :, win[0]] and
 * sketch row G[e] (G: FP64 [N][q]) updates X, Y ([p][nA][ld*], float or double):
 *   xi = X[:,aa]-X[:,bb], eta = G[e]-(Y[:,aa]-Y[:,bb]), D = 1+u[aa]-u[bb],
 *   X -= u xi^T / D, Y += u eta^T / D,
 * and the caches h, t ([p][N] FP64) through w^X = X xi, w^Y = Y eta (es: int32 [N][2]).
 * d_tmp: polar_maintain_tmp_bytes(p, nA, q). */
size_t polar_maintain_tmp_bytes(int p, int nA, int q);
int polar_maintain(void* d_X, int ldx, void* d_Y, int ldy, int xy_f32, int p, int nA, int q,
                   const void* d_U, int u_f32, int ldu, const int32_t* d_win, const double* d_G,
                   const int32_t* d_es, int N, double* d_h, double* d_t, void* d_tmp,
                   polar_stream_t stream);
/* Column-split maintenance (the q sketch columns spread over several GPUs, each holding
 * its own columns of X, Y and G): the same X, Y update on this GPU's q columns, with this
 * GPU's share of the cache change written to d_dh, d_dt ([p][N] FP64) instead of h, t:
 *   dh = cc^2 |xi|^2 - 2 cc (w^X[a] - w^X[b]),  dt = cc^2 |eta|^2 + 2 cc (w^Y[a] - w^Y[b]),
 * cc = (u[a] - u[b]) / D, norms and w over the local columns.  The shares summed over the
 * GPUs (an all-reduce) enter the caches through polar_cache_apply:
 *   h = max(0, h + dh), t = max(0, t + dt)   (count = p * N entries).
 * The reference's maintenance (polar_gpu.py:242-249) is the one-GPU case; it has no
 * column split. */
int polar_maintain_split(void* d_X, int ldx, void* d_Y, int ldy, int xy_f32, int p, int nA, int q,
                         const void* d_U, int u_f32, int ldu, const int32_t* d_win, const double* d_G,
                         const int32_t* d_es, int N, double* d_dh, double* d_dt, void* d_tmp,
                         polar_stream_t stream);
int polar_cache_apply(double* d_h, const double* d_dh, double* d_t, const double* d_dt, int64_t count,
                      polar_stream_t stream);

/* ---- F update (polar_gpu.py:250): with e = *sel, (a, b) = cand[e]:
 *      F[a] += G[e]; F[b] -= G[e]  (FP64 rows of q) ---- */
int polar_rank1_rows(double* d_F, int ldf, int q, const double* d_G, const int64_t* d_cand,
                     const int64_t* d_sel, polar_stream_t stream);

#ifdef __cplusplus
}
#endif
#endif /* POLAR_H */
