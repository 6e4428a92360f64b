// Sketch construction on the device (sm_100a): orthonormal row blocks, column centring and
// the incidence product F += C_0^T U (realworld/polar_gpu.py:137-165).
//
// The reference draws Gaussian q x q blocks from NumPy's generator, QR-factorises them on
// the host, fixes the signs so that R has a positive diagonal and uses the transposed Q
// factors as rows.  The draws stay on the host here (the generator's stream is what makes
// a seed reproduce the reference's sketches); the factorisation, the centring and the
// scatter of edge rows onto their endpoints run here.  A QR with a positive diagonal is
// unique, so classical Gram-Schmidt with one re-orthogonalisation pass (CGS2) in FP64
// yields the same Q as the reference's Householder factorisation, up to rounding.
#include <cuda_runtime.h>

#include <cmath>

#include "common.cuh"
#include "host_util.h"

namespace polar {

constexpr int kOrthThreads = 256;
constexpr int kOrthMaxQ = 128;

// One CTA per block: the block's q columns g_0..g_{q-1} (column j = entries G[b][r][j],
// r = 0..q-1) are orthonormalised in order; W row b*q + i receives column i of Q
// (scaled by scale[b*q + i] when given).  Rows at or past `rows` (the last block's
// padding) are not written.  Shared memory: Q (q x q, column-major) and q coefficients.
__global__ void __launch_bounds__(kOrthThreads) block_orth_kernel(const double* __restrict__ G, long long rows,
                                                                   int q, const double* __restrict__ scale,
                                                                   double* __restrict__ W, int ldw) {
  extern __shared__ double sm[];
  double* Qs = sm;              // Qs[j * q + r] = Q[r][j]
  double* cf = sm + q * q;      // projection coefficients
  __shared__ double s_norm;
  const long long b = blockIdx.x;
  const double* Gb = G + (size_t)b * q * q;
  for (int t = threadIdx.x; t < q * q; t += blockDim.x) {
    const int r = t / q, j = t % q;
    Qs[j * q + r] = Gb[t];
  }
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
  for (int j = 0; j < q; ++j) {
    double* v = Qs + j * q;
    for (int pass = 0; pass < 2; ++pass) {
      // cf[k] = Q_k . v for k < j (one warp per k)
      for (int k = warp; k < j; k += nwarp) {
        const double* qk = Qs + k * q;
        double s = 0.0;
        for (int r = lane; r < q; r += 32) s += qk[r] * v[r];
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (lane == 0) cf[k] = s;
      }
      __syncthreads();
      // v -= sum_k cf[k] Q_k (one thread per entry, k in order)
      for (int r = threadIdx.x; r < q; r += blockDim.x) {
        double x = v[r];
        for (int k = 0; k < j; ++k) x -= cf[k] * Qs[k * q + r];
        v[r] = x;
      }
      __syncthreads();
    }
    if (warp == 0) {
      double s = 0.0;
      for (int r = lane; r < q; r += 32) s += v[r] * v[r];
      for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
      if (lane == 0) s_norm = sqrt(s);
    }
    __syncthreads();
    const double inv = 1.0 / s_norm;
    for (int r = threadIdx.x; r < q; r += blockDim.x) v[r] *= inv;
    __syncthreads();
  }
  // W[b*q + i][c] = Q[c][i] = Qs[i * q + c]
  for (int t = threadIdx.x; t < q * q; t += blockDim.x) {
    const int i = t / q, c = t % q;
    const long long row = b * q + i;
    if (row < rows) {
      const double sc = scale ? scale[row] : 1.0;
      W[(size_t)row * ldw + c] = Qs[i * q + c] * sc;
    }
  }
}

// Column sums of W (rows x q) per CTA, rows in CTA-contiguous ranges, fixed order.
__global__ void column_partials_kernel(const double* __restrict__ W, long long rows, int q, int ldw,
                                       double* __restrict__ part) {
  const long long per = (rows + gridDim.x - 1) / gridDim.x;
  const long long r0 = (long long)blockIdx.x * per;
  const long long r1 = r0 + per < rows ? r0 + per : rows;
  for (int c = threadIdx.x; c < q; c += blockDim.x) {
    double s = 0.0;
    for (long long r = r0; r < r1; ++r) s += W[(size_t)r * ldw + c];
    part[(size_t)blockIdx.x * q + c] = s;
  }
}

// mean[c] = (sum of the partials in CTA order) / rows; one CTA.
__global__ void column_means_kernel(const double* __restrict__ part, int nparts, int q, long long rows,
                                    double* __restrict__ mean) {
  for (int c = threadIdx.x; c < q; c += blockDim.x) {
    double s = 0.0;
    for (int b = 0; b < nparts; ++b) s += part[(size_t)b * q + c];
    mean[c] = s / (double)rows;
  }
}

// W -= column means.
__global__ void center_columns_kernel(double* __restrict__ W, long long rows, int q, int ldw,
                                      const double* __restrict__ mean) {
  const long long total = rows * q;
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    const long long r = t / q;
    const int c = (int)(t % q);
    W[(size_t)r * ldw + c] -= mean[c];
  }
}

// F[i] += sum over the incidence row of i (edges in ascending order) of sign * U[e]:
// one warp per vertex, lanes over columns; the sum runs in the row's order.
__global__ void incidence_apply_kernel(int n, const int32_t* __restrict__ indptr, const int32_t* __restrict__ eidx,
                                       const int8_t* __restrict__ sign, const double* __restrict__ U, int ldu, int q,
                                       double* __restrict__ F, int ldf) {
  const int lane = threadIdx.x & 31;
  const long long i = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (i >= n) return;
  const int lo = indptr[i], hi = indptr[i + 1];
  for (int c = lane; c < q; c += 32) {
    double s = F[(size_t)i * ldf + c];
    for (int k = lo; k < hi; ++k) {
      const double u = U[(size_t)eidx[k] * ldu + c];
      s += sign[k] > 0 ? u : -u;
    }
    F[(size_t)i * ldf + c] = s;
  }
}

}  // namespace polar

using namespace polar;

extern "C" int polar_block_orth(const double* d_G, int64_t rows, int q, const double* d_scale, double* d_W, int ldw,
                                polar_stream_t stream) {
  clear_error();
  if (!d_G || !d_W) return set_error(POLAR_ERR_BAD_ARG, "null pointer");
  if (q < 1 || q > kOrthMaxQ || rows < 0 || ldw < q) return set_error(POLAR_ERR_BAD_ARG, "bad sizes");
  if (rows == 0) return POLAR_OK;
  const long long nb = (rows + q - 1) / q;
  if (nb > 0x7fffffffLL) return set_error(POLAR_ERR_BAD_ARG, "too many blocks");
  const size_t smem = sizeof(double) * ((size_t)q * q + q);
  static bool attr = false;
  if (!attr) {
    cudaFuncSetAttribute(block_orth_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)(sizeof(double) * (kOrthMaxQ * kOrthMaxQ + kOrthMaxQ)));
    attr = true;
  }
  block_orth_kernel<<<(unsigned)nb, kOrthThreads, smem, (cudaStream_t)stream>>>(d_G, rows, q, d_scale, d_W, ldw);
  count_launch();
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return set_cuda_error("block_orth_kernel", e);
  return POLAR_OK;
}

extern "C" size_t polar_center_columns_tmp_bytes(int q) { return sizeof(double) * 1025 * (size_t)(q > 0 ? q : 1); }

extern "C" int polar_center_columns(double* d_W, int64_t rows, int q, int ldw, void* d_tmp, size_t tmp_bytes,
                                    polar_stream_t stream) {
  clear_error();
  if (!d_W || !d_tmp) return set_error(POLAR_ERR_BAD_ARG, "null pointer");
  if (q < 1 || q > 1024 || rows < 1 || ldw < q) return set_error(POLAR_ERR_BAD_ARG, "bad sizes");
  if (tmp_bytes < polar_center_columns_tmp_bytes(q)) return set_error(POLAR_ERR_WORKSPACE, "tmp too small");
  cudaStream_t st = (cudaStream_t)stream;
  int nparts = (int)((rows + 255) / 256);
  if (nparts > 1024) nparts = 1024;
  double* part = (double*)d_tmp;        // nparts x q partial sums
  double* mean = part + (size_t)1024 * q;  // q column means
  column_partials_kernel<<<nparts, 128, 0, st>>>(d_W, rows, q, ldw, part);
  column_means_kernel<<<1, 128, 0, st>>>(part, nparts, q, rows, mean);
  const long long total = rows * q;
  long long g = (total + 255) / 256;
  if (g > 4096) g = 4096;
  center_columns_kernel<<<(unsigned)g, 256, 0, st>>>(d_W, rows, q, ldw, mean);
  count_launch(3);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return set_cuda_error("center_columns", e);
  return POLAR_OK;
}

extern "C" int polar_incidence_apply(int n, const int32_t* d_indptr, const int32_t* d_eidx, const int8_t* d_sign,
                                     const double* d_U, int ldu, int q, double* d_F, int ldf, polar_stream_t stream) {
  clear_error();
  if (!d_indptr || !d_U || !d_F) return set_error(POLAR_ERR_BAD_ARG, "null pointer");
  if (n < 0 || q < 1 || ldu < q || ldf < q) return set_error(POLAR_ERR_BAD_ARG, "bad sizes");
  if (n == 0) return POLAR_OK;
  const long long threads = (long long)n * 32;
  const unsigned grid = (unsigned)((threads + 255) / 256);
  incidence_apply_kernel<<<grid, 256, 0, (cudaStream_t)stream>>>(n, d_indptr, d_eidx, d_sign, d_U, ldu, q, d_F, ldf);
  count_launch();
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return set_cuda_error("incidence_apply_kernel", e);
  return POLAR_OK;
}
