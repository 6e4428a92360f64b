// polar_spmm_noalloc: the standalone operator apply Y = (M + shift I) X with its heavy-row
// scratch in a fixed device array instead of caller memory.
//
// Some callers cannot allocate device memory at the moment they want one operator
// apply: code running under another framework's caching allocator that must not
// grow it, a host callback or signal-free path that may not call cudaMalloc, or a
// plugin that owns no allocator at all.  For them this entry point uses a
// file-scope __device__ buffer of kNoAllocScratchBytes, fixed when the module loads.
//
// Limits, stated once here and in the header:
//  * scratch need (polar_spmm_scratch_bytes) above kNoAllocScratchBytes is rejected with
//    POLAR_ERR_WORKSPACE before anything is launched;
//  * the first call on each device resolves the buffer's address with
//    cudaGetSymbolAddress (which may load the module); make that first call before any
//    stream capture;
//  * the buffer is shared by every call on a device, so calls that overlap in time
//    (other streams, other host threads) race on it and must be serialised by the caller.
#include <cuda_runtime.h>

#include <cstdio>
#include <mutex>

#include "polar.h"
#include "host_util.h"

namespace polar {
namespace {

constexpr size_t kNoAllocScratchBytes = size_t(8) << 20;  // 8 MiB
constexpr int kMaxDevices = 64;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

std::mutex g_noalloc_mu;
void* g_noalloc_ptr[kMaxDevices] = {};

// Address of g_noalloc_scratch on the current device, resolved once per device.
int noalloc_scratch(void** out) {
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return set_cuda_error("polar_spmm_noalloc: cudaGetDevice", e);
  if (dev < 0 || dev >= kMaxDevices) return set_error(POLAR_ERR_UNSUPPORTED, "polar_spmm_noalloc: device index above 63");
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  if (!g_noalloc_ptr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return set_cuda_error("polar_spmm_noalloc: cudaGetSymbolAddress", e);
    g_noalloc_ptr[dev] = p;
  }
  *out = g_noalloc_ptr[dev];
  return POLAR_OK;
}

}  // namespace
}  // namespace polar

using namespace polar;

extern "C" int polar_spmm_noalloc(const polar_graph* g, int precision, int R, double shift, const void* d_X,
                                  int ldx, void* d_Y, int ldy, polar_stream_t stream) {
  clear_error();
  if (!g || !d_X || !d_Y) return set_error(POLAR_ERR_BAD_ARG, "polar_spmm_noalloc: null pointer");
  if (precision != POLAR_FP64 && precision != POLAR_MIXED)
    return set_error(POLAR_ERR_BAD_ARG, "polar_spmm_noalloc: precision");
  const size_t need = polar_spmm_scratch_bytes(g, precision, R);
  if (need > kNoAllocScratchBytes) {
    static thread_local char msg[192];
    snprintf(msg, sizeof(msg),
             "polar_spmm_noalloc: graph needs %zu bytes of heavy-row scratch, above the fixed %zu; "
             "use polar_spmm with caller scratch",
             need, kNoAllocScratchBytes);
    return set_error(POLAR_ERR_WORKSPACE, msg);
  }
  void* scratch = nullptr;
  int rc = noalloc_scratch(&scratch);
  if (rc != POLAR_OK) return rc;
  // Chunk partials are written before they are read; the heavy-row arrival counters
  // must start at zero.  They sit after the partials, as polar_spmm lays them out.
  const size_t es = precision == POLAR_MIXED ? 4 : 8;
  const size_t part = ((size_t)(g->nchunks > 0 ? g->nchunks : 1) * 128 * es + 255) & ~size_t(255);
  cudaError_t e = cudaMemsetAsync(static_cast<char*>(scratch) + part, 0, need - part, (cudaStream_t)stream);
  if (e != cudaSuccess) return set_cuda_error("polar_spmm_noalloc: clear counters", e);
  return polar_spmm(g, precision, R, shift, d_X, ldx, d_Y, ldy, scratch, stream);
}
