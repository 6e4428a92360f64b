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
//    stream capture.  The address is cached with the unique id of the context it was
//    resolved in (cuCtxGetId, fetched through cudaGetDriverEntryPointByVersion so the
//    library does not link libcuda); a call in a new context, for instance after
//    cudaDeviceReset, resolves it again;
//  * arguments are checked, with polar_spmm's own checks, before the counter clear is
//    queued: a rejected call leaves nothing on the stream;
//  * the buffer is shared by every call on a device, so calls that overlap in time
//    (other streams, other host threads) race on it and must be serialised by the caller.
#include <cuda.h>
#include <cudaTypedefs.h>
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
unsigned long long g_noalloc_ctx[kMaxDevices] = {};  // cuCtxGetId of the context g_noalloc_ptr was resolved in

PFN_cuCtxGetCurrent_v4000 g_ctx_current = nullptr;
PFN_cuCtxGetId_v12000 g_ctx_id = nullptr;

// Unique id of the current context (0 when none is current yet).
int current_context_id(unsigned long long* id) {
  if (!g_ctx_current || !g_ctx_id) {
    cudaDriverEntryPointQueryResult q1, q2;
    void* f1 = nullptr;
    void* f2 = nullptr;
    cudaError_t e = cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", &f1, 4000, cudaEnableDefault, &q1);
    if (e != cudaSuccess || q1 != cudaDriverEntryPointSuccess || !f1)
      return set_error(POLAR_ERR_CUDA, "polar_spmm_noalloc: cuCtxGetCurrent entry point");
    e = cudaGetDriverEntryPointByVersion("cuCtxGetId", &f2, 12000, cudaEnableDefault, &q2);
    if (e != cudaSuccess || q2 != cudaDriverEntryPointSuccess || !f2)
      return set_error(POLAR_ERR_CUDA, "polar_spmm_noalloc: cuCtxGetId entry point");
    g_ctx_current = reinterpret_cast<PFN_cuCtxGetCurrent_v4000>(f1);
    g_ctx_id = reinterpret_cast<PFN_cuCtxGetId_v12000>(f2);
  }
  CUcontext ctx = nullptr;
  if (g_ctx_current(&ctx) != CUDA_SUCCESS) return set_error(POLAR_ERR_CUDA, "polar_spmm_noalloc: cuCtxGetCurrent");
  *id = 0;
  if (ctx && g_ctx_id(ctx, id) != CUDA_SUCCESS) return set_error(POLAR_ERR_CUDA, "polar_spmm_noalloc: cuCtxGetId");
  return POLAR_OK;
}

// Address of g_noalloc_scratch on the current device, resolved once per device and
// context.
int noalloc_scratch(void** out) {
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return set_cuda_error("polar_spmm_noalloc: cudaGetDevice", e);
  if (dev < 0 || dev >= kMaxDevices) return set_error(POLAR_ERR_UNSUPPORTED, "polar_spmm_noalloc: device index above 63");
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  // cudaGetSymbolAddress makes the device's primary context current if none is, so the
  // context id is read after it when nothing is cached yet.
  unsigned long long ctx = 0;
  int rc = current_context_id(&ctx);
  if (rc != POLAR_OK) return rc;
  if (!g_noalloc_ptr[dev] || ctx == 0 || ctx != g_noalloc_ctx[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return set_cuda_error("polar_spmm_noalloc: cudaGetSymbolAddress", e);
    rc = current_context_id(&ctx);
    if (rc != POLAR_OK) return rc;
    g_noalloc_ptr[dev] = p;
    g_noalloc_ctx[dev] = ctx;
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
  const int rc0 = spmm_check_args(g, precision, R, d_X, ldx, d_Y, ldy);
  if (rc0 != POLAR_OK) return rc0;
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
  const size_t part = spmm_counter_offset(g, precision);
  cudaError_t e = cudaMemsetAsync(static_cast<char*>(scratch) + part, 0, need - part, (cudaStream_t)stream);
  if (e != cudaSuccess) return set_cuda_error("polar_spmm_noalloc: clear counters", e);
  return polar_spmm(g, precision, R, shift, d_X, ldx, d_Y, ldy, scratch, stream);
}
