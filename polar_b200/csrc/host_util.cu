// Error text and per-workspace solve records for the C ABI.
#include <cstdio>
#include <mutex>
#include <string>
#include <unordered_map>
#include <atomic>
#include <vector>

#include "host_util.h"
#include "polar.h"

namespace polar {

static thread_local std::string g_err;
static std::mutex g_mu;
static std::unordered_map<void*, SolveRecord> g_solves;

int set_error(int code, const char* msg) {
  g_err = msg ? msg : "";
  return code;
}

int set_cuda_error(const char* what, cudaError_t e) {
  char buf[512];
  snprintf(buf, sizeof(buf), "%s: %s (%d)", what, cudaGetErrorString(e), (int)e);
  g_err = buf;
  return POLAR_ERR_CUDA;
}

void clear_error() { g_err.clear(); }

void remember_solve(void* ws, int* ctl, long long* stats, int ld, int grid, int block) {
  std::lock_guard<std::mutex> lk(g_mu);
  g_solves[ws] = SolveRecord{ctl, stats, ld, grid, block, false, 0, 0, 0};
}

void remember_solve_done(void* ws, int status, long long iterations, long long flushes, int ld, int grid, int block) {
  std::lock_guard<std::mutex> lk(g_mu);
  g_solves[ws] = SolveRecord{nullptr, nullptr, ld, grid, block, true, status, iterations, flushes};
}

bool lookup_solve(void* ws, SolveRecord* out) {
  std::lock_guard<std::mutex> lk(g_mu);
  auto it = g_solves.find(ws);
  if (it == g_solves.end()) return false;
  *out = it->second;
  return true;
}

static std::atomic<long long> g_launches{0};
static bool g_timing = false;
static std::vector<cudaEvent_t> g_event_pool;
static std::vector<TimedLaunch> g_pending;
static long long g_cls_count[KC_COUNT];
static double g_cls_ms[KC_COUNT];
static double g_cls_bytes[KC_COUNT];

void count_launch(int n) { g_launches += n; }
bool timing_on() { return g_timing; }

cudaEvent_t timing_event() {
  std::lock_guard<std::mutex> lk(g_mu);
  if (!g_event_pool.empty()) {
    cudaEvent_t e = g_event_pool.back();
    g_event_pool.pop_back();
    return e;
  }
  cudaEvent_t e;
  cudaEventCreate(&e);
  return e;
}

void timing_push(const TimedLaunch& t) {
  std::lock_guard<std::mutex> lk(g_mu);
  g_pending.push_back(t);
}

void timing_collect() {
  std::lock_guard<std::mutex> lk(g_mu);
  for (const TimedLaunch& t : g_pending) {
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, t.a, t.b) == cudaSuccess) {
      g_cls_count[t.cls] += 1;
      g_cls_ms[t.cls] += ms;
      g_cls_bytes[t.cls] += t.bytes;
    }
    g_event_pool.push_back(t.a);
    g_event_pool.push_back(t.b);
  }
  g_pending.clear();
}

void timing_add(int cls, double bytes, float ms) {
  std::lock_guard<std::mutex> lk(g_mu);
  g_cls_count[cls] += 1;
  g_cls_ms[cls] += ms;
  g_cls_bytes[cls] += bytes;
}

}  // namespace polar

extern "C" long long polar_launch_count(void) { return polar::g_launches.load(); }

extern "C" void polar_set_kernel_timing(int on) {
  std::lock_guard<std::mutex> lk(polar::g_mu);
  polar::g_timing = on != 0;
  for (int i = 0; i < polar::KC_COUNT; ++i) {
    polar::g_cls_count[i] = 0;
    polar::g_cls_ms[i] = 0.0;
    polar::g_cls_bytes[i] = 0.0;
  }
}

extern "C" int polar_kernel_timing(int cls, long long* launches, double* ms, double* bytes) {
  if (cls < 0 || cls >= polar::KC_COUNT) return POLAR_ERR_BAD_ARG;
  std::lock_guard<std::mutex> lk(polar::g_mu);
  if (launches) *launches = polar::g_cls_count[cls];
  if (ms) *ms = polar::g_cls_ms[cls];
  if (bytes) *bytes = polar::g_cls_bytes[cls];
  return POLAR_OK;
}

extern "C" const char* polar_last_error(void) { return polar::g_err.c_str(); }
extern "C" int polar_version(void) { return 1; }
