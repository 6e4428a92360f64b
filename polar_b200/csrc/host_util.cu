// Error text and per-workspace solve records for the C ABI.
#include <cstdio>
#include <mutex>
#include <string>
#include <unordered_map>

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

}  // namespace polar

extern "C" const char* polar_last_error(void) { return polar::g_err.c_str(); }
extern "C" int polar_version(void) { return 1; }
