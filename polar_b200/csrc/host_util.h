// Host-side helpers shared by the libpolar translation units.
#pragma once
#include <cuda_runtime.h>

#include "polar.h"

namespace polar {

// polar_spmm's argument checks (everything but the scratch pointer) and the offset of its
// heavy-row arrival counters inside the scratch; shared with polar_spmm_noalloc.
int spmm_check_args(const polar_graph* g, int precision, int R, const void* d_X, int ldx, const void* d_Y, int ldy);
size_t spmm_counter_offset(const polar_graph* g, int precision);
// The L2 policy set by polar_set_l2_policy (also applied by the standalone apply) and the
// solver's SpMM lanes per row for a padded width.
int l2_mode_setting();
size_t l2_hot_bytes_setting();
int mk_spmm_lanes(int precision, int ld);

int set_error(int code, const char* msg);
int set_cuda_error(const char* what, cudaError_t e);
void clear_error();

struct SolveRecord {
  int* ctl;
  long long* stats;
  int ld, grid, block;
  bool done;  // solve already completed on the host side (kernel-per-phase driver)
  int status;
  long long iterations, flushes;
};
void remember_solve(void* ws, int* ctl, long long* stats, int ld, int grid, int block);
void remember_solve_done(void* ws, int status, long long iterations, long long flushes, int ld, int grid, int block);
bool lookup_solve(void* ws, SolveRecord* out);

// Kernel instrumentation: every launch of a libpolar kernel is counted; with timing on,
// the solver's kernels are bracketed by CUDA events and their device time and
// algorithmic bytes are accumulated per class.
enum KernelClass { KC_SPMM = 0, KC_RESID, KC_DIR, KC_FLUSH, KC_INIT, KC_OTHER, KC_HEAVY, KC_COUNT };
void count_launch(int n = 1);
bool timing_on();
struct TimedLaunch {
  int cls;
  double bytes;
  cudaEvent_t a, b;
};
cudaEvent_t timing_event();
void timing_push(const TimedLaunch& t);
void timing_collect();  // after a stream sync: fold finished pairs into the totals
void timing_add(int cls, double bytes, float ms);

}  // namespace polar
