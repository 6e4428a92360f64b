// Host-side helpers shared by the libpolar translation units.
#pragma once
#include <cuda_runtime.h>

namespace polar {

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

}  // namespace polar
