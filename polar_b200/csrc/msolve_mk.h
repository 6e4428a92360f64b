// Multi-kernel (CUDA graph) multi-shift CG driver.
#pragma once
#include <cuda_runtime.h>

#include "solver_core.cuh"

namespace polar {

struct MkResult {
  int err;
  int capped;
  long long iterations;
  long long flushes;
  int grid;
};

// Runs a whole solve (blocking: returns after the stream is synchronised).
template <typename T, int VEC, bool W, int E>
int mk_solve(const SolvePrm<T>& host_prm, SolvePrm<T>* dev_prm, cudaStream_t st, MkResult* out);

// Largest grid any of the solver's partial-sum kernels uses (sizes the partial buffer).
template <typename T, int VEC, bool W, int E>
int mk_grid_max();

}  // namespace polar
