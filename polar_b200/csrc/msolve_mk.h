// Multi-kernel (CUDA graph) multi-shift CG driver.
#pragma once
#include <cuda_runtime.h>

#include <vector>

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

// Runs many independent solves concurrently, each on its own stream ordered after `st`,
// with every grid scaled by frac[b]; `st` waits for all of them on return.
template <typename T, int VEC, bool W, int E>
int mk_solve_batch(const std::vector<SolvePrm<T>>& prms, const std::vector<double>& frac, cudaStream_t st,
                   std::vector<MkResult>& out);

// Largest grid any of the solver's partial-sum kernels uses (sizes the partial buffer).
template <typename T, int VEC, bool W, int E>
int mk_grid_max();

}  // namespace polar
