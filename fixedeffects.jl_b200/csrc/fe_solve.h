// fe_solve.h -- internal entry of the solve drivers (fe_solve.cu).
#pragma once

#include <stdint.h>

#include "fe_plan.h"

namespace fe {

struct SolveReq {
  void* Y = nullptr;       // device, column-major N x ncols, leading dimension ld
  int32_t dtype = 0;       // 0: float64, 1: float32
  int64_t ncols = 0;
  int64_t ld = 0;
  int32_t precision = 0;   // 0 FP64, 1 MIXED, 2 FP32
  double tol = 1e-8;
  int64_t maxiter = 10000;
  bool residuals = true;   // false: solve_coefficients!
  int64_t* iters = nullptr;          // per column
  uint8_t* converged = nullptr;      // per column
  int64_t* prob_iters = nullptr;     // optional [nprob][ncols]
  uint8_t* prob_converged = nullptr; // optional [nprob][ncols]
  double* const* coefs = nullptr;    // host, per FE (coefficients mode)
  // optional per-tile hooks on the host (transfers of host buffers overlapped
  // with the solve): before_tile runs before a tile's first launch is
  // enqueued, after_tile after its last; a non-zero return aborts the solve
  int (*before_tile)(void* ctx, int64_t col0, int ncols) = nullptr;
  int (*after_tile)(void* ctx, int64_t col0, int ncols) = nullptr;
  void* hook_ctx = nullptr;
};

// column-tile width of the next tile when `remaining` columns are left
int tile_width(const fe_plan* pl, int64_t remaining);
int solve(fe_plan* pl, const SolveReq& rq);
int prof_flush(fe_plan* pl);

}  // namespace fe
