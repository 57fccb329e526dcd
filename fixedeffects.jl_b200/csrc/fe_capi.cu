// fe_capi.cu -- extern "C" entry points of include/fe_b200.h.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "../../include/fe_b200.h"
#include "fe_plan.h"
#include "fe_solve.h"
#include "fe_staging.h"

using fe::set_error;

namespace {

int check_plan(fe_plan* p) {
  if (!p) {
    set_error("plan is NULL");
    return FE_ERR_INVALID;
  }
  return FE_OK;
}

int create_common(fe_plan** out, int32_t nprob, const int64_t* n_obs, int32_t K,
                  const int64_t* const* refs, const int64_t* n_levels,
                  const double* const* interaction, const double* weights, int32_t device,
                  fe_exchange_fn xchg = nullptr, void* xchg_ctx = nullptr) {
  if (!out) {
    set_error("out is NULL");
    return FE_ERR_INVALID;
  }
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    (void)cudaGetLastError();
    set_error("no CUDA device available");
    return FE_ERR_CUDA;
  }
  if (device < 0 || device >= ndev) {
    set_error("device ordinal out of range");
    return FE_ERR_INVALID;
  }
  fe_plan* pl = new (std::nothrow) fe_plan();
  if (!pl) {
    set_error("host allocation failed");
    return FE_ERR_ALLOC;
  }
  pl->xchg = xchg;
  pl->xchg_ctx = xchg_ctx;
  int st = fe::plan_build(pl, nprob, n_obs, K, refs, n_levels, interaction, weights, device);
  if (st) {
    fe::plan_destroy(pl);
    return st;
  }
  *out = pl;
  return FE_OK;
}

// Host columns of a solve, moved through the device staging buffer (the
// columns side by side, leading dimension N).  Pinned columns: every tile's
// upload is queued at once on an upload stream with one event per tile, the
// tile's solve waits for its event, and its download runs on a download
// stream once the solve is done, so transfers in both directions overlap the
// solves of the other tiles.  Pageable columns go through the plan's pinned
// staging ring (fe_staging.cu), with the same overlap; small pageable solves
// are copied tile by tile on the plan's stream.
struct HostXfer {
  fe_plan* pl = nullptr;
  void* const* cols = nullptr;
  size_t bytes = 0;  // per column
  bool pinned = false;
  fe::PageableStager* stager = nullptr;  // pageable columns through the pinned ring
  cudaStream_t up = nullptr, down = nullptr;
  std::vector<cudaEvent_t> ev;  // per tile: upload done, then solve done
  std::vector<int64_t> tile0;   // first column of each tile
  size_t tile = 0;
  char* stage() const { return static_cast<char*>(pl->ws.ystage.p); }
  // waits for the staged downloads; the first staging error, or 0
  int end_staging() {
    fe::PageableStager* x = stager;
    stager = nullptr;
    return fe::stager_end(x);
  }
  ~HostXfer() {
    end_staging();
    if (up) cudaStreamSynchronize(up);
    if (down) cudaStreamSynchronize(down);
    for (cudaEvent_t e : ev) cudaEventDestroy(e);
    if (up) cudaStreamDestroy(up);
    if (down) cudaStreamDestroy(down);
  }
};

int xfer_error(const char* what, cudaError_t e) {
  (void)cudaGetLastError();
  set_error(std::string(what) + ": " + cudaGetErrorString(e));
  return FE_ERR_CUDA;
}

int xfer_before(void* ctx, int64_t col0, int nc) {
  HostXfer& x = *static_cast<HostXfer*>(ctx);
  if (x.stager) return fe::stager_before_tile(x.stager, x.tile);
  cudaError_t e = cudaSuccess;
  if (x.pinned) {
    e = cudaStreamWaitEvent(x.pl->stream, x.ev[2 * x.tile], 0);
  } else {
    for (int j = 0; j < nc && e == cudaSuccess; ++j)
      e = cudaMemcpyAsync(x.stage() + (size_t)(col0 + j) * x.bytes, x.cols[col0 + j], x.bytes,
                          cudaMemcpyHostToDevice, x.pl->stream);
  }
  return e == cudaSuccess ? 0 : xfer_error("host to device copy failed", e);
}

int xfer_after(void* ctx, int64_t col0, int nc) {
  HostXfer& x = *static_cast<HostXfer*>(ctx);
  if (x.stager) return fe::stager_after_tile(x.stager, x.tile++);
  cudaError_t e = cudaSuccess;
  cudaStream_t s = x.pl->stream;
  if (x.pinned) {
    e = cudaEventRecord(x.ev[2 * x.tile + 1], s);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(x.down, x.ev[2 * x.tile + 1], 0);
    s = x.down;
  }
  for (int j = 0; j < nc && e == cudaSuccess; ++j)
    e = cudaMemcpyAsync(x.cols[col0 + j], x.stage() + (size_t)(col0 + j) * x.bytes, x.bytes,
                        cudaMemcpyDeviceToHost, s);
  ++x.tile;
  return e == cudaSuccess ? 0 : xfer_error("device to host copy failed", e);
}

bool is_pinned(const void* p) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    (void)cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeHost;
}

// Y: device matrix (cols == nullptr, leading dimension ld) or host columns.
int solve_common(fe_plan* plan, void* Y, void* const* cols, int32_t dtype, int64_t ncols,
                 int64_t ld, int32_t precision, double tol, int64_t maxiter,
                 int64_t* iterations, uint8_t* converged) {
  int st = check_plan(plan);
  if (st) return st;
  if (dtype != FE_DTYPE_F64 && dtype != FE_DTYPE_F32) {
    set_error("dtype must be FE_DTYPE_F64 or FE_DTYPE_F32");
    return FE_ERR_INVALID;
  }
  if (precision < 0 || precision > 2) {
    set_error("precision must be FE_PREC_FP64, FE_PREC_MIXED or FE_PREC_FP32");
    return FE_ERR_INVALID;
  }
  const bool host = cols != nullptr;
  if (ncols < 0 || (ncols > 0 && !host && !Y && plan->N > 0)) {
    set_error("Y is NULL or ncols < 0");
    return FE_ERR_INVALID;
  }
  if (host && plan->N > 0)
    for (int64_t j = 0; j < ncols; ++j)
      if (!cols[j]) {
        set_error("column " + std::to_string(j) + " is NULL");
        return FE_ERR_INVALID;
      }
  if (ld < plan->N) {
    set_error("ld must be >= the number of observations");
    return FE_ERR_INVALID;
  }
  if (!(tol >= 0.0) || maxiter < 1) {
    set_error("tol must be >= 0 and maxiter >= 1");
    return FE_ERR_INVALID;
  }
  if (ncols == 0) return FE_OK;
  const size_t es = dtype == FE_DTYPE_F64 ? 8 : 4;
  fe::SolveReq rq;
  rq.dtype = dtype;
  rq.ncols = ncols;
  rq.precision = precision;
  rq.tol = tol;
  rq.maxiter = maxiter;
  rq.residuals = true;
  rq.iters = iterations;
  rq.converged = converged;
  plan->last_prob_iters.assign((size_t)plan->nprob * ncols, 0);
  plan->last_prob_conv.assign((size_t)plan->nprob * ncols, 0);
  rq.prob_iters = plan->last_prob_iters.data();
  rq.prob_converged = plan->last_prob_conv.data();
  if (cudaSetDevice(plan->device) != cudaSuccess) {
    set_error("cudaSetDevice failed");
    return FE_ERR_CUDA;
  }
  const int64_t N = plan->N;
  HostXfer x;
  if (host && N > 0) {
    st = plan->ws.ystage.ensure((size_t)N * ncols * es);
    if (st) return st;
    x.pl = plan;
    x.cols = cols;
    x.bytes = (size_t)N * es;
    x.pinned = true;
    for (int64_t j = 0; j < ncols && x.pinned; ++j) x.pinned = is_pinned(cols[j]);
    for (int64_t c0 = 0; c0 < ncols; c0 += std::min<int64_t>(fe::tile_width(plan, ncols - c0),
                                                              ncols - c0))
      x.tile0.push_back(c0);
    x.tile0.push_back(ncols);
    if (!x.pinned && (size_t)N * (size_t)ncols * es >= fe::kStageMinBytes) {
      st = fe::stager_begin(plan, cols, x.bytes, x.tile0, x.stage(), &x.stager);
      if (st) return st;
    } else if (x.pinned) {
      cudaError_t e = cudaStreamCreateWithFlags(&x.up, cudaStreamNonBlocking);
      if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&x.down, cudaStreamNonBlocking);
      // the uploads must not overtake work already queued on the plan's
      // stream that reads the staging buffer
      cudaEvent_t start = nullptr;
      if (e == cudaSuccess) e = cudaEventCreateWithFlags(&start, cudaEventDisableTiming);
      if (e == cudaSuccess) e = cudaEventRecord(start, plan->stream);
      if (e == cudaSuccess) e = cudaStreamWaitEvent(x.up, start, 0);
      if (start) cudaEventDestroy(start);
      for (size_t t = 0; t + 1 < x.tile0.size() && e == cudaSuccess; ++t) {
        cudaEvent_t a = nullptr, b = nullptr;
        e = cudaEventCreateWithFlags(&a, cudaEventDisableTiming);
        if (e == cudaSuccess) x.ev.push_back(a);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b, cudaEventDisableTiming);
        if (e == cudaSuccess) x.ev.push_back(b);
        for (int64_t j = x.tile0[t]; j < x.tile0[t + 1] && e == cudaSuccess; ++j)
          e = cudaMemcpyAsync(x.stage() + (size_t)j * x.bytes, cols[j], x.bytes,
                              cudaMemcpyHostToDevice, x.up);
        if (e == cudaSuccess) e = cudaEventRecord(a, x.up);
      }
      if (e != cudaSuccess) return xfer_error("host to device copy failed", e);
    }
    rq.Y = plan->ws.ystage.p;
    rq.ld = N;
    rq.before_tile = xfer_before;
    rq.after_tile = xfer_after;
    rq.hook_ctx = &x;
  } else {
    rq.Y = Y;
    rq.ld = ld;
  }
  st = fe::solve(plan, rq);
  if (st) return st;
  if ((st = x.end_staging())) return st;
  cudaError_t e = cudaStreamSynchronize(plan->stream);
  if (e == cudaSuccess && x.down) e = cudaStreamSynchronize(x.down);
  if (e != cudaSuccess) {
    set_error(std::string("stream synchronize failed: ") + cudaGetErrorString(e));
    return FE_ERR_CUDA;
  }
  return FE_OK;
}

}  // namespace

extern "C" {

int fe_version(void) { return FE_B200_VERSION; }

const char* fe_last_error(void) { return fe::last_error(); }

int fe_plan_create(fe_plan** out, int64_t n_obs, int32_t n_fe, const int64_t* const* refs,
                   const int64_t* n_levels, const double* const* interaction,
                   const double* weights, int32_t device) {
  fe::DeviceRestore restore_device;
  if (n_obs < 0) {
    set_error("n_obs must be >= 0");
    return FE_ERR_INVALID;
  }
  return create_common(out, 1, &n_obs, n_fe, refs, n_levels, interaction, weights, device);
}

int fe_plan_create_sharded(fe_plan** out, int64_t n_obs, int32_t n_fe, const int64_t* const* refs,
                           const int64_t* n_levels, const double* const* interaction,
                           const double* weights, int32_t device, fe_exchange_fn exchange,
                           void* ctx) {
  fe::DeviceRestore restore_device;
  if (!exchange) {
    set_error("a sharded plan needs an exchange function");
    return FE_ERR_INVALID;
  }
  if (n_obs < 1) {
    // every rank takes part in every exchange, so none may be empty
    set_error("a sharded plan needs at least one observation on every rank");
    return FE_ERR_INVALID;
  }
  return create_common(out, 1, &n_obs, n_fe, refs, n_levels, interaction, weights, device,
                       exchange, ctx);
}

int fe_plan_create_batch(fe_plan** out, int32_t n_problems, const int64_t* n_obs, int32_t n_fe,
                         const int64_t* const* refs, const int64_t* n_levels,
                         const double* const* interaction, const double* weights,
                         int32_t device) {
  fe::DeviceRestore restore_device;
  return create_common(out, n_problems, n_obs, n_fe, refs, n_levels, interaction, weights, device);
}

int fe_plan_update_weights(fe_plan* plan, const double* weights) {
  fe::DeviceRestore restore_device;
  int st = check_plan(plan);
  if (st) return st;
  return fe::plan_update_weights(plan, weights);
}

int fe_plan_set_stream(fe_plan* plan, void* stream) {
  fe::DeviceRestore restore_device;
  int st = check_plan(plan);
  if (st) return st;
  if (cudaStreamSynchronize(plan->stream) != cudaSuccess) {
    set_error("stream synchronize failed");
    return FE_ERR_CUDA;
  }
  if (stream) {
    if (plan->own_stream) cudaStreamDestroy(plan->stream);
    plan->own_stream = false;
    plan->stream = static_cast<cudaStream_t>(stream);
  } else if (!plan->own_stream) {
    cudaSetDevice(plan->device);
    if (cudaStreamCreateWithFlags(&plan->stream, cudaStreamNonBlocking) != cudaSuccess) {
      set_error("stream creation failed");
      return FE_ERR_CUDA;
    }
    plan->own_stream = true;
  }
  return FE_OK;
}

int fe_plan_set_option(fe_plan* plan, int32_t option, double value) {
  fe::DeviceRestore restore_device;
  int st = check_plan(plan);
  if (st) return st;
  switch (option) {
    case FE_OPT_TILE: {
      const int v = (int)value;
      if (v != 0 && v != 1 && v != 2 && v != 4 && v != 8 && v != 16 && v != 32) {
        set_error("tile must be 0 or a power of two <= 32");
        return FE_ERR_INVALID;
      }
      plan->opt_tile = v;
      return FE_OK;
    }
    case FE_OPT_CHECK_EVERY:
      if (value < 1) {
        set_error("check interval must be >= 1");
        return FE_ERR_INVALID;
      }
      plan->opt_check_every = (int)value;
      return FE_OK;
    case FE_OPT_MAX_ROUNDS:
      if (value < 1) {
        set_error("max rounds must be >= 1");
        return FE_ERR_INVALID;
      }
      plan->opt_max_rounds = (int)value;
      return FE_OK;
    case FE_OPT_PROFILE:
      plan->prof.on = value != 0;
      return FE_OK;
    case FE_OPT_INNER_RHO:
      if (!(value > 0 && value < 1)) {
        set_error("inner rho must be in (0, 1)");
        return FE_ERR_INVALID;
      }
      plan->opt_inner_rho = value;
      return FE_OK;
    case FE_OPT_FUSE:
      plan->opt_fuse = value != 0 ? 1 : 0;
      return FE_OK;
    case FE_OPT_AUTOTUNE:
      plan->opt_autotune = value != 0 ? 1 : 0;
      return FE_OK;
    case FE_OPT_MIXED_WARM_START:
      plan->opt_mixed_warm = value != 0 ? 1 : 0;
      return FE_OK;
    case FE_OPT_GRAPH:
      plan->opt_graph = value != 0 ? 1 : 0;
      return FE_OK;
    case FE_OPT_ABSORB:
      plan->opt_absorb = value != 0 ? 1 : 0;
      return FE_OK;
    case FE_OPT_FUSED_DEMEAN:
      plan->opt_exdm = value != 0 ? 1 : 0;
      return FE_OK;
    case FE_OPT_FUSED_RESID: {
      const int v = (int)value;
      if (v < -1 || v > 2) {
        set_error("fused residual option must be -1 (default), 0, 1 or 2");
        return FE_ERR_INVALID;
      }
      plan->opt_fused_resid = v;
      return FE_OK;
    }
    case FE_OPT_ABSORB_SCALE:
      plan->opt_abs_scale = value != 0 ? 1 : 0;
      return FE_OK;
    case FE_OPT_FIRM_ATOMIC: {
      const int v = (int)value;
      if (v < -1 || v > 1) {
        set_error("gathered-FE reduction option must be -1 (tuned), 0 or 1");
        return FE_ERR_INVALID;
      }
      plan->opt_firm_atomic = v;
      return FE_OK;
    }
    case FE_OPT_EXDM_PIPE: {
      const int v = (int)value;
      if (v < -1 || v > 3) {
        set_error("pipelined absorbed kernel option must be -1 (default), 0 (off), 1, 2 or 3");
        return FE_ERR_INVALID;
      }
      plan->opt_exdm_pipe = v;
      return FE_OK;
    }
    case FE_OPT_ROWSUM_VARIANT: {
      const int v = (int)value;
      if (v < -1 || v > 1) {
        set_error("row-sum variant must be -1 (default), 0 or 1");
        return FE_ERR_INVALID;
      }
      plan->opt_rowsum_variant = v;
      return FE_OK;
    }
    case FE_OPT_EXPAND_VARIANT:
    case FE_OPT_SEGSUM_VARIANT: {
      const int v = (int)value;
      const int vmax = 5;
      if (v < -1 || v > vmax) {
        set_error("kernel variant must be -1 (default) or 0..5");
        return FE_ERR_INVALID;
      }
      (option == FE_OPT_EXPAND_VARIANT ? plan->opt_ex_variant : plan->opt_seg_variant) = v;
      return FE_OK;
    }
    default:
      set_error("unknown option");
      return FE_ERR_INVALID;
  }
}

int fe_plan_destroy(fe_plan* plan) {
  fe::DeviceRestore restore_device;
  if (!plan) return FE_OK;
  return fe::plan_destroy(plan);
}

int fe_solve_residuals(fe_plan* plan, void* Y, int32_t dtype, int64_t ncols, int64_t ld,
                       int32_t precision, double tol, int64_t maxiter, int64_t* iterations,
                       uint8_t* converged) {
  fe::DeviceRestore restore_device;
  int st = check_plan(plan);
  if (st) return st;
  if (ncols < 0 || (ncols > 0 && !Y && plan->N > 0)) {
    set_error("Y is NULL or ncols < 0");
    return FE_ERR_INVALID;
  }
  const size_t es = dtype == FE_DTYPE_F64 ? 8 : 4;
  std::vector<void*> cols((size_t)ncols);
  for (int64_t j = 0; j < ncols; ++j)
    cols[(size_t)j] = Y ? static_cast<char*>(Y) + (size_t)j * (size_t)ld * es : nullptr;
  return solve_common(plan, nullptr, cols.data(), dtype, ncols, ld, precision, tol, maxiter,
                      iterations, converged);
}

int fe_solve_residuals_columns(fe_plan* plan, void* const* columns, int32_t dtype, int64_t ncols,
                               int32_t precision, double tol, int64_t maxiter,
                               int64_t* iterations, uint8_t* converged) {
  fe::DeviceRestore restore_device;
  int st = check_plan(plan);
  if (st) return st;
  if (ncols < 0 || (ncols > 0 && !columns)) {
    set_error("columns is NULL or ncols < 0");
    return FE_ERR_INVALID;
  }
  return solve_common(plan, nullptr, columns, dtype, ncols, plan->N, precision, tol, maxiter,
                      iterations, converged);
}

int fe_solve_residuals_device(fe_plan* plan, void* Y_dev, int32_t dtype, int64_t ncols,
                              int64_t ld, int32_t precision, double tol, int64_t maxiter,
                              int64_t* iterations, uint8_t* converged) {
  fe::DeviceRestore restore_device;
  return solve_common(plan, Y_dev, nullptr, dtype, ncols, ld, precision, tol, maxiter, iterations,
                      converged);
}

int fe_solve_coefficients(fe_plan* plan, const void* y, int32_t dtype, int32_t precision,
                          double tol, int64_t maxiter, double* const* coefs,
                          int64_t* iterations, uint8_t* converged) {
  fe::DeviceRestore restore_device;
  int st = check_plan(plan);
  if (st) return st;
  if (dtype != FE_DTYPE_F64 && dtype != FE_DTYPE_F32) {
    set_error("dtype must be FE_DTYPE_F64 or FE_DTYPE_F32");
    return FE_ERR_INVALID;
  }
  if (precision < 0 || precision > 2) {
    set_error("precision must be FE_PREC_FP64, FE_PREC_MIXED or FE_PREC_FP32");
    return FE_ERR_INVALID;
  }
  if ((!y && plan->N > 0) || !coefs) {
    set_error("y and coefs are required");
    return FE_ERR_INVALID;
  }
  for (int k = 0; k < plan->K; ++k)
    if (!coefs[k] && plan->nlev[k] > 0) {
      set_error("coefs[k] is NULL");
      return FE_ERR_INVALID;
    }
  if (!(tol >= 0.0) || maxiter < 1) {
    set_error("tol must be >= 0 and maxiter >= 1");
    return FE_ERR_INVALID;
  }
  if (cudaSetDevice(plan->device) != cudaSuccess) {
    set_error("cudaSetDevice failed");
    return FE_ERR_CUDA;
  }
  const int64_t N = plan->N;
  const size_t es = dtype == FE_DTYPE_F64 ? 8 : 4;
  fe::SolveReq rq;
  rq.dtype = dtype;
  rq.ncols = 1;
  rq.ld = N;
  rq.precision = precision;
  rq.tol = tol;
  rq.maxiter = maxiter;
  rq.residuals = false;
  rq.iters = iterations;
  rq.converged = converged;
  rq.coefs = coefs;
  plan->last_prob_iters.assign((size_t)plan->nprob, 0);
  plan->last_prob_conv.assign((size_t)plan->nprob, 0);
  rq.prob_iters = plan->last_prob_iters.data();
  rq.prob_converged = plan->last_prob_conv.data();
  if (N > 0) {
    st = plan->ws.ystage.ensure((size_t)N * es);
    if (st) return st;
    cudaError_t e = cudaMemcpyAsync(plan->ws.ystage.p, y, (size_t)N * es, cudaMemcpyHostToDevice,
                                    plan->stream);
    if (e != cudaSuccess) {
      set_error(std::string("host to device copy failed: ") + cudaGetErrorString(e));
      return FE_ERR_CUDA;
    }
    rq.Y = plan->ws.ystage.p;
  }
  // solve_coefficients! always runs LSMR, even with one fixed effect
  const int save_tile = plan->opt_tile;
  plan->opt_tile = 1;
  st = fe::solve(plan, rq);
  plan->opt_tile = save_tile;
  return st;
}

int fe_plan_problem_results(fe_plan* plan, int64_t* iterations, uint8_t* converged) {
  fe::DeviceRestore restore_device;
  int st = check_plan(plan);
  if (st) return st;
  if (iterations)
    std::copy(plan->last_prob_iters.begin(), plan->last_prob_iters.end(), iterations);
  if (converged) std::copy(plan->last_prob_conv.begin(), plan->last_prob_conv.end(), converged);
  return FE_OK;
}

int fe_plan_last_solve_info(fe_plan* plan, int64_t ncols, double* test2, int32_t* rounds,
                            int64_t* lsmr_iters) {
  fe::DeviceRestore restore_device;
  int st = check_plan(plan);
  if (st) return st;
  const int64_t n = std::min<int64_t>(ncols, (int64_t)plan->last_test2.size());
  for (int64_t j = 0; j < n; ++j) {
    if (test2) test2[j] = plan->last_test2[(size_t)j];
    if (rounds) rounds[j] = plan->last_rounds[(size_t)j];
    if (lsmr_iters) lsmr_iters[j] = plan->last_iters_raw[(size_t)j];
  }
  return FE_OK;
}

int fe_plan_get_integer_plan(fe_plan* plan, int32_t* perm0, int64_t* const* offsets,
                             int32_t* const* segperm) {
  fe::DeviceRestore restore_device;
  int st = check_plan(plan);
  if (st) return st;
  cudaSetDevice(plan->device);
  const int64_t N = plan->N;
  if (perm0 && N > 0) {
    if (cudaMemcpy(perm0, plan->d_obs_src.p, (size_t)N * 4, cudaMemcpyDeviceToHost) != cudaSuccess) {
      set_error("copy of the integer plan failed");
      return FE_ERR_CUDA;
    }
  }
  for (int k = 0; k < plan->K; ++k) {
    if (offsets && offsets[k])
      std::copy(plan->seg_off[k].begin(), plan->seg_off[k].begin() + plan->nlev[k] + 1, offsets[k]);
    if (segperm && segperm[k] && plan->seg_len[k] > 0) {
      if (plan->perm_identity[k]) {
        for (int64_t q = 0; q < plan->seg_len[k]; ++q) segperm[k][q] = (int32_t)q;
      } else if (cudaMemcpy(segperm[k], plan->d_perm[k].p, (size_t)plan->seg_len[k] * 4,
                            cudaMemcpyDeviceToHost) != cudaSuccess) {
        set_error("copy of the integer plan failed");
        return FE_ERR_CUDA;
      }
    }
  }
  return FE_OK;
}

int fe_plan_get_scales(fe_plan* plan, double* const* scales) {
  fe::DeviceRestore restore_device;
  int st = check_plan(plan);
  if (st) return st;
  if (!scales) {
    set_error("scales is NULL");
    return FE_ERR_INVALID;
  }
  cudaSetDevice(plan->device);
  cudaStreamSynchronize(plan->stream);
  for (int k = 0; k < plan->K; ++k)
    if (scales[k] && plan->nlev[k] > 0 &&
        cudaMemcpy(scales[k], plan->d_scale_d[k].p, (size_t)plan->nlev[k] * 8,
                   cudaMemcpyDeviceToHost) != cudaSuccess) {
      set_error("copy of the scales failed");
      return FE_ERR_CUDA;
    }
  return FE_OK;
}

int fe_plan_primary(fe_plan* plan, int32_t* primary) {
  fe::DeviceRestore restore_device;
  int st = check_plan(plan);
  if (st) return st;
  if (primary) *primary = plan->primary;
  return FE_OK;
}

int fe_plan_kernel_stat(fe_plan* plan, int32_t index, char* name, int64_t name_len,
                        int64_t* launches, double* total_ms, double* alg_bytes) {
  fe::DeviceRestore restore_device;
  int st = check_plan(plan);
  if (st) return st;
  fe::prof_flush(plan);
  if (index < 0 || index >= (int32_t)plan->prof.stats.size()) {
    set_error("kernel stat index out of range");
    return FE_ERR_INVALID;
  }
  auto it = plan->prof.stats.begin();
  std::advance(it, index);
  const fe::KernelStat& s = it->second;
  if (name && name_len > 0) {
    std::strncpy(name, s.name.c_str(), (size_t)name_len - 1);
    name[name_len - 1] = '\0';
  }
  if (launches) *launches = s.launches;
  if (total_ms) *total_ms = s.ms;
  if (alg_bytes) *alg_bytes = s.bytes;
  return FE_OK;
}

int fe_plan_kernel_times(fe_plan* plan, int32_t index, float* ms, int64_t max_launches,
                         int64_t* launches) {
  fe::DeviceRestore restore_device;
  int st = check_plan(plan);
  if (st) return st;
  fe::prof_flush(plan);
  if (index < 0 || index >= (int32_t)plan->prof.stats.size()) {
    set_error("kernel stat index out of range");
    return FE_ERR_INVALID;
  }
  auto it = plan->prof.stats.begin();
  std::advance(it, index);
  const std::vector<float>& t = it->second.times;
  if (launches) *launches = (int64_t)t.size();
  if (ms && max_launches > 0)
    std::copy(t.begin(), t.begin() + std::min<int64_t>(max_launches, (int64_t)t.size()), ms);
  return FE_OK;
}

int fe_plan_reset_stats(fe_plan* plan) {
  fe::DeviceRestore restore_device;
  int st = check_plan(plan);
  if (st) return st;
  fe::prof_flush(plan);
  plan->prof.stats.clear();
  return FE_OK;
}

}  // extern "C"
