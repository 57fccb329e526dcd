// fe_scalar.cu -- the LSMR scalar recurrences, one CTA per instance, in FP64.
//
// Restates src/utils/lsmr.jl:46-222 (lambda = 0).  Built with -fmad=false so
// every multiply and add rounds separately, as in the reference's scalar code.
//
// The vector updates of iteration k (lsmr.jl:138-142) run one iteration late,
// fused into the next reduce kernel; the stopping test of iteration k
// therefore runs once ||x_k|| is known, in the ALPHA phase of iteration k+1.
// x is then exactly x_k, as in the reference.
#include <cuda_runtime.h>

#include "fe_internal.h"

namespace fe {

// Kernel coefficients of a stopped instance: the expand keeps U
// (U <- 0*(A v) + 1*U) and the P-side update is skipped (upd_mode 0, no v).
__device__ static void deactivate(Inst& s) {
  s.active = 0;
  s.ex_av = 0.0;
  s.ex_au = 1.0;
  s.upd_mode = 0;
  s.do_v = 0;
}

__device__ static void lsmr_test(Inst& s) {
  // src/utils/lsmr.jl:188-215
  const double test1 = s.normr / s.normb;
  const double test2 = s.normAr / (s.normA * s.normr);
  const double test3 = 1.0 / s.condA;
  const double t1 = test1 / (1.0 + s.normA * s.normx / s.normb);
  const double rtol = s.btol + s.atol * s.normA * s.normx / s.normb;
  int istop = 0;
  if (s.iter >= s.maxiter) istop = 7;
  else if (1.0 + test3 <= 1.0) istop = 6;
  else if (1.0 + test2 <= 1.0) istop = 5;
  else if (1.0 + t1 <= 1.0) istop = 4;
  else if (test3 <= s.ctol) istop = 3;
  else if (test2 <= s.atol) istop = 2;
  else if (test1 <= rtol) istop = 1;
  if (!istop && s.mode_inner) {
    // inner solve of the mixed mode: stop once the FP64 outer test is
    // expected to pass, or once normAr fell by inner_rho (the FP32 floor)
    const double nAt = sqrt(s.normA2_prev + s.normA * s.normA);
    if (s.normAr <= s.inner_theta_tol * nAt * s.normr || s.normAr <= s.inner_rho * s.normAr0)
      istop = 2;
  }
  s.istop = istop;
}

__device__ static void lsmr_rotate(Inst& s) {
  // src/utils/lsmr.jl:113-186, lambda = 0
  const double lambda = 0.0;
  const double alphahat = sqrt(s.alphabar * s.alphabar + lambda * lambda);
  const double chat = s.alphabar / alphahat;
  const double shat = lambda / alphahat;
  const double rhoold = s.rho;
  s.rho = sqrt(alphahat * alphahat + s.beta * s.beta);
  const double c = alphahat / s.rho;
  const double sn = s.beta / s.rho;
  const double thetanew = sn * s.alpha;
  s.alphabar = c * s.alpha;
  const double rhobarold = s.rhobar;
  const double zetaold = s.zeta;
  const double thetabar = s.sbar * s.rho;
  const double rhotemp = s.cbar * s.rho;
  s.rhobar = sqrt((s.cbar * s.rho) * (s.cbar * s.rho) + thetanew * thetanew);
  s.cbar = s.cbar * s.rho / s.rhobar;
  s.sbar = thetanew / s.rhobar;
  s.zeta = s.cbar * s.zetabar;
  s.zetabar = -s.sbar * s.zetabar;
  // coefficients of the (deferred) vector update, lsmr.jl:138-142
  s.c1 = -thetabar * s.rho / (rhoold * rhobarold);
  s.c2 = s.zeta / (s.rho * s.rhobar);
  s.c3 = -thetanew / s.rho;
  // estimate of ||r||
  const double betaacute = chat * s.betadd;
  const double betacheck = -shat * s.betadd;
  const double betahat = c * betaacute;
  s.betadd = -sn * betaacute;
  const double thetatildeold = s.thetatilde;
  const double rhotildeold = sqrt(s.rhodold * s.rhodold + thetabar * thetabar);
  const double ctildeold = s.rhodold / rhotildeold;
  const double stildeold = thetabar / rhotildeold;
  s.thetatilde = stildeold * s.rhobar;
  s.rhodold = ctildeold * s.rhobar;
  s.betad = -stildeold * s.betad + ctildeold * betahat;
  s.tautildeold = (zetaold - thetatildeold * s.tautildeold) / rhotildeold;
  const double taud = (s.zeta - s.thetatilde * s.tautildeold) / s.rhodold;
  s.d = s.d + betacheck * betacheck;
  s.normr = sqrt(s.d + (s.betad - taud) * (s.betad - taud) + s.betadd * s.betadd);
  // estimate of ||A|| and cond(A)
  s.normA2 = s.normA2 + s.beta * s.beta;
  s.normA = sqrt(s.normA2);
  s.normA2 = s.normA2 + s.alpha * s.alpha;
  s.maxrbar = s.maxrbar > rhobarold ? s.maxrbar : rhobarold;
  if (s.iter > 1) s.minrbar = s.minrbar < rhobarold ? s.minrbar : rhobarold;
  const double mx = s.maxrbar > rhotemp ? s.maxrbar : rhotemp;
  const double mn = s.minrbar < rhotemp ? s.minrbar : rhotemp;
  s.condA = mx / mn;
  s.normAr = fabs(s.zetabar);
}

// Initial values of src/utils/lsmr.jl:68-100 given alpha, beta.
__device__ static void lsmr_init(Inst& s, int init_mode) {
  s.zetabar = s.alpha * s.beta;
  s.alphabar = s.alpha;
  s.rho = 1.0;
  s.rhobar = 1.0;
  s.cbar = 1.0;
  s.sbar = 0.0;
  s.betadd = s.beta;
  s.betad = 0.0;
  s.rhodold = 1.0;
  s.tautildeold = 0.0;
  s.thetatilde = 0.0;
  s.zeta = 0.0;
  s.d = 0.0;
  s.normA = -1.0;
  s.condA = -1.0;
  s.normx = -1.0;
  s.normA2 = s.alpha * s.alpha;
  s.maxrbar = 0.0;
  s.minrbar = 1e100;
  s.normb = s.beta;
  s.istop = 0;
  s.normr = s.beta;
  s.normAr = s.alpha * s.beta;
  s.iter = 0;
  s.pending = 0;
  s.upd_mode = init_mode;  // h <- v, hbar <- 0 (and x <- 0) at the next reduce
  s.do_v = 1;
  s.active = (s.normAr != 0.0 && s.maxiter > 0 && !s.skip_lsmr) ? 1 : 0;
  // a NaN or infinite right-hand side: the reference runs maxiter iterations
  // on NaN norms (no test can pass) and reports istop = 7, not converged;
  // here the instance stops at once with the same verdict
  if (!isfinite(s.normAr)) {
    s.active = 0;
    s.istop = 7;
  }
  s.ex_av = s.s_v;
  s.ex_au = -s.alpha * s.u_scale;
  if (!s.active) deactivate(s);
}

__global__ void __launch_bounds__(kScalarThreads) k_scalar(ScalarArgs a) {
  __shared__ double red[3][kScalarThreads];
  const int id = blockIdx.x;
  const int prob = id / a.C, j = id - prob * a.C;
  double s0 = 0.0, s1 = 0.0, s2 = 0.0;
  if (a.part0) {
    const int64_t lo = a.off0[prob], hi = a.off0[prob + 1];
    const double* p = a.part0 + (int64_t)j * a.S0;
    for (int64_t q = lo + threadIdx.x; q < hi; q += kScalarThreads) s0 += p[q];
  }
  if (a.part1 || a.part2) {
    const int64_t lo = a.off1[prob], hi = a.off1[prob + 1];
    const double* p1 = a.part1 ? a.part1 + (int64_t)j * a.S1 : nullptr;
    const double* p2 = a.part2 ? a.part2 + (int64_t)j * a.S1 : nullptr;
    for (int64_t q = lo + threadIdx.x; q < hi; q += kScalarThreads) {
      if (p1) s1 += p1[q];
      if (p2) s2 += p2[q];
    }
  }
  red[0][threadIdx.x] = s0;
  red[1][threadIdx.x] = s1;
  red[2][threadIdx.x] = s2;
  __syncthreads();
  for (int h = kScalarThreads / 2; h > 0; h >>= 1) {
    if ((int)threadIdx.x < h) {
      red[0][threadIdx.x] += red[0][threadIdx.x + h];
      red[1][threadIdx.x] += red[1][threadIdx.x + h];
      red[2][threadIdx.x] += red[2][threadIdx.x + h];
    }
    __syncthreads();
  }
  if (threadIdx.x != 0) return;
  s0 = red[0][0];
  s1 = red[1][0];
  s2 = red[2][0];
  Inst& s = a.inst[id];
  switch (a.phase) {
    case PH_INIT_BETA: {
      // u = b - A x; beta = ||u||; u /= beta  (lsmr.jl:63-65)
      s.beta = sqrt(s0);
      s.u_scale = s.beta > 0 ? 1.0 / s.beta : 1.0;
      s.rd_acc = s.u_scale;
      s.rd_v = 0.0;
      s.do_v = 1;
      s.upd_mode = 0;
      s.active = 1;
      s.pending = 0;
      if (id == 0) a.counters[0] = 0;
      break;
    }
    case PH_INIT_ALPHA: {
      // v = A'u; alpha = ||v||; v /= alpha  (lsmr.jl:66-68)
      s.alpha = sqrt(s1);
      s.s_v = s.alpha > 0 ? 1.0 / s.alpha : 1.0;
      lsmr_init(s, a.init_mode);
      atomicAdd(a.counters, s.active);
      break;
    }
    case PH_BETA: {
      // counters[2]: instances running in this iteration (read by the
      // reductions that follow); counters[0] collects the next count
      if (id == 0) {
        a.counters[2] = a.counters[0];
        a.counters[0] = 0;
      }
      if (!s.active) break;
      // beta = ||u||; if beta > 0: u /= beta, v = A'u - beta v  (lsmr.jl:104-108)
      s.beta = sqrt(s0);
      if (s.beta > 0) {
        s.u_scale = 1.0 / s.beta;
        s.rd_acc = s.u_scale;
        s.rd_v = s.beta * s.s_v;
        s.do_v = 1;
      } else {
        s.u_scale = 1.0;
        s.do_v = 0;
      }
      break;
    }
    case PH_ALPHA: {
      if (!s.active) break;
      if (s.pending) {
        s.normx = sqrt(s2);
        lsmr_test(s);
        s.pending = 0;
        if (s.istop) {
          deactivate(s);
          break;
        }
      }
      s.iter += 1;
      if (s.do_v) {
        s.alpha = sqrt(s1);
        s.s_v = s.alpha > 0 ? 1.0 / s.alpha : 1.0;
      }
      lsmr_rotate(s);
      s.upd_mode = 2;
      s.pending = 1;
      s.ex_av = s.s_v;
      s.ex_au = -s.alpha * s.u_scale;
      atomicAdd(a.counters, 1);
      break;
    }
    case PH_OUTER: {
      // FP64 iterative refinement: r = b - A x64 and g = A'r were computed in
      // FP64; test them with the reference's tests 1 and 2, else start another
      // FP32 inner LSMR on the correction problem min ||r - A dx||.
      if (!s.outer_active) break;
      const double nr = sqrt(s0), ng = sqrt(s1), nx = sqrt(s2);
      if (s.outer_rounds == 0) {
        s.normb0 = nr;
        s.normA2_prev = 0.0;
        s.iter_total = 0;
      } else {
        s.iter_total += s.iter;
        if (s.iter > 0) s.normA2_prev += s.normA * s.normA;
      }
      const double nAt = sqrt(s.normA2_prev);
      if (!isfinite(nr) || !isfinite(ng)) {
        // a NaN or infinite right-hand side: stop, not converged (the
        // reference's verdict after maxiter iterations on NaN norms)
        s.last_test2 = nr * ng;
        s.converged = 0;
        s.outer_active = 0;
        deactivate(s);
        break;
      }
      bool conv = false;
      s.last_test2 = (nAt > 0 && nr > 0) ? ng / (nAt * nr) : (ng == 0.0 ? 0.0 : 1.0);
      if (s.skip_lsmr || ng == 0.0 || nr == 0.0) {
        conv = true;
      } else if (nAt > 0) {
        const double test2 = ng / (nAt * nr);
        const double test1 = nr / s.normb0;
        const double rtol = s.tol_b + s.tol_a * nAt * nx / s.normb0;
        conv = (test2 <= s.tol_a) || (test1 <= rtol);
      }
      if (conv) {
        s.converged = 1;
        s.outer_active = 0;
        deactivate(s);
        break;
      }
      if (s.iter_total >= s.maxiter_total || s.outer_rounds >= s.max_rounds) {
        s.converged = 0;
        s.outer_active = 0;
        deactivate(s);
        break;
      }
      s.outer_rounds += 1;
      s.mode_inner = 1;
      s.maxiter = s.maxiter_total - s.iter_total;
      // u0 = r/||r||, v0 = A'u0/alpha0 with A'u0 = g/||r|| computed in FP64
      s.beta = nr;
      s.u_scale = 1.0 / nr;
      s.alpha = ng / nr;
      s.s_v = 1.0 / ng;
      lsmr_init(s, 3);
      s.normAr0 = s.normAr;
      atomicAdd(a.counters, 1);      // LSMR running (read by the first beta phase)
      atomicAdd(a.counters + 1, 1);  // refinement running
      atomicAdd(a.counters + 2, 1);  // running, for kernels before the first beta
      break;
    }
    default:
      break;
  }
}

void launch_scalar(const ScalarArgs& a, int n_inst, cudaStream_t s) {
  k_scalar<<<n_inst, kScalarThreads, 0, s>>>(a);
}

}  // namespace fe
