/*
 * fe_oracle.c -- TEST INFRASTRUCTURE ONLY (the parity checker).
 *
 * CPU FP64 restatement of the FixedEffects.jl v3.1.0 solver path:
 *   src/SolverCPU.jl                 preconditioner, gather!/scatter!
 *   src/AbstractFixedEffectLinearMap.jl  mul! pair
 *   src/FixedEffectCoefficients.jl   block-vector norm/fill/rmul!/copyto!/axpy!
 *   src/utils/lsmr.jl                LSMR (Fong & Saunders), lambda = 0
 *   src/AbstractFixedEffectSolver.jl solve_residuals!/solve_coefficients!
 *   src/FixedEffect.jl               components/normalize!/full
 *   ext/MetalExt.jl:40-64            stable counting sort (bucketize_refs)
 * Loaded only by tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline; the product library never links or calls this file.
 *
 * The reduce (gather!) is serial in ascending observation order, exactly as
 * src/SolverCPU.jl:20-27; the expand (scatter!) and cache! are threaded over
 * 100_000-row chunks like GroupedArrays.@spawn_for_chunks
 * (src/SolverCPU.jl:31,92).  Each chunk writes disjoint rows, so results do
 * not depend on the thread count.
 */
#define _GNU_SOURCE
#include "fe_oracle.h"

#include <math.h>
#include <pthread.h>
#include <stdatomic.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>

#define CHUNK 100000

/* ------------------------------------------------------------------------ */
/* chunked parallel-for (stand-in for GroupedArrays.@spawn_for_chunks)       */
/* ------------------------------------------------------------------------ */
typedef void (*chunk_fn)(void* ctx, int64_t lo, int64_t hi);
typedef struct {
  chunk_fn fn;
  void* ctx;
  int64_t n;
  atomic_llong next;
} pfor_t;

static void* pfor_worker(void* arg) {
  pfor_t* p = (pfor_t*)arg;
  for (;;) {
    long long c = atomic_fetch_add(&p->next, 1);
    int64_t lo = (int64_t)c * CHUNK;
    if (lo >= p->n) break;
    int64_t hi = lo + CHUNK < p->n ? lo + CHUNK : p->n;
    p->fn(p->ctx, lo, hi);
  }
  return NULL;
}

static int g_threads = 1;

static void parallel_for_chunks(int64_t n, chunk_fn fn, void* ctx) {
  int64_t nchunks = (n + CHUNK - 1) / CHUNK;
  int nt = g_threads;
  if (nt > nchunks) nt = (int)nchunks;
  if (nt <= 1) {
    if (n > 0) fn(ctx, 0, n);
    return;
  }
  pfor_t p;
  p.fn = fn;
  p.ctx = ctx;
  p.n = n;
  atomic_init(&p.next, 0);
  pthread_t th[256];
  if (nt > 256) nt = 256;
  int started = 0;
  for (int t = 1; t < nt; ++t)
    if (pthread_create(&th[started], NULL, pfor_worker, &p) == 0) ++started;
  pfor_worker(&p);
  for (int t = 0; t < started; ++t) pthread_join(th[t], NULL);
}

static int resolve_threads(int32_t nthreads) {
  if (nthreads > 0) return nthreads;
  long c = sysconf(_SC_NPROCESSORS_ONLN);
  return c > 0 ? (int)c : 1;
}

/* ------------------------------------------------------------------------ */
/* reductions                                                                */
/* ------------------------------------------------------------------------ */
/* pairwise sum of squares (Julia's sum(abs2, x) is pairwise with 1024-wide
 * leaves: Base.mapreduce_impl) */
static double sumsq(const double* x, int64_t n) {
  if (n <= 1024) {
    double s = 0.0;
    for (int64_t i = 0; i < n; ++i) s += x[i] * x[i];
    return s;
  }
  int64_t h = n >> 1;
  return sumsq(x, h) + sumsq(x + h, n - h);
}

static double vnorm(const double* x, int64_t n) { return sqrt(sumsq(x, n)); }

/* ------------------------------------------------------------------------ */
/* linear map A = D' diag(scale) with sqrt(w) and interaction folded in      */
/* ------------------------------------------------------------------------ */
typedef struct {
  int64_t N;
  int32_t K;
  const int64_t* const* refs;
  const int64_t* nlev;
  double** scales; /* K x nlev[k] */
  double** caches; /* K x N */
} map_t;

/* scale!: src/SolverCPU.jl:78-89 (serial accumulation, zero-sum guard of
 * issue #97) */
void ora_scale(double* scale, int64_t n, const int64_t* refs,
               const double* interaction, const double* weights, int64_t N) {
  for (int64_t l = 0; l < n; ++l) scale[l] = 0.0;
  for (int64_t i = 0; i < N; ++i) {
    double a = interaction ? interaction[i] : 1.0;
    double w = weights ? weights[i] : 1.0;
    scale[refs[i] - 1] += (a * a) * w;
  }
  for (int64_t l = 0; l < n; ++l)
    scale[l] = scale[l] > 0 ? (1.0 / sqrt(scale[l])) : 0.0;
}

typedef struct {
  double* cache;
  const int64_t* refs;
  const double* interaction;
  const double* weights;
  const double* scale;
} cache_ctx;

static void cache_chunk(void* c, int64_t lo, int64_t hi) {
  cache_ctx* x = (cache_ctx*)c;
  for (int64_t i = lo; i < hi; ++i) {
    double a = x->interaction ? x->interaction[i] : 1.0;
    double w = x->weights ? x->weights[i] : 1.0;
    x->cache[i] = a * sqrt(w) * x->scale[x->refs[i] - 1];
  }
}

/* cache!: src/SolverCPU.jl:91-95 */
static void ora_cache(double* cache, const int64_t* refs,
                      const double* interaction, const double* weights,
                      const double* scale, int64_t N) {
  cache_ctx c = {cache, refs, interaction, weights, scale};
  parallel_for_chunks(N, cache_chunk, &c);
}

/* gather! (A' side, reduce by level): src/SolverCPU.jl:21-27, serial */
static void ora_gather(double* fecoef, const int64_t* refs, double alpha,
                       const double* y, const double* cache, int64_t N) {
  for (int64_t i = 0; i < N; ++i) fecoef[refs[i] - 1] += alpha * y[i] * cache[i];
}

typedef struct {
  double* y;
  double alpha;
  const double* fecoef;
  const int64_t* refs;
  const double* cache;
} scatter_ctx;

static void scatter_chunk(void* c, int64_t lo, int64_t hi) {
  scatter_ctx* x = (scatter_ctx*)c;
  for (int64_t i = lo; i < hi; ++i)
    x->y[i] += x->alpha * x->fecoef[x->refs[i] - 1] * x->cache[i];
}

/* scatter! (A side, expand to observations): src/SolverCPU.jl:29-34 */
static void ora_scatter(double* y, double alpha, const double* fecoef,
                        const int64_t* refs, const double* cache, int64_t N) {
  scatter_ctx c = {y, alpha, fecoef, refs, cache};
  parallel_for_chunks(N, scatter_chunk, &c);
}

/* block vector (FixedEffectCoefficients) helpers:
 * src/FixedEffectCoefficients.jl:21-55 */
static double bnorm_blk(const map_t* m, double* const* x) {
  double out = 0.0;
  for (int k = 0; k < m->K; ++k) out += sumsq(x[k], m->nlev[k]);
  return sqrt(out);
}
static void bfill_blk(const map_t* m, double* const* x, double a) {
  for (int k = 0; k < m->K; ++k)
    for (int64_t l = 0; l < m->nlev[k]; ++l) x[k][l] = a;
}
static void brmul_blk(const map_t* m, double* const* x, double a) {
  for (int k = 0; k < m->K; ++k)
    for (int64_t l = 0; l < m->nlev[k]; ++l) x[k][l] *= a;
}
static void bcopy_blk(const map_t* m, double* const* dst, double* const* src) {
  for (int k = 0; k < m->K; ++k)
    memcpy(dst[k], src[k], sizeof(double) * (size_t)m->nlev[k]);
}
static void baxpy_blk(const map_t* m, double a, double* const* x, double* const* y) {
  for (int k = 0; k < m->K; ++k)
    for (int64_t l = 0; l < m->nlev[k]; ++l) y[k][l] += a * x[k][l];
}

/* mul!(fecoefs, A', y, alpha, beta): src/AbstractFixedEffectLinearMap.jl:26-35 */
static void mul_adj(const map_t* m, double* const* fecoefs, const double* y,
                    double alpha, double beta) {
  brmul_blk(m, fecoefs, beta);
  for (int k = 0; k < m->K; ++k)
    ora_gather(fecoefs[k], m->refs[k], alpha, y, m->caches[k], m->N);
}

/* mul!(y, A, fecoefs, alpha, beta): src/AbstractFixedEffectLinearMap.jl:37-44 */
static void mul_fwd(const map_t* m, double* y, double* const* fecoefs,
                    double alpha, double beta) {
  for (int64_t i = 0; i < m->N; ++i) y[i] *= beta;
  for (int k = 0; k < m->K; ++k)
    ora_scatter(y, alpha, fecoefs[k], m->refs[k], m->caches[k], m->N);
}

/* ------------------------------------------------------------------------ */
/* LSMR: src/utils/lsmr.jl:46-222 (lambda = 0)                               */
/* ------------------------------------------------------------------------ */
typedef struct {
  int converged;
  int64_t mvps;
  int istop;
} conv_t;

static conv_t ora_lsmr(const map_t* m, double* const* x, double* b,
                       double* const* v, double* const* h, double* const* hbar,
                       double atol, double btol, double conlim,
                       int64_t maxiter, double* trace, int64_t trace_cap) {
  const double lambda = 0.0;
  double ctol = conlim > 0 ? 1.0 / conlim : 0.0;
  /* u = b - A x ; beta = ||u|| (lsmr.jl:63-65) */
  double* u = b;
  mul_fwd(m, u, x, -1.0, 1.0);
  double beta = vnorm(u, m->N);
  if (beta > 0) {
    double ib = 1.0 / beta;
    for (int64_t i = 0; i < m->N; ++i) u[i] *= ib;
  }
  mul_adj(m, v, u, 1.0, 0.0);
  double alpha = bnorm_blk(m, v);
  if (alpha > 0) brmul_blk(m, v, 1.0 / alpha);

  double zetabar = alpha * beta;
  double alphabar = alpha;
  double rho = 1.0, rhobar = 1.0, cbar = 1.0, sbar = 0.0;
  bcopy_blk(m, h, v);
  bfill_blk(m, hbar, 0.0);

  double betadd = beta, betad = 0.0, rhodold = 1.0, tautildeold = 0.0;
  double thetatilde = 0.0, zeta = 0.0, d = 0.0;
  double normA = -1.0, condA = -1.0, normx = -1.0;
  double normA2 = alpha * alpha;
  double maxrbar = 0.0, minrbar = 1e100;
  double normb = beta;
  int istop = 0;
  double normr = beta;
  double normAr = alpha * beta;
  int64_t iter = 0;
  (void)normr;
  if (normAr != 0) {
    while (iter < maxiter) {
      iter += 1;
      mul_fwd(m, u, v, 1.0, -alpha);
      beta = vnorm(u, m->N);
      if (beta > 0) {
        double ib = 1.0 / beta;
        for (int64_t i = 0; i < m->N; ++i) u[i] *= ib;
        mul_adj(m, v, u, 1.0, -beta);
        alpha = bnorm_blk(m, v);
        if (alpha > 0) brmul_blk(m, v, 1.0 / alpha);
      }
      /* rotation Qhat_{k,2k+1} */
      double alphahat = sqrt(alphabar * alphabar + lambda * lambda);
      double chat = alphabar / alphahat;
      double shat = lambda / alphahat;
      /* rotation Q_i */
      double rhoold = rho;
      rho = sqrt(alphahat * alphahat + beta * beta);
      double c = alphahat / rho;
      double s = beta / rho;
      double thetanew = s * alpha;
      alphabar = c * alpha;
      /* rotation Qbar_i */
      double rhobarold = rhobar;
      double zetaold = zeta;
      double thetabar = sbar * rho;
      double rhotemp = cbar * rho;
      rhobar = sqrt((cbar * rho) * (cbar * rho) + thetanew * thetanew);
      cbar = cbar * rho / rhobar;
      sbar = thetanew / rhobar;
      zeta = cbar * zetabar;
      zetabar = -sbar * zetabar;
      /* update h, hbar, x (lsmr.jl:138-142) */
      brmul_blk(m, hbar, -thetabar * rho / (rhoold * rhobarold));
      baxpy_blk(m, 1.0, h, hbar);
      baxpy_blk(m, zeta / (rho * rhobar), hbar, x);
      brmul_blk(m, h, -thetanew / rho);
      baxpy_blk(m, 1.0, v, h);
      /* estimate of ||r|| */
      double betaacute = chat * betadd;
      double betacheck = -shat * betadd;
      double betahat = c * betaacute;
      betadd = -s * betaacute;
      double thetatildeold = thetatilde;
      double rhotildeold = sqrt(rhodold * rhodold + thetabar * thetabar);
      double ctildeold = rhodold / rhotildeold;
      double stildeold = thetabar / rhotildeold;
      thetatilde = stildeold * rhobar;
      rhodold = ctildeold * rhobar;
      betad = -stildeold * betad + ctildeold * betahat;
      tautildeold = (zetaold - thetatildeold * tautildeold) / rhotildeold;
      double taud = (zeta - thetatilde * tautildeold) / rhodold;
      d = d + betacheck * betacheck;
      normr = sqrt(d + (betad - taud) * (betad - taud) + betadd * betadd);
      /* estimate ||A|| */
      normA2 = normA2 + beta * beta;
      normA = sqrt(normA2);
      normA2 = normA2 + alpha * alpha;
      /* estimate cond(A) */
      maxrbar = maxrbar > rhobarold ? maxrbar : rhobarold;
      if (iter > 1) minrbar = minrbar < rhobarold ? minrbar : rhobarold;
      double mx = maxrbar > rhotemp ? maxrbar : rhotemp;
      double mn = minrbar < rhotemp ? minrbar : rhotemp;
      condA = mx / mn;
      /* convergence tests (lsmr.jl:188-215) */
      normAr = fabs(zetabar);
      normx = bnorm_blk(m, x);
      double test1 = normr / normb;
      double test2 = normAr / (normA * normr);
      double test3 = 1.0 / condA;
      double t1 = test1 / (1.0 + normA * normx / normb);
      double rtol = btol + atol * normA * normx / normb;
      if (iter >= maxiter) istop = 7;
      else if (1 + test3 <= 1) istop = 6;
      else if (1 + test2 <= 1) istop = 5;
      else if (1 + t1 <= 1) istop = 4;
      else if (test3 <= ctol) istop = 3;
      else if (test2 <= atol) istop = 2;
      else if (test1 <= rtol) istop = 1;
      if (trace && iter <= trace_cap) {
        double* t = trace + (iter - 1) * ORA_TRACE_WIDTH;
        t[0] = alpha; t[1] = beta; t[2] = normr; t[3] = normAr; t[4] = normA;
        t[5] = condA; t[6] = normx; t[7] = test1; t[8] = test2; t[9] = istop;
      }
      if (istop) break;
    }
  }
  conv_t r;
  r.istop = istop;
  r.converged = !(istop == 3 || istop == 6 || istop == 7);
  r.mvps = iter;
  return r;
}

/* ------------------------------------------------------------------------ */
/* solver object (FixedEffectSolverCPU, src/SolverCPU.jl:43-76)              */
/* ------------------------------------------------------------------------ */
typedef struct {
  map_t m;
  const double* weights;
  double *b, *r;
  double **x, **v, **h, **hbar;
  double* slab;
} solver_t;

static void solver_free(solver_t* s) {
  free(s->slab);
  free(s->m.scales);
  free(s->m.caches);
  free(s->x);
  free(s->v);
  free(s->h);
  free(s->hbar);
}

static int validate(int64_t N, int32_t K, const int64_t* const* refs,
                    const int64_t* nlev) {
  if (N < 0 || K < 1 || !refs || !nlev) return ORA_ERR_INVALID;
  for (int k = 0; k < K; ++k) {
    if (!refs[k] || nlev[k] < 0) return ORA_ERR_INVALID;
    for (int64_t i = 0; i < N; ++i)
      if (refs[k][i] < 1 || refs[k][i] > nlev[k]) return ORA_ERR_INVALID;
  }
  return ORA_OK;
}

/* AbstractFixedEffectSolver{Float64}(fes, w, Val{:cpu}) + update_weights!:
 * src/SolverCPU.jl:55-76 */
static int solver_init(solver_t* s, int64_t N, int32_t K,
                       const int64_t* const* refs, const int64_t* nlev,
                       const double* const* interaction,
                       const double* weights) {
  memset(s, 0, sizeof(*s));
  s->m.N = N;
  s->m.K = K;
  s->m.refs = refs;
  s->m.nlev = nlev;
  s->weights = weights;
  int64_t P = 0;
  for (int k = 0; k < K; ++k) P += nlev[k];
  size_t total = (size_t)(2 * N + (int64_t)K * N + 5 * P);
  s->slab = (double*)calloc(total > 0 ? total : 1, sizeof(double));
  s->m.scales = (double**)calloc((size_t)K, sizeof(double*));
  s->m.caches = (double**)calloc((size_t)K, sizeof(double*));
  s->x = (double**)calloc((size_t)K, sizeof(double*));
  s->v = (double**)calloc((size_t)K, sizeof(double*));
  s->h = (double**)calloc((size_t)K, sizeof(double*));
  s->hbar = (double**)calloc((size_t)K, sizeof(double*));
  if (!s->slab || !s->m.scales || !s->m.caches || !s->x || !s->v || !s->h ||
      !s->hbar) {
    solver_free(s);
    return ORA_ERR_ALLOC;
  }
  double* p = s->slab;
  s->b = p; p += N;
  s->r = p; p += N;
  for (int k = 0; k < K; ++k) { s->m.caches[k] = p; p += N; }
  for (int k = 0; k < K; ++k) { s->m.scales[k] = p; p += nlev[k]; }
  for (int k = 0; k < K; ++k) { s->x[k] = p; p += nlev[k]; }
  for (int k = 0; k < K; ++k) { s->v[k] = p; p += nlev[k]; }
  for (int k = 0; k < K; ++k) { s->h[k] = p; p += nlev[k]; }
  for (int k = 0; k < K; ++k) { s->hbar[k] = p; p += nlev[k]; }
  for (int k = 0; k < K; ++k)
    ora_scale(s->m.scales[k], nlev[k], refs[k],
              interaction ? interaction[k] : NULL, weights, N);
  for (int k = 0; k < K; ++k)
    ora_cache(s->m.caches[k], refs[k], interaction ? interaction[k] : NULL,
              weights, s->m.scales[k], N);
  return ORA_OK;
}

/* solve_residuals!(r, feM): src/AbstractFixedEffectSolver.jl:49-68 */
static void solver_residuals(solver_t* s, double* y, double tol,
                             int64_t maxiter, int64_t* iters, int32_t* conv,
                             double* trace, int64_t trace_cap) {
  const int64_t N = s->m.N;
  memcpy(s->r, y, sizeof(double) * (size_t)N);
  if (s->weights)
    for (int64_t i = 0; i < N; ++i) s->r[i] *= sqrt(s->weights[i]);
  memcpy(s->b, s->r, sizeof(double) * (size_t)N);
  mul_adj(&s->m, s->x, s->b, 1.0, 0.0);
  int64_t iter = 1;
  int converged = 1;
  if (s->m.K > 1) {
    conv_t c = ora_lsmr(&s->m, s->x, s->b, s->v, s->h, s->hbar, tol, tol, 1e8,
                        maxiter - 1, trace, trace_cap);
    iter = c.mvps + 1;
    converged = c.converged;
  }
  mul_fwd(&s->m, s->r, s->x, -1.0, 1.0);
  if (s->weights)
    for (int64_t i = 0; i < N; ++i) s->r[i] /= sqrt(s->weights[i]);
  memcpy(y, s->r, sizeof(double) * (size_t)N);
  if (iters) *iters = iter;
  if (conv) *conv = converged;
}

int ora_solve_residuals(int64_t N, int32_t K, const int64_t* const* refs,
                        const int64_t* nlev, const double* const* interaction,
                        const double* weights, double* y, double tol,
                        int64_t maxiter, int32_t nthreads, int64_t* iters,
                        int32_t* converged, double* trace, int64_t trace_cap) {
  int st = validate(N, K, refs, nlev);
  if (st) return st;
  g_threads = resolve_threads(nthreads);
  solver_t s;
  st = solver_init(&s, N, K, refs, nlev, interaction, weights);
  if (st) return st;
  solver_residuals(&s, y, tol, maxiter, iters, converged, trace, trace_cap);
  solver_free(&s);
  return ORA_OK;
}

/* collection method: src/AbstractFixedEffectSolver.jl:74-97 */
int ora_solve_residuals_cols(int64_t N, int32_t K, const int64_t* const* refs,
                             const int64_t* nlev,
                             const double* const* interaction,
                             const double* weights, double* Y, int64_t ncols,
                             double tol, int64_t maxiter, int32_t nthreads,
                             int64_t* iters, int32_t* converged) {
  int st = validate(N, K, refs, nlev);
  if (st) return st;
  g_threads = resolve_threads(nthreads);
  solver_t s;
  st = solver_init(&s, N, K, refs, nlev, interaction, weights);
  if (st) return st;
  for (int64_t j = 0; j < ncols; ++j)
    solver_residuals(&s, Y + j * N, tol, maxiter, iters ? iters + j : NULL,
                     converged ? converged + j : NULL, NULL, 0);
  solver_free(&s);
  return ORA_OK;
}

/* ------------------------------------------------------------------------ */
/* components / normalize! / full: src/FixedEffect.jl:57-140                 */
/* ------------------------------------------------------------------------ */
static int64_t uf_find(int64_t* parent, int64_t a) {
  while (parent[a] != a) {
    parent[a] = parent[parent[a]];
    a = parent[a];
  }
  return a;
}

/* Labels the connected components of the bipartite observation/level graph
 * over the FEs listed in idx[0..nidx).  The reference runs a BFS from every
 * unvisited observation in ascending order (src/FixedEffect.jl:68-98);
 * union-find over the levels gives the same partition.  Components are
 * numbered in order of their first observation.  level_comp[k] (offsets
 * into one array) receives the component id of every level, -1 for levels
 * that no observation uses. */
static int64_t components_idx(int64_t N, const int64_t* const* refs,
                              const int64_t* nlev, const int32_t* idx,
                              int32_t nidx, int64_t* comp_of_obs,
                              int64_t* level_comp, int64_t* level_off) {
  int64_t total = 0;
  for (int j = 0; j < nidx; ++j) {
    level_off[j] = total;
    total += nlev[idx[j]];
  }
  level_off[nidx] = total;
  int64_t* parent = (int64_t*)malloc(sizeof(int64_t) * (size_t)(total + 1));
  if (!parent) return -1;
  for (int64_t a = 0; a < total; ++a) parent[a] = a;
  for (int64_t i = 0; i < N; ++i) {
    int64_t a = uf_find(parent, level_off[0] + refs[idx[0]][i] - 1);
    for (int j = 1; j < nidx; ++j) {
      int64_t b = uf_find(parent, level_off[j] + refs[idx[j]][i] - 1);
      if (a != b) {
        if (a < b) { parent[b] = a; }
        else { parent[a] = b; a = b; }
      }
    }
  }
  for (int64_t a = 0; a < total; ++a) level_comp[a] = -1;
  /* root -> component id, in order of first observation */
  int64_t* root_id = (int64_t*)malloc(sizeof(int64_t) * (size_t)(total + 1));
  if (!root_id) { free(parent); return -1; }
  for (int64_t a = 0; a < total; ++a) root_id[a] = -1;
  int64_t ncomp = 0;
  for (int64_t i = 0; i < N; ++i) {
    int64_t r = uf_find(parent, level_off[0] + refs[idx[0]][i] - 1);
    if (root_id[r] < 0) root_id[r] = ncomp++;
    if (comp_of_obs) comp_of_obs[i] = root_id[r];
  }
  for (int64_t i = 0; i < N; ++i)
    for (int j = 0; j < nidx; ++j) {
      int64_t a = level_off[j] + refs[idx[j]][i] - 1;
      level_comp[a] = root_id[uf_find(parent, a)];
    }
  free(root_id);
  free(parent);
  return ncomp;
}

int64_t ora_components(int64_t N, int32_t K, const int64_t* const* refs,
                       const int64_t* nlev, int64_t* comp_of_obs) {
  if (validate(N, K, refs, nlev)) return -1;
  int32_t* idx = (int32_t*)malloc(sizeof(int32_t) * (size_t)K);
  int64_t* level_off = (int64_t*)malloc(sizeof(int64_t) * (size_t)(K + 1));
  int64_t total = 0;
  for (int k = 0; k < K; ++k) { idx[k] = k; total += nlev[k]; }
  int64_t* level_comp = (int64_t*)malloc(sizeof(int64_t) * (size_t)(total + 1));
  int64_t nc = -1;
  if (idx && level_off && level_comp)
    nc = components_idx(N, refs, nlev, idx, K, comp_of_obs, level_comp,
                        level_off);
  free(idx);
  free(level_off);
  free(level_comp);
  return nc;
}

/* normalize!/rescale!: src/FixedEffect.jl:106-135.  Within every connected
 * component, every FE except the first (of the non-interacted ones) is
 * demeaned over the component's levels, and the sum of those means is added
 * to the first FE. */
static int normalize_coefs(int64_t N, int32_t K, const int64_t* const* refs,
                           const int64_t* nlev,
                           const double* const* interaction,
                           double* const* coefs) {
  int32_t* idx = (int32_t*)malloc(sizeof(int32_t) * (size_t)K);
  if (!idx) return ORA_ERR_ALLOC;
  int32_t nidx = 0;
  for (int k = 0; k < K; ++k)
    if (!interaction || !interaction[k]) idx[nidx++] = k;
  if (nidx < 2) { free(idx); return ORA_OK; }
  int64_t* level_off = (int64_t*)malloc(sizeof(int64_t) * (size_t)(nidx + 1));
  int64_t total = 0;
  for (int j = 0; j < nidx; ++j) total += nlev[idx[j]];
  int64_t* level_comp = (int64_t*)malloc(sizeof(int64_t) * (size_t)(total + 1));
  if (!level_off || !level_comp) {
    free(idx); free(level_off); free(level_comp);
    return ORA_ERR_ALLOC;
  }
  int64_t nc = components_idx(N, refs, nlev, idx, nidx, NULL, level_comp,
                              level_off);
  if (nc < 0) {
    free(idx); free(level_off); free(level_comp);
    return ORA_ERR_ALLOC;
  }
  double* sum = (double*)calloc((size_t)(nc + 1), sizeof(double));
  int64_t* cnt = (int64_t*)calloc((size_t)(nc + 1), sizeof(int64_t));
  double* m = (double*)calloc((size_t)(nc + 1), sizeof(double));
  if (!sum || !cnt || !m) {
    free(idx); free(level_off); free(level_comp); free(sum); free(cnt); free(m);
    return ORA_ERR_ALLOC;
  }
  for (int j = nidx - 1; j >= 1; --j) {
    int k = idx[j];
    memset(sum, 0, sizeof(double) * (size_t)nc);
    memset(cnt, 0, sizeof(int64_t) * (size_t)nc);
    for (int64_t l = 0; l < nlev[k]; ++l) {
      int64_t c = level_comp[level_off[j] + l];
      if (c < 0) continue;
      sum[c] += coefs[k][l];
      cnt[c] += 1;
    }
    for (int64_t c = 0; c < nc; ++c) sum[c] = cnt[c] ? sum[c] / (double)cnt[c] : 0.0;
    for (int64_t l = 0; l < nlev[k]; ++l) {
      int64_t c = level_comp[level_off[j] + l];
      if (c < 0) continue;
      coefs[k][l] -= sum[c];
    }
    for (int64_t c = 0; c < nc; ++c) m[c] += sum[c];
  }
  int k0 = idx[0];
  for (int64_t l = 0; l < nlev[k0]; ++l) {
    int64_t c = level_comp[level_off[0] + l];
    if (c >= 0) coefs[k0][l] += m[c];
  }
  free(idx); free(level_off); free(level_comp); free(sum); free(cnt); free(m);
  return ORA_OK;
}

/* solve_coefficients!(r, feM): src/AbstractFixedEffectSolver.jl:147-160 */
int ora_solve_coefficients(int64_t N, int32_t K, const int64_t* const* refs,
                           const int64_t* nlev,
                           const double* const* interaction,
                           const double* weights, const double* y, double tol,
                           int64_t maxiter, int32_t nthreads,
                           double* const* coef_levels,
                           double* const* coef_full, int64_t* iters,
                           int32_t* converged) {
  int st = validate(N, K, refs, nlev);
  if (st) return st;
  g_threads = resolve_threads(nthreads);
  solver_t s;
  st = solver_init(&s, N, K, refs, nlev, interaction, weights);
  if (st) return st;
  memcpy(s.b, y, sizeof(double) * (size_t)N);
  if (weights)
    for (int64_t i = 0; i < N; ++i) s.b[i] *= sqrt(weights[i]);
  bfill_blk(&s.m, s.x, 0.0);
  conv_t c = ora_lsmr(&s.m, s.x, s.b, s.v, s.h, s.hbar, tol, tol, 1e8, maxiter,
                      NULL, 0);
  for (int k = 0; k < K; ++k)
    for (int64_t l = 0; l < nlev[k]; ++l) s.x[k][l] *= s.m.scales[k][l];
  st = normalize_coefs(N, K, refs, nlev, interaction, s.x);
  if (st == ORA_OK) {
    for (int k = 0; k < K; ++k) {
      if (coef_levels && coef_levels[k])
        memcpy(coef_levels[k], s.x[k], sizeof(double) * (size_t)nlev[k]);
      if (coef_full && coef_full[k])
        for (int64_t i = 0; i < N; ++i) coef_full[k][i] = s.x[k][refs[k][i] - 1];
    }
    if (iters) *iters = c.mvps / 2;
    if (converged) *converged = c.converged;
  }
  solver_free(&s);
  return st;
}

/* ------------------------------------------------------------------------ */
/* integer plan: stable counting sort of ext/MetalExt.jl:40-64               */
/* ------------------------------------------------------------------------ */
/* bucketize_refs restated with 0-based positions: counts per level, exclusive
 * prefix offsets, then observations placed in ascending order inside their
 * level's bucket. */
static void bucketize(const int64_t* key, int64_t N, int64_t n, int64_t* offsets,
                      int32_t* perm, int64_t* next) {
  for (int64_t l = 0; l <= n; ++l) offsets[l] = 0;
  for (int64_t i = 0; i < N; ++i) offsets[key[i]] += 1; /* key is 1-based */
  /* offsets[l] now holds count of level l (1-based shift) */
  offsets[0] = 0;
  for (int64_t l = 1; l <= n; ++l) offsets[l] += offsets[l - 1];
  for (int64_t l = 0; l < n; ++l) next[l] = offsets[l];
  for (int64_t i = 0; i < N; ++i) perm[next[key[i] - 1]++] = (int32_t)i;
}

int ora_integer_plan(int64_t N, int32_t K, const int64_t* const* refs,
                     const int64_t* nlev, int32_t primary, int32_t* perm0,
                     int64_t* const* offsets, int32_t* const* segperm) {
  int st = validate(N, K, refs, nlev);
  if (st) return st;
  if (primary < 0 || primary >= K || !perm0 || !offsets) return ORA_ERR_INVALID;
  int64_t nmax = 0;
  for (int k = 0; k < K; ++k) nmax = nlev[k] > nmax ? nlev[k] : nmax;
  int64_t* next = (int64_t*)malloc(sizeof(int64_t) * (size_t)(nmax + 1));
  int64_t* key = (int64_t*)malloc(sizeof(int64_t) * (size_t)(N + 1));
  int32_t* tmp = (int32_t*)malloc(sizeof(int32_t) * (size_t)(N + 1));
  if (!next || !key || !tmp) { free(next); free(key); free(tmp); return ORA_ERR_ALLOC; }
  bucketize(refs[primary], N, nlev[primary], offsets[primary], perm0, next);
  for (int k = 0; k < K; ++k) {
    for (int64_t p = 0; p < N; ++p) key[p] = refs[k][perm0[p]];
    int32_t* out = (segperm && segperm[k]) ? segperm[k] : tmp;
    bucketize(key, N, nlev[k], offsets[k], out, next);
  }
  free(next); free(key); free(tmp);
  return ORA_OK;
}
