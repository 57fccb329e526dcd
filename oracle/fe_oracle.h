/*
 * fe_oracle.h -- TEST INFRASTRUCTURE ONLY (the parity checker).
 *
 * A CPU, FP64 restatement of FixedEffects.jl v3.1.0's solver path, written in
 * plain C.  Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline
 * leg may load it; the product library never links or calls it.
 *
 * Every function cites the reference file:line it restates (paths relative to
 * the FixedEffects.jl project root).
 */
#ifndef FE_ORACLE_H
#define FE_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes (0 = OK). */
#define ORA_OK 0
#define ORA_ERR_INVALID 1
#define ORA_ERR_ALLOC 2

/* Per-iteration trace record written by the LSMR restatement when a trace
 * buffer is given (one record per LSMR iteration, 10 doubles):
 *   alpha, beta, normr, normAr, normA, condA, normx, test1, test2, istop */
#define ORA_TRACE_WIDTH 10

/*
 * solve_residuals!(y, fes, w; double_precision=true, tol, maxiter)
 *   src/AbstractFixedEffectSolver.jl:37-68 with the CPU backend of
 *   src/SolverCPU.jl and LSMR of src/utils/lsmr.jl.
 * refs[k][i] are 1-based level ids in 1..nlev[k].  interaction[k] may be NULL
 * (UnitWeights).  weights may be NULL (UnitWeights).  y is overwritten with
 * the residuals.  iters/converged receive the reference's return values
 * (mvps + 1, isconverged).  nthreads <= 0 means "all online cores".
 */
int ora_solve_residuals(int64_t N, int32_t K, const int64_t* const* refs,
                        const int64_t* nlev, const double* const* interaction,
                        const double* weights, double* y, double tol,
                        int64_t maxiter, int32_t nthreads, int64_t* iters,
                        int32_t* converged, double* trace, int64_t trace_cap);

/* The collection method: src/AbstractFixedEffectSolver.jl:74-97 (one solver,
 * columns solved one after the other).  Y is column-major N x ncols. */
int ora_solve_residuals_cols(int64_t N, int32_t K, const int64_t* const* refs,
                             const int64_t* nlev,
                             const double* const* interaction,
                             const double* weights, double* Y, int64_t ncols,
                             double tol, int64_t maxiter, int32_t nthreads,
                             int64_t* iters, int32_t* converged);

/*
 * solve_coefficients!(y, fes, w): src/AbstractFixedEffectSolver.jl:137-160,
 * then normalize!/full of src/FixedEffect.jl:106-140.
 * coef_levels[k] receives nlev[k] normalized coefficients (may be NULL);
 * coef_full[k] receives the N per-observation values fecoef[refs[i]]
 * (may be NULL).  iters receives div(mvps, 2).
 */
int ora_solve_coefficients(int64_t N, int32_t K, const int64_t* const* refs,
                           const int64_t* nlev,
                           const double* const* interaction,
                           const double* weights, const double* y, double tol,
                           int64_t maxiter, int32_t nthreads,
                           double* const* coef_levels,
                           double* const* coef_full, int64_t* iters,
                           int32_t* converged);

/* Jacobi preconditioner scale!: src/SolverCPU.jl:78-89 (serial, ascending i). */
void ora_scale(double* scale, int64_t n, const int64_t* refs,
               const double* interaction, const double* weights, int64_t N);

/*
 * Integer plan restatement: the stable counting sort of
 * ext/MetalExt.jl:40-64 (bucketize_refs), applied first to the primary FE
 * (giving the observation order perm0) and then to every FE over the
 * primary-sorted positions.
 *   perm0[p]     = original observation (0-based) at sorted position p
 *   offsets[k]   = nlev[k]+1 exclusive prefix counts (0-based)
 *   segperm[k][q]= sorted position of the q-th entry of FE k's level order
 * segperm[primary] is the identity and may be NULL.
 */
int ora_integer_plan(int64_t N, int32_t K, const int64_t* const* refs,
                     const int64_t* nlev, int32_t primary, int32_t* perm0,
                     int64_t* const* offsets, int32_t* const* segperm);

/* Connected components of the observation/level graph, as in
 * src/FixedEffect.jl:68-98; returns the number of components and writes the
 * component id of every observation (numbered in order of first
 * observation). */
int64_t ora_components(int64_t N, int32_t K, const int64_t* const* refs,
                       const int64_t* nlev, int64_t* comp_of_obs);

#ifdef __cplusplus
}
#endif
#endif
