/*
 * fe_b200.h -- C ABI of the B200-native fixed-effects LSMR library
 * (libfe_b200.so, built for sm_100a).
 *
 * This is the drop-in boundary for FixedEffects.jl's GPU solver path.  A host
 * binding (a Julia ccall extension, Python ctypes, ...) calls these functions
 * with plain pointers and sizes; no CUDA, torch or Julia types appear here.
 * Each declaration names the reference interface it replaces (paths are
 * relative to the FixedEffects.jl project root).
 *
 * Conventions
 *   - Every function returns a status: FE_OK (0) or an FE_ERR_* code; the
 *     message of the last error of the calling thread is fe_last_error().
 *     Input errors are reported, never thrown; non-convergence is not an
 *     error (it is returned in `converged`, as the reference does).
 *   - refs are 1-based level ids, as FixedEffect.refs in the reference
 *     (src/FixedEffect.jl:7-21).  interaction[k] == NULL means
 *     UnitWeights; weights == NULL means UnitWeights.
 *   - Y is column-major (Julia layout): column j starts at Y + j*ld.
 *   - A plan is not thread-safe; different plans may be used concurrently.
 *     The plan owns all device memory; host buffers are borrowed for the
 *     duration of a call.  For host-buffer calls, pinned (page-locked)
 *     memory gives full PCIe bandwidth.
 */
#ifndef FE_B200_H
#define FE_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define FE_B200_VERSION 1

/* status codes */
#define FE_OK 0
#define FE_ERR_INVALID 1 /* bad argument (lengths, level ids, null pointers) */
#define FE_ERR_CUDA 2    /* CUDA runtime error (message in fe_last_error) */
#define FE_ERR_ALLOC 3   /* device allocation failed */
#define FE_ERR_TIMEOUT 4 /* a bounded device wait gave up */

/* precision modes (the reference's `double_precision` keyword,
 * src/AbstractFixedEffectSolver.jl:37-43) */
#define FE_PREC_FP64 0  /* FP64 bulk + FP64 scalars: double_precision = true  */
#define FE_PREC_MIXED 1 /* FP32 bulk + FP64 scalars + FP64 refinement to tol  */
#define FE_PREC_FP32 2  /* FP32 bulk + FP64 scalars, no refinement            */

/* element types of Y */
#define FE_DTYPE_F64 0
#define FE_DTYPE_F32 1

/* plan options (fe_plan_set_option) */
#define FE_OPT_TILE 1        /* column-tile width cap: 0 auto (<=32), 1,2,4,..,32 */
#define FE_OPT_CHECK_EVERY 2 /* LSMR iterations between host convergence checks */
#define FE_OPT_MAX_ROUNDS 3  /* FP64 refinement rounds (FE_PREC_MIXED) */
#define FE_OPT_PROFILE 4     /* 1: time every launch with CUDA events */
#define FE_OPT_INNER_RHO 5   /* FP32 inner-solve floor (relative ||A'r|| drop) */
#define FE_OPT_FUSE 6        /* 1 (default): 32-column tiles of single-problem plans
                                reduce the primary FE and up to two small FEs in one
                                contiguous row-sum pass; 0: every FE by the
                                level-order segsum */
#define FE_OPT_EXPAND_VARIANT 7 /* expand kernel variant 0..5, -1 = default */
#define FE_OPT_SEGSUM_VARIANT 8 /* segsum kernel variant 0..5, -1 = default */
#define FE_OPT_AUTOTUNE 9    /* 1 (default): time the kernel variants on the first
                                solve of a tile shape; the choice is kept in the
                                plan and in the tuning cache file
                                ($FE_B200_TUNE_CACHE, "off" disables) */
#define FE_OPT_MIXED_WARM_START 10 /* FE_PREC_MIXED residual solves start from
                                      x0 = A'b like the reference (1, default)
                                      or from x0 = 0 (0) */
#define FE_OPT_GRAPH 11      /* 1 (default): replay the LSMR iterations between host
                                convergence checks from a captured CUDA graph */
#define FE_OPT_ROWSUM_VARIANT 12 /* row-sum pass: -1 default, 0 rows staged in shared
                                    memory (cp.async ring), 1 rows in registers */
#define FE_OPT_ABSORB 14     /* 1 (default): FE_PREC_MIXED residual solves (tiles of
                                every width) of single-problem plans with 2+ FEs, and of
                                batch plans whose problems all hold the primary FE and
                                another (tiles narrower than 32 columns), project the
                                primary FE out of the least-squares problem and run LSMR
                                over the other FEs' levels (same residuals, fewer and
                                cheaper iterations); 0: LSMR over all FEs */
#define FE_OPT_FUSED_DEMEAN 15 /* 1 (default): the absorbed loop computes and projects
                                  the rows in one kernel; 0: expand, then demean */
#define FE_OPT_ABSORB_SCALE 16 /* 1 (default): the absorbed LSMR scales the other FEs'
                                  columns by 1 / ||M a_l|| (their norms after the
                                  projection); 0: by the Jacobi scale 1 / ||a_l|| */
#define FE_OPT_EXDM_PIPE 17  /* absorbed loop kernel: the pipelined fused kernel (the
                                next item's rows and gathered coefficient rows staged
                                by asynchronous copies) where the plan fits it (at most
                                one gathered non-primary FE, staging within the
                                shared-memory limit): -1 (default) the first
                                configuration that fits, 1 small-FE sums in one table
                                per lane group, 2 one table per warp, 3 one table per
                                warp in CTAs of 4 warps, three per SM (measured on 10M
                                rows x 32 columns: 846, 1075 and 910 us per launch);
                                0: the unpipelined kernel */

#define FE_OPT_FIRM_ATOMIC 18 /* absorbed loop with one gathered non-primary FE (the pipelined
                                 kernel, configuration 1) whose levels have at most 1024
                                 positions each: 0 (default) the deterministic level-order
                                 segmented sum; 1: its level sums A'u added by vector
                                 reductions (red.global.add) inside the fused kernel, not
                                 bitwise reproducible; -1: both ways timed once per plan
                                 shape (one iteration's kernels) and the faster kept (tuning
                                 cache kind 300).  FEs with larger levels always take the
                                 segmented sum.  Measured on 10M rows x 32 columns: faster
                                 per iteration on a uniform FE, slower per solve (the FP32
                                 sums in no fixed order cost iterations). */
#define FE_OPT_FUSED_RESID 19 /* absorbed FE_PREC_MIXED residual solves, refinement rounds
                                 after the first: the FP64 residual b - A_r x and its
                                 projection in one pass over the rows.  -1 (default): 2
                                 where the plan has at most 4 FEs, else 0; 2: the
                                 projection kernel gathers the other FEs' pre-scaled
                                 FP64 rows itself (the same sums as 0); 1: the staged
                                 fused kernel (measured slower: it holds one CTA per
                                 SM); 0: the residual kernel, then the projection */

typedef struct fe_plan fe_plan;

/* Library version (FE_B200_VERSION). */
int fe_version(void);

/* Message of the last failed call on this thread ("" if none). */
const char* fe_last_error(void);

/*
 * Groups observation keys into fixed-effect level ids on `device`: the
 * GroupedArray compaction behind FixedEffect(keys...) (src/FixedEffect.jl:18-21).
 * keys[j] holds n int64 keys (host memory); refs_out[i] (host, n values)
 * becomes the 1-based rank of observation i's key tuple among the distinct
 * tuples in lexicographic ascending order, and *n_levels_out the number of
 * distinct tuples.  Dense key ranges use presence flags and a prefix sum,
 * others a radix sort.
 */
int fe_group_keys(const int64_t* const* keys, int32_t n_keys, int64_t n, int32_t device,
                  int64_t* refs_out, int64_t* n_levels_out);

/*
 * Builds a solver plan on `device`: uploads the refs, validates them, builds
 * the integer plan on the GPU (stable radix sorts by level, the same order as
 * stable counting sorts), and computes the Jacobi preconditioner on the GPU.
 * Replaces AbstractFixedEffectSolver{T}(fes, w, Val{:CUDA})
 * (ext/CUDAExt.jl:99-110) and its update_weights! (ext/CUDAExt.jl:112-121);
 * CPU counterpart src/SolverCPU.jl:55-95.
 *   refs[k]        n_obs level ids in 1..n_levels[k]
 *   interaction[k] n_obs values or NULL; `interaction` itself may be NULL
 *   weights        n_obs non-negative weights or NULL
 */
int fe_plan_create(fe_plan** out, int64_t n_obs, int32_t n_fe, const int64_t* const* refs,
                   const int64_t* n_levels, const double* const* interaction,
                   const double* weights, int32_t device);

/*
 * A plan over many independent problems solved together (one batched LSMR
 * with per-problem scalars and stopping tests).  Observations of all problems
 * are concatenated (problem p has n_obs[p] rows); refs[k] holds the
 * problem-local 1-based level ids, and n_levels is [n_problems][n_fe].  A
 * problem without FE k has n_levels[p*n_fe+k] == 0 and refs entries 0.
 * No reference counterpart as a single call: it batches many
 * AbstractFixedEffectSolver objects (ext/CUDAExt.jl:99-110).
 */
int fe_plan_create_batch(fe_plan** out, int32_t n_problems, const int64_t* n_obs, int32_t n_fe,
                         const int64_t* const* refs, const int64_t* n_levels,
                         const double* const* interaction, const double* weights,
                         int32_t device);

/*
 * Observation sharding of one problem over several GPUs (one process per GPU).
 *
 * fe_exchange_fn: replaces the `count` elements at `buf` (device memory of
 * the plan's device; dtype FE_XCHG_F64 or FE_XCHG_F32) with their elementwise
 * sum over all ranks, ordered on `stream` (a cudaStream_t; completing the sum
 * before returning also satisfies the ordering).  Returns 0 on success; a
 * non-zero return fails the library call with FE_ERR_CUDA.  Every rank's
 * plan calls it the same number of times in the same order with the same
 * counts, as long as every rank makes the same library calls with the same
 * column counts, tolerances and options.
 *
 * fe_plan_create_sharded builds the plan of one rank's share of the
 * observations of a single problem.  refs hold GLOBAL 1-based level ids and
 * n_levels the GLOBAL level counts (the same on every rank); the share must
 * hold whole levels of the primary FE (the FE with the most levels, the
 * first of them on ties), so no primary level has observations on two
 * ranks, and at least one observation.  The preconditioner (Jacobi scales
 * src/SolverCPU.jl:78-89, and the absorbed-mode column norms) is computed
 * from sums exchanged over the ranks.  Every solve then runs LSMR over the
 * global problem: each iteration exchanges the per-column norms of the local
 * rows and the per-level sums A'u of the local rows (the step between the
 * two matrix-vector products of src/utils/lsmr.jl:104-109); the
 * coefficient-side vectors are replicated and stay bitwise identical on
 * every rank, because the exchanged sums are.  Residuals are returned for
 * the rank's own observations; fe_solve_coefficients returns the same global
 * coefficients on every rank (fe_normalize_coefficients, whose connected
 * components span all ranks' observations, refuses a sharded plan).  Graph replay is off for sharded plans (the
 * exchange runs between kernel launches).  No counterpart in the reference,
 * which solves on one device (ext/CUDAExt.jl:99-165).
 */
typedef int (*fe_exchange_fn)(void* ctx, void* buf, int64_t count, int32_t dtype, void* stream);
#define FE_XCHG_F64 0
#define FE_XCHG_F32 1
int fe_plan_create_sharded(fe_plan** out, int64_t n_obs, int32_t n_fe, const int64_t* const* refs,
                           const int64_t* n_levels, const double* const* interaction,
                           const double* weights, int32_t device, fe_exchange_fn exchange,
                           void* ctx);

/* update_weights!(feM, w): src/SolverCPU.jl:67-76, ext/CUDAExt.jl:112-121. */
int fe_plan_update_weights(fe_plan* plan, const double* weights);

/* Runs the plan's work on a caller stream (a cudaStream_t passed as void*);
 * NULL restores the plan's own stream. */
int fe_plan_set_stream(fe_plan* plan, void* stream);

/* Sets an FE_OPT_* option. */
int fe_plan_set_option(fe_plan* plan, int32_t option, double value);

/* Frees the plan and all its device memory. */
int fe_plan_destroy(fe_plan* plan);

/*
 * solve_residuals!(Y, feM; tol, maxiter) for every column of Y, in place
 * (host memory).  Replaces src/AbstractFixedEffectSolver.jl:49-68 and the
 * column loop of :74-97 (columns are batched, up to 32 per LSMR tile).
 * iterations[j] = LSMR iterations + 1 (the reference's ch.mvps + 1);
 * converged[j] = the reference's ch.isconverged (FE_PREC_MIXED: the FP64
 * tests passed).  With several problems a column reports the maximum
 * iterations and the conjunction of convergence flags over problems
 * (fe_plan_problem_results gives them per problem).
 * Host transfers: with pinned (page-locked) columns the uploads and downloads
 * of each 32-column tile overlap the solves of the other tiles; pageable
 * columns are copied tile by tile.
 */
int fe_solve_residuals(fe_plan* plan, void* Y, int32_t dtype, int64_t ncols, int64_t ld,
                       int32_t precision, double tol, int64_t maxiter, int64_t* iterations,
                       uint8_t* converged);

/* As fe_solve_residuals with Y in device memory (no host copies). */
int fe_solve_residuals_device(fe_plan* plan, void* Y_dev, int32_t dtype, int64_t ncols,
                              int64_t ld, int32_t precision, double tol, int64_t maxiter,
                              int64_t* iterations, uint8_t* converged);

/*
 * solve_residuals!(xs::AbstractVector{<:AbstractVector}, feM; tol, maxiter)
 * (src/AbstractFixedEffectSolver.jl:74-97), the collection form that
 * FixedEffectModels.jl calls: columns[j] is a separate host vector of n_obs
 * values, solved in place.  The columns are batched like the columns of a
 * matrix (fe_solve_residuals), with no host-side gathering into one matrix;
 * results as fe_solve_residuals.
 */
int fe_solve_residuals_columns(fe_plan* plan, void* const* columns, int32_t dtype, int64_t ncols,
                               int32_t precision, double tol, int64_t maxiter,
                               int64_t* iterations, uint8_t* converged);

/*
 * solve_coefficients!(y, feM; tol, maxiter) up to, not including, the
 * normalisation: LSMR from x = 0 (src/AbstractFixedEffectSolver.jl:147-157)
 * and coefs[k][l] = x_k[l] * scale_k[l] for l < n_levels[k] (host memory).
 * normalize!/full (src/FixedEffect.jl:106-140) follow as
 * fe_normalize_coefficients and fe_full_coefficients.
 * iterations = div(ch.mvps, 2) as the reference returns.
 */
int fe_solve_coefficients(fe_plan* plan, const void* y, int32_t dtype, int32_t precision,
                          double tol, int64_t maxiter, double* const* coefs,
                          int64_t* iterations, uint8_t* converged);

/* normalize!(fecoefs, fes) (src/FixedEffect.jl:106-135) on the device: within
 * each connected component of the observation/level graph of the FEs without
 * an interaction, every such FE but the first is demeaned and the means are
 * added to the first.  coefs[k]: n_levels[k] doubles in host memory
 * (coefs_on_device = 0) or device memory, normalized in place; interacted FEs
 * are left as they are.  Deterministic (exact fixed-point component sums). */
int fe_normalize_coefficients(fe_plan* plan, double* const* coefs, int32_t coefs_on_device);

/* full(fecoefs, fes) (src/FixedEffect.jl:137-140): out[k][i] =
 * coefs[k][refs_k[i]] for every observation i, in the caller's order (N
 * doubles per FE); host or device memory on either side. */
int fe_full_coefficients(fe_plan* plan, const double* const* coefs, int32_t coefs_on_device,
                         double* const* out, int32_t out_on_device);

/* Per-problem iterations/convergence of the last solve: [n_problems][ncols]. */
int fe_plan_problem_results(fe_plan* plan, int64_t* iterations, uint8_t* converged);

/* Diagnostics of the last solve per column: the FP64 test2 of the last
 * refinement round, the number of rounds, and the raw LSMR iteration count. */
int fe_plan_last_solve_info(fe_plan* plan, int64_t ncols, double* test2, int32_t* rounds,
                            int64_t* lsmr_iters);

/*
 * The integer plan, for bit-exact checks against the stable counting sort of
 * ext/MetalExt.jl:40-64 (bucketize_refs):
 *   perm0[p]      original observation (0-based) at sorted position p
 *   offsets[k]    n_levels[k]+1 level offsets into FE k's level order
 *   segperm[k][q] sorted position of entry q of FE k's level order
 * For a batch plan the observations are sorted problem by problem (each by
 * its primary level; a problem without the primary FE keeps its order),
 * n_levels[k] is the total over problems, levels are numbered problem after
 * problem, and FE k's level order leaves out the problems without FE k.
 * Any output pointer may be NULL.
 */
int fe_plan_get_integer_plan(fe_plan* plan, int32_t* perm0, int64_t* const* offsets,
                             int32_t* const* segperm);

/* Jacobi scales scale_k (src/SolverCPU.jl:78-89), n_levels[k] values per FE. */
int fe_plan_get_scales(fe_plan* plan, double* const* scales);

/* Index of the FE whose levels order the observations. */
int fe_plan_primary(fe_plan* plan, int32_t* primary);

/* Launch statistics collected with FE_OPT_PROFILE: kernel `index`'s name,
 * launches, total CUDA-event milliseconds and algorithmic bytes.  Returns
 * FE_ERR_INVALID past the last kernel. */
int fe_plan_kernel_stat(fe_plan* plan, int32_t index, char* name, int64_t name_len,
                        int64_t* launches, double* total_ms, double* alg_bytes);
/* The CUDA-event milliseconds of each launch of kernel `index` (FE_OPT_PROFILE),
 * in launch order: up to max_launches values into ms, the count in *launches.
 * Launches that found every instance stopped return at once, so the typical
 * working launch is read off this list rather than the mean. */
int fe_plan_kernel_times(fe_plan* plan, int32_t index, float* ms, int64_t max_launches,
                         int64_t* launches);
int fe_plan_reset_stats(fe_plan* plan);

/*
 * fe_plan_scales_noalloc -- no counterpart in the reference.
 *
 * Recomputes the Jacobi scales of fixed effect `fe_index` of an existing plan
 * (the values fe_plan_get_scales returns, src/SolverCPU.jl:78-89) into
 * `scale_out_dev`, n_levels[fe_index] doubles of DEVICE memory, enqueued on
 * `stream` (NULL: the plan's stream), without allocating any device memory.
 * It is for callers that cannot call cudaMalloc at that point, because the
 * device heap is not theirs to grow: a caller whose device memory belongs to
 * its own pool or runtime (Julia's CUDA.jl allocator hands out memory from a
 * pool it owns, so a cudaMalloc behind its back can fail once the pool holds
 * the free memory), or one that runs under a fixed device-memory budget.
 *
 * Its scratch is one file-scope device array of FE_NOALLOC_SCRATCH_BYTES
 * (8 MiB) that every GPU which loads the library holds until the process
 * exits.  It holds the fixed effect's level sums (about 1e6 levels at most)
 * and the piece partials of the plan's long levels; a fixed effect that does
 * not fit is rejected with FE_ERR_INVALID and a message.  The array's device
 * address is looked up (cudaGetSymbolAddress) with the plan's device current
 * on every call; the first call on a device may also load the library's
 * device code, so make that first call before any stream capture.  All calls
 * share the array and it keeps the last call's contents (each call clears
 * what must start at zero): calls that overlap on the GPU race and must be
 * serialized by the caller.  A caller stream is ordered after the work
 * already queued on the plan's stream (an event recorded there); the caller
 * orders any later use of the output itself.
 */
#define FE_NOALLOC_SCRATCH_BYTES (8u << 20)
int fe_plan_scales_noalloc(fe_plan* plan, int32_t fe_index, double* scale_out_dev, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* FE_B200_H */
