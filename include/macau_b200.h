/* macau_b200.h -- C ABI of the sm_100a Gibbs-sweep library for BPMF / Macau.
 *
 * The library replaces the hot path of jaak-s/macau 0.5.3 (one Gibbs sweep of MacauX::run,
 * lib/macau-cpp/macau.cpp:110-147): the per-row latent sampler (sample_latent_blas,
 * latentprior.cpp:361-385), the Normal-Wishart hyperprior update (CondNormalWishart,
 * mvnormal.cpp:314-336) and, for side information, the block-CG solve of the link matrix
 * (solve_blockcg, linop.h:207-343).  The reference has no C ABI; each entry below names the
 * C++ member or Cython function it stands in for.
 *
 * Conventions
 *   - Matrices are column-major like the reference's Eigen storage: a latent matrix is K x N
 *     (column n = the K-vector of entity n), Lambda is K x K, beta is K x nfeat.
 *   - Every entry point returns 0 on success or a negative MG_ERR_* code; mg_last_error()
 *     gives the message.  Entry points never throw and are not thread-safe per context.
 *   - All device work of one context runs on one CUDA stream owned by the context; calls are
 *     synchronous from the caller's point of view unless stated otherwise.
 *   - Random draws are keyed (seed, sweep, mode, purpose, index) through Philox-4x32-10, so a
 *     run is reproducible for a given seed.
 */
#ifndef MACAU_B200_H
#define MACAU_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Error codes (negative) */
#define MG_OK 0
#define MG_ERR_ARG (-1)        /* invalid argument (reference: ValueError / runtime_error) */
#define MG_ERR_CHOL (-2)       /* "Cholesky Decomposition failed!" (latentprior.cpp:374-376) */
#define MG_ERR_CG (-3)         /* block-CG breakdown, or a solve that reached its iteration cap
                                  without converging (the reference stops silently, linop.h:279) */
#define MG_ERR_CUDA (-4)       /* CUDA runtime error */
#define MG_ERR_STATE (-5)      /* call out of order (e.g. sweep before data) */
#define MG_ERR_TIMEOUT (-6)    /* a bounded device-side wait gave up */
#define MG_ERR_NOGPU (-7)      /* no sm_100 device */

/* Arithmetic of the sampler. */
#define MG_COMPUTE_FP64 0      /* everything in FP64 (parity with the FP64 oracle <= 1e-9) */
#define MG_COMPUTE_MIXED 1     /* BF16 Gram / FP32 accumulate, FP32 Cholesky + FP64 retry,
                                  FP32 block-CG with FP64 residual replacement; FP64 hyperprior */

typedef struct mg_ctx mg_ctx;

typedef struct mg_config {
  int num_latent;     /* K: Macau::num_latent (macau.h:13) */
  double precision;   /* alpha of FixedGaussianNoise (noisemodels.h:32-39) */
  uint64_t seed;      /* key of every random draw */
  int compute;        /* MG_COMPUTE_FP64 or MG_COMPUTE_MIXED */
  int verbose;        /* print one status line per iteration like MacauX::printStatus */
  int device;         /* CUDA device ordinal */
} mg_config;

typedef struct mg_stats {
  double sweeps;            /* sweeps run since mg_init */
  double seconds_sample;    /* device time in the latent samplers (CUDA events) */
  double seconds_prior;     /* device time in the hyperprior / beta updates */
  double seconds_eval;      /* device time in test evaluation */
  int64_t retries[2];       /* mixed mode: rows re-factorised in FP64, per mode (cumulative) */
  int64_t rows_sampled[2];  /* rows sampled, per mode (cumulative) */
  int cg_iters[2];          /* block-CG iterations of the last beta update, per mode */
  int graph_captured;       /* 1 when sweeps replay a captured CUDA graph */
  int64_t kernel_launches;  /* kernels launched by sweeps / phases since mg_init */
  int64_t h2d_bytes;        /* host->device bytes copied by the library (process total) */
  int64_t d2h_bytes;        /* device->host bytes copied by the library (process total) */
  int64_t ntasks[2];        /* latent-sampler work items per mode (rows + split parts) */
  int64_t nnz[2];           /* training entries per mode after duplicate summing */
} mg_stats;

/* Context lifetime.  Replaces `make_macau_fixed(2, K, precision)` (macau.cpp:214-220) plus
 * MacauX construction on a 2-mode matrix; mg_set_noise_adaptive switches the noise model to
 * AdaptiveGaussianNoise. */
int mg_create(mg_ctx** out, const mg_config* cfg);
void mg_destroy(mg_ctx* ctx);
const char* mg_last_error(const mg_ctx* ctx);

/* Macau::setRelationData(int* idx, int nmodes, double* values, int nnz, int* dims)
 * (macau.h:39; MatrixData::setTrain, sparsetensor.cpp:92-106).  idx is nnz x nmodes
 * column-major (row indices, then column indices); nmodes must be 2.  Duplicate (i, j) entries
 * are summed like Eigen's setFromTriplets.  The arrays are copied; host buffers may be freed
 * afterwards. */
int mg_set_relation_data(mg_ctx* ctx, const int32_t* idx, int nmodes, const double* values,
                         int64_t nnz, const int32_t* dims);

/* Macau::setRelationDataTest(...) (macau.h:40; MatrixData::setTest, sparsetensor.cpp:108-117). */
int mg_set_relation_data_test(mg_ctx* ctx, const int32_t* idx, int nmodes,
                              const double* values, int64_t nnz, const int32_t* dims);

/* Macau::setRelationData(int* rows, int* cols, double* values, int N, int nrows, int ncols)
 * (macau.h:37; MatrixData::setTrain, sparsetensor.cpp:78-85) and its test-set twin
 * (macau.h:38; sparsetensor.cpp:87-90): the same data as the idx forms above, with the row and
 * the column indices in two arrays, so a caller holding them apart needs no nnz x 2 copy. */
int mg_set_relation_data_rc(mg_ctx* ctx, const int32_t* rows, const int32_t* cols,
                            const double* values, int64_t nnz, int nrows, int ncols);
int mg_set_relation_data_test_rc(mg_ctx* ctx, const int32_t* rows, const int32_t* cols,
                                 const double* values, int64_t nnz, int nrows, int ncols);

/* Side information for `mode` (MacauPrior<SparseDoubleFeat>, latentprior.h:82-125, built by
 * make_prior, macau.pyx:154-192): F is nrows x nfeat given as COO; vals == NULL means a binary
 * matrix (all ones).  lambda_beta / tol are MacauPrior::setLambdaBeta / setTol.  Without this
 * call the mode uses the BPMF prior (BPMFPrior, latentprior.h:53-79). */
int mg_set_side(mg_ctx* ctx, int mode, const int32_t* rows, const int32_t* cols,
                const double* vals, int64_t nnz, int nrows, int nfeat, double lambda_beta,
                double tol);

/* Univariate side-information prior for `mode`: replaces `make_one_prior` (macau.pyx:194-214,
 * used by macau(univariate=True)) -> MacauOnePrior<SparseFeat | SparseDoubleFeat>(K, F) +
 * setLambdaBeta (macauoneprior.cpp:16-39, macauoneprior.h:47).  F is nrows x nfeat COO; vals ==
 * NULL means binary.  Each sweep then redraws the mode's latents one coordinate at a time
 * (macauoneprior.cpp:41-95) and its prior with sample_mu_lambda / sample_beta / compute_uhat /
 * sample_lambda_beta (macauoneprior.cpp:189-290).  mg_get_hyper reports the mean of the K
 * lambda_beta values, like getLinkLambda (macauoneprior.h:46). */
int mg_set_side_univariate(mg_ctx* ctx, int mode, const int32_t* rows, const int32_t* cols,
                           const double* vals, int64_t nnz, int nrows, int nfeat,
                           double lambda_beta);

/* The K per-dimension lambda_beta values of a univariate prior (MacauOnePrior::lambda_beta). */
int mg_get_lambda_beta_univariate(mg_ctx* ctx, int mode, double* out);

/* Macau::setSamples (macau.h:36). */
int mg_set_samples(mg_ctx* ctx, int burnin, int nsamples);

/* MacauX::init (macau.cpp:72-86): latents to zero, priors to their initial hyperparameters
 * (BPMFPrior::init / MacauPrior::init, latentprior.cpp:84-99, 181-216). */
int mg_init(mg_ctx* ctx);

/* One iteration `iter` of MacauX::run (macau.cpp:110-147): sample mode 0, sample mode 1,
 * update prior 0, update prior 1, evaluate the test set with n = iter < burnin ? 0 : iter-burnin
 * (when eval != 0).  Replays a captured CUDA graph when the sweep has no host-side decision. */
int mg_sweep(mg_ctx* ctx, int iter, int eval);

/* `count` consecutive sweeps starting at `first_iter` without returning to the caller in
 * between (no per-sweep host synchronisation). */
int mg_sweeps(mg_ctx* ctx, int first_iter, int count, int eval);

/* Device time of `count` sweeps starting at `first_iter`, measured with CUDA events on the
 * context's stream (benchmark support; no reference counterpart).  With phase_events = 0 the
 * sweeps run as they would in mg_sweeps (captured graph when possible) and *total_seconds
 * receives the elapsed time; with phase_events = 1 they run un-captured with events between
 * phases and phase_seconds[0..6] receives the summed time of sample mode 0, sample mode 1,
 * update prior 0, update prior 1, evaluation, then the Gram kernel of the tensor-core sampler
 * alone in mode 0 and mode 1 (0 when that sampler is not used). */
int mg_time_sweeps(mg_ctx* ctx, int first_iter, int count, int eval, int phase_events,
                   double* total_seconds, double* phase_seconds);

/* MacauX::run (macau.cpp:94-148): mg_init, then burnin + nsamples sweeps with evaluation. */
int mg_run(mg_ctx* ctx);

/* Phase-level entry points (used by parity tests and by hosts that drive the loop):
 * ILatentPrior::sample_latents for one mode (latentprior.cpp:30-37, 69-77, 219-227) and
 * ILatentPrior::update_prior (latentprior.cpp:79-81, 255-264), with the draws of sweep `iter`.
 * `z` optionally injects the K x N standard normals of the row sampler (NULL = keyed draws). */
int mg_sample_latents(mg_ctx* ctx, int mode, int iter, const double* z);
int mg_update_prior(mg_ctx* ctx, int mode, int iter);

/* Adaptive Gaussian noise in place of the fixed precision of mg_config: replaces
 * `make_macau_adaptive(2, K, sn_init, sn_max)` (macau.cpp:222-228, called by macau.pyx:391-392
 * with sn_init = 1 for precision="adaptive").  AdaptiveGaussianNoise::init
 * (noisemodels.cpp:14-33) at mg_init: var_total = mean squared deviation of the training values
 * from their mean (1 when not positive or NaN), alpha = (sn_init + 1) / var_total, cap
 * alpha_max = (sn_max + 1) / var_total.  Each sweep then redraws alpha after the priors
 * (AdaptiveGaussianNoise::update, noisemodels.cpp:55-81).  Call before mg_init; it undoes a
 * previous mg_init. */
int mg_set_noise_adaptive(mg_ctx* ctx, double sn_init, double sn_max);

/* AdaptiveGaussianNoise::update (noisemodels.cpp:55-81) with the draw of sweep `iter`: alpha ~
 * Gamma(1/2 + nnz/2, rate var_total/2 + SSE/2) capped at alpha_max, SSE the squared training
 * residuals under the current latents.  A no-op under fixed noise. */
int mg_update_noise(mg_ctx* ctx, int iter);

/* out[0] = current noise precision alpha, out[1] = alpha_max (the fixed precision under fixed
 * noise), out[2] = var_total of the training values. */
int mg_get_noise(mg_ctx* ctx, double* out);

/* FixedGaussianNoise::evalModel -> eval_rmse (noisemodels.cpp:161-166, bpmfutils.h:86-114). */
int mg_eval(mg_ctx* ctx, int n);

/* State access (K x N column-major latents; K x K Lambda; K mu; K x nfeat beta; K x N Uhat). */
int mg_get_latents(mg_ctx* ctx, int mode, double* out);
int mg_set_latents(mg_ctx* ctx, int mode, const double* in);
int mg_get_hyper(mg_ctx* ctx, int mode, double* mu, double* Lambda, double* lambda_beta);
int mg_set_hyper(mg_ctx* ctx, int mode, const double* mu, const double* Lambda,
                 const double* lambda_beta);
int mg_get_beta(mg_ctx* ctx, int mode, double* beta);
int mg_get_uhat(mg_ctx* ctx, int mode, double* uhat);
int mg_get_dims(mg_ctx* ctx, int64_t* nrow, int64_t* ncol, int64_t* ntrain, int64_t* ntest,
                double* mean_value);

/* ---- Row-sharded chains over several GPUs (no reference counterpart; the reference's own
 * distributed form is the MPI split of block-CG's right-hand sides, macau_mpi.cpp:380-397).
 * Within a half-sweep the rows of a mode are independent given the other mode's latents and
 * the hyperparameters, so each rank's context samples a contiguous row range and the ranks
 * exchange the new rows (an all-gather into every rank's latent buffer) before the next
 * half-sweep.  Every rank then holds the same latents, and mg_update_prior computes the same
 * hyperparameters on each rank from them (same data, same kernels, same keyed draws): the
 * N-rank chain is the 1-rank chain.  Draws are keyed by the global row index.
 *   mg_set_row_range   rows [lo, hi) of `mode` sampled by this context (after the training
 *                      data; the split of long rows keeps the whole mode's threshold)
 *   mg_latents_device  device buffer of the mode's latents as the samplers write them: rows of
 *                      *row_stride values of *elem_bytes bytes (8: FP64 mode, 4: the FP32 master
 *                      of mixed mode), for the caller's collective
 *   mg_latents_changed after rows of that buffer were written from outside: refreshes the
 *                      samplers' derived copy (mixed mode: the 16-bit gather copy), on the
 *                      context's stream
 *   mg_get_stream      the context's CUDA stream (cudaStream_t), to order collectives with the
 *                      context's kernels */
int mg_set_row_range(mg_ctx* ctx, int mode, int64_t lo, int64_t hi);
int mg_latents_device(mg_ctx* ctx, int mode, void** ptr, int* row_stride, int* elem_bytes);
int mg_latents_changed(mg_ctx* ctx, int mode);
int mg_get_stream(mg_ctx* ctx, void** stream);

/* Results: Macau::getRmseTest / getPredictions / getStds / getTestData (macau.h:45-51,
 * macau.cpp:174-188).  rmse[0] = posterior-mean RMSE, rmse[1] = last single-sample RMSE.
 * Test data rows are (row, col, value) in the CSC order of the test matrix, ntest x 3
 * column-major like MatrixData::getTestData (sparsetensor.cpp:63-76). */
int mg_get_rmse(mg_ctx* ctx, double* rmse);
int mg_get_predictions(mg_ctx* ctx, double* out);
int mg_get_stds(mg_ctx* ctx, double* out);
int mg_get_test_data(mg_ctx* ctx, double* out);
int mg_get_stats(mg_ctx* ctx, mg_stats* out);

/* ---- Many independent BPMF chains in one set of launches ----
 * P problems, each what `macau.bpmf(Y_p, Ytest_p, num_latent=K_p, precision=precision)` runs
 * (MacauX with two BPMF priors, macau.cpp:110-147, latentprior.cpp:69-99), sampled together in
 * mixed precision (BF16 tensor-core Grams, FP32 Cholesky with FP64 retry, FP64 hyperpriors):
 * each sweep is one captured CUDA graph with one Gram launch and one finish launch per mode for
 * all problems.  Problem p uses seed seeds[p] and its local row / column indices for its keyed
 * draws, so its chain draws what a single context with that seed draws.  K_p <= 32.  The
 * reference has no batched form; it runs one Macau object per problem. */
typedef struct mg_batch mg_batch;
int mg_batch_create(mg_batch** out, int nprob, const int32_t* nrows, const int32_t* ncols,
                    const int32_t* num_latent, const uint64_t* seeds, double precision,
                    int device);
void mg_batch_destroy(mg_batch* b);
const char* mg_batch_last_error(const mg_batch* b);
/* Problem p's train entries are rows / cols / vals[train_off[p] .. train_off[p + 1]) in its own
 * indices (duplicates summed), its test entries trows / tcols / tvals[test_off[p] ..
 * test_off[p + 1]). */
int mg_batch_set_data(mg_batch* b, const int64_t* train_off, const int32_t* rows,
                      const int32_t* cols, const double* vals, const int64_t* test_off,
                      const int32_t* trows, const int32_t* tcols, const double* tvals);
/* MacauX::init for every problem (latents zero, mu = 0, Lambda = 10 I); evaluation averages the
 * sweeps from `burnin` on. */
int mg_batch_init(mg_batch* b, int burnin);
int mg_batch_sweeps(mg_batch* b, int first_iter, int count, int eval);
/* Device time of `count` sweeps without evaluation (CUDA events on the batch's stream). */
int mg_batch_time_sweeps(mg_batch* b, int first_iter, int count, double* seconds);
/* Problem `prob`'s latents of `mode` (nrows_p x K_p row-major, i.e. K_p x N column-major). */
int mg_batch_get_latents(mg_batch* b, int prob, int mode, double* out);
/* out[2 p] = posterior-mean test RMSE of problem p, out[2 p + 1] = single-sample RMSE. */
int mg_batch_get_rmse(mg_batch* b, double* out);
/* out[0..4] = total rows, total columns, total train entries, FP64 retries in mode 0 and 1. */
int mg_batch_get_info(mg_batch* b, int64_t* out);

/* Switches of the implementation (no reference counterpart):
 *   "graph"            (default 1) replay captured CUDA graphs for sweeps without host-side
 *                      decisions
 *   "tensor_core_gram" (default 1) mixed mode: run the K = 32 row Grams on the tcgen05 tensor
 *                      cores
 *   "fused_finish"     (default 1) the tensor-core sampler finishes each row (factor, solves,
 *                      draw) in its Gram kernel's epilogue; 0 = Gram records in HBM and a
 *                      separate finish kernel (the same arithmetic; an FP32 factor that fails
 *                      is redone in FP64 from the CSR when fused, from the record otherwise)
 *   "tc_wait_us"       (default 0 = about 2 s) budget of each barrier wait of the tensor-core
 *                      sampler in microseconds; a wait that runs out ends the launch with
 *                      MG_ERR_TIMEOUT and leaves the context usable after mg_init
 *   "tc_wait_test"     (default 0; tests only) 1 = the tensor-core sampler's MMA warp first
 *                      waits on a barrier that nothing arrives on, so that wait runs out
 *   "cg_max_iter"      (default 100000, the reference's cap, linop.h:279) iterations of each
 *                      block-CG solve; a solve that reaches the cap keeps its last iterate, the
 *                      update completes, and the call returns MG_ERR_CG ("block-CG did not
 *                      converge within N iterations")
 *   "cg_fp32"          (default 0) mixed mode: run the Macau block-CG in FP32 with an FP64
 *                      residual replacement every 20 iterations instead of FP64; set before
 *                      mg_init
 *   "gram_precision"   (default 0) mixed mode: inputs of the row Grams, 0 = BF16, 1 = FP16,
 *                      2 = TF32 (the FP32 latents rounded to TF32 as they are gathered); FP32
 *                      accumulation, factor and solves in every case.  1 and 2 use the CUDA-core
 *                      sampler at every K.  Set before mg_init (it undoes a previous mg_init).
 *   "autotune"         (default 0) run mg_autotune at the end of mg_init: 1 with the choice
 *                      cache (set before mg_set_relation_data, a cached choice also shapes
 *                      the task lists built there), 2 always timing the candidates
 *   "split_threshold"  the row samplers' work split for both modes, in [256, 16384] entries
 *                      (default nnz / (32 * SMs) clamped to that range); after the training data
 *   "cta_groups"       row groups per CTA of the CUDA-core sampler (0 = default; 4 or 2 at
 *                      K <= 32, 2 or 1 at K = 64, FP64 or BF16 Grams)
 *   "group_mix"        (default 16) order of the tensor-core sampler's row groups (four rows
 *                      each) in its work queue: 0 = by descending length; n in [1, 64] = long
 *                      and short groups interleaved, a finished row weighed as n k-blocks of
 *                      gathers, so that each CTA meets both at once.  Changes no result. */
int mg_set_option(mg_ctx* ctx, const char* name, int value);

/* ---- Autotuner of the row samplers (no reference counterpart; the reference's OpenMP
 * `schedule(dynamic, 2)` row loop, latentprior.cpp:73, has no shape to tune) ----
 * For each mode, times every candidate work split of the row sampler (rows longer than the
 * split threshold are cut into parts; thresholds nnz / (d * 16 * SMs), d = 1, 2, 4, 8, 16,
 * clamped to [256, 16384] entries) and, for the CUDA-core sampler, its CTA shapes, as half-sweeps
 * on the current state, and keeps the fastest.  Latents, hyperparameters and counters are
 * restored, so the chain continues as if untuned (only split rows' summation order can change).
 * Choices are cached per process, and in the file named by MACAU_B200_TUNE_CACHE if set, by
 * (sampler, K, SM count, the rows' log2 length histogram); use_cache = 0 always re-times.
 * Call after mg_init. */
int mg_autotune(mg_ctx* ctx, int use_cache);

typedef struct mg_tuning {
  int64_t split_threshold; /* entries: longer rows are split into parts */
  int cta_groups;          /* row groups per CTA of the CUDA-core sampler (0: tensor-core) */
  int tensor_core;         /* 1 when the mode's Grams run on the tcgen05 sampler */
  int state;               /* 0 default shape, 1 timed by mg_autotune, 2 taken from the cache */
  int candidates;          /* candidates timed */
  double ms_best;          /* half-sweep time of the choice (ms) */
  double ms_default;       /* half-sweep time of the default shape (ms) */
  int finish_ctas_per_sm;  /* batch: CTAs per SM of the row finish (0 for a context) */
} mg_tuning;
int mg_get_tuning(mg_ctx* ctx, int mode, mg_tuning* out);

/* The same autotuner for the batched sampler (mg_batch): per mode, the split threshold of the
 * Gram task list over every problem's rows and the row finish's CTAs per SM (8, 4 or 16;
 * reported in finish_ctas_per_sm).  Call after mg_batch_init; the chains continue as if
 * untuned. */
int mg_batch_autotune(mg_batch* b, int use_cache);
int mg_batch_get_tuning(mg_batch* b, int mode, mg_tuning* out);

/* macau.blockcg(X, B, reg, tol) (macau.pyx:67-91 -> solve_blockcg, linop.h:229-343) on the GPU:
 * solves (F'F + reg I) X' = B' for nrhs right-hand sides with the reference's 32+8 RHS blocking
 * (linop.h:207-226).  F is nrows x nfeat COO (vals NULL = binary); B and X are nrhs x nfeat
 * column-major.  Unlike the reference wrapper (which drops its solution), X is returned.
 * compute selects FP64 or FP32-with-FP64-residual-replacement.  *niter receives the summed
 * iteration count of the blocks and *seconds the device time. */
int mg_blockcg(const int32_t* rows, const int32_t* cols, const double* vals, int64_t nnz,
               int nrows, int nfeat, const double* B, int nrhs, double reg, double tol,
               int compute, double* X, int* niter, double* seconds);

/* Hyperprior update without device allocation.  No counterpart in the reference: it exists for
 * callers that cannot call cudaMalloc when they resample the Normal-Wishart hyperparameters --
 * a process whose memory pool already owns the device memory, or a loop that cannot take
 * cudaMalloc's implicit synchronisation.  It draws the same (mu, Lambda) as mg_update_prior does
 * for a BPMF prior (the posterior of the latent vectors' mean and precision under the
 * Normal-Wishart prior, then one draw of each), from device inputs into device outputs:
 *   U           N latent vectors of K doubles, vector n at U + n * stride (device)
 *   mu0, T      prior mean (K) and scale matrix (K x K, column-major), device
 *   kappa, nu   prior strength (> 0) and degrees of freedom (>= K); a BPMF prior uses 2 and K
 *   seed, sweep, mode  key of the Wishart / mean draws (same keys as mg_update_prior)
 *   mu_out, Lambda_out device outputs (K and K x K); stream: cudaStream_t (NULL = default)
 *   err / errlen optional caller buffer for a message (NULL allowed)
 * Its scratch is one fixed 2.3 MB array in the library (every GPU that loads the library holds
 * it until exit), so K is limited to 64; larger K, nu < K or kappa <= 0 return MG_ERR_ARG.  All
 * calls share that array and it keeps the last call's contents: calls whose kernels overlap on
 * the GPU race.  The first call in a device's CUDA context looks the array's address up.
 * Synchronous: it reads the status word back and waits for `stream`. */
int mg_normal_wishart_noalloc(const double* U, int64_t N, int K, int stride, const double* mu0,
                              double kappa, const double* T, int nu, uint64_t seed,
                              uint32_t sweep, int mode, double* mu_out, double* Lambda_out,
                              void* stream, char* err, int errlen);

#ifdef __cplusplus
}
#endif
#endif /* MACAU_B200_H */
