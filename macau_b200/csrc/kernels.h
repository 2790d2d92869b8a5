// Host-side launch functions of the sm_100a kernels (one translation unit per kernel family).
#pragma once
#include <cuda_runtime.h>

#include <vector>

#include "common.cuh"

namespace mg {

// ---- data layout construction (build_kernels.cu) ----
// COO (device) -> CSR of the rows and CSR of the columns, indices ascending, duplicates summed
// in input order.  Output arrays hold nnz entries (capacity); returns the unique count.
long long build_csr_pair(const int* d_r, const int* d_c, const double* d_v, long long nnz,
                         long long nrow, long long ncol, long long* row_ptr, int* row_idx,
                         double* row_val, long long* col_ptr, int* col_idx, double* col_val,
                         cudaStream_t s);
// COO (device) -> triplets sorted by (major, minor) with duplicates summed in input order into
// out_major / out_minor / out_val (capacity nnz); returns the unique count.  Both builders throw
// MG_ERR_ARG (`what` for this one) when an index is outside the dimensions.
long long build_coo_sorted(const int* d_major, const int* d_minor, const double* d_v,
                           long long nnz, long long nmajor, long long nminor, const char* what,
                           int* out_major, int* out_minor, double* out_val, cudaStream_t s);
// out[e] = {idx[e], float bits of (val[e] - mean) * alpha}
void launch_pack(const int* idx, const double* val, long long n, double mean, double alpha,
                 uint2* out, cudaStream_t s);
// Row r of `packed` (ptr) copied to pptr[r] and padded to pptr[r + 1] with {sentinel, 0}.
void launch_pad(const long long* ptr, const long long* pptr, long long nrows, const uint2* packed,
                unsigned sentinel, uint2* out, cudaStream_t s);

// ---- latent sampler (sample_kernels.cu, gram_tc.cu) ----
// gram (mixed only): the Gram precision, 0 = BF16 gathers, 1 = FP16 gathers (p.other is the FP16
// copy, p.half_copy set), 2 = TF32 (p.other is the FP32 master copy, rounded as it is read).
// groups: row groups per CTA (0 or any value not offered by sample_group_options: the
// default shape).
void launch_sample(const SampleParams& p, int KP, bool mixed, int gram, cudaStream_t s,
                   int num_sms, int groups = 0);
// The default CTA shape of the CUDA-core sampler at KP, and the shapes the autotuner may pick
// from (the default first).
int sample_default_groups(int KP);
std::vector<int> sample_group_options(int KP, bool mixed, int gram);
// Sum over the n values of (v[i] - center), or of its square when sq, on the device in a fixed
// order; returns it to the host (synchronises the stream).
double value_moment(const double* v, long long n, double center, bool sq, cudaStream_t s);
// dst[i] = src[i] rounded to BF16 (half = false) or FP16 (half = true), n values.
void launch_copy16(const float* src, void* dst, long long n, bool half, cudaStream_t s);
// Mixed-precision sampler whose Grams run on the tcgen05 tensor cores (KP = 32 only).  It reads
// the 16-entry padded packed CSR and its task list (p.packed / p.tasks, built by the context) and
// gathers the other factor's BF16 rows from p.other, whose row nother is all zeros (the padding
// sentinel).  split_rows lists the nsplit rows whose Grams are split into parts, as {row,
// parts, scratch slot of part 0, 0} (their partial Grams go to p.scratch, 1056 doubles per
// slot).
//   fused (and not p.one): k_gram_tc<true> finishes every unsplit row in its epilogue; if
//     nsplit > 0, k_sum_parts writes the split rows' Grams to records 0 .. nsplit - 1 of `gram`
//     and k_finish_tc finishes them.  `gram` needs max(1, nsplit) records.
//   otherwise: k_gram_tc<false> writes every row's Gram record (`gram` holds nrows records of
//     32 * 32 + 32 floats), k_sum_parts the split rows', then k_finish_tc (k_finish_one_tc when
//     p.one) finishes all rows.
// Returns false when the configuration is not covered (caller uses the CUDA-core kernel).
// `mid`, if given, is recorded after k_gram_tc (per-kernel timing).
bool launch_sample_tc(const SampleParams& p, float* gram, const int4* split_rows, int nsplit,
                      int KP, cudaStream_t s, int num_sms, cudaEvent_t mid = nullptr,
                      bool fused = true);
// Doubles of the fused kernel's FP64-redo work area (SampleParams::retry_work) for a grid of
// num_sms CTAs.
size_t tc_retry_work_doubles(int num_sms);
// The Gram half of launch_sample_tc: k_gram_tc (+ k_sum_parts), no finish.  Returns false when
// the configuration is not covered.
bool launch_gram_tc(const SampleParams& p, float* gram, const int4* split_rows, int nsplit,
                    int KP, cudaStream_t s, int num_sms, cudaEvent_t mid = nullptr);

// ---- hyperprior / eval (hyper_kernels.cu) ----
struct NwWork {
  double* vec;  // 3*K
  double* m0;   // K*K each
  double* m1;
  double* m2;
  double* m3;
};
int stats_blocks(long long N);
// Sums `nparts` records of `len` doubles (stats partials) into one record, in a fixed order.
void launch_reduce_parts(const double* parts, int nparts, int len, double* out, cudaStream_t s);
void launch_stats(const void* U, bool f32, const double* Uhat, long long N, int K, int stride,
                  int uhat_stride, double* partials, int nblocks, cudaStream_t s);
void launch_normal_wishart(const double* partials, int nparts, long long N, int K,
                           const double* mu0, double kappa, const double* T0, int nu,
                           const double* bb_partials, int bb_nparts, const double* lambda_beta,
                           const NwWork& w, Ctl* ctl, unsigned long long seed, int mode,
                           double* mu_out, double* Lambda_out, cudaStream_t s);
// Both modes' BPMF prior updates (BPMFPrior::update_prior, latentprior.cpp:79-81) at once, for
// K <= 32: statistics, reduction and Normal-Wishart draw of mode m from the latents U[m]
// (N[m] rows, stride `stride`), partials[m] (nblocks[m] records, rows_per_block[m] rows each)
// and final_[m] as work, into mu[m] / Lambda[m].  Three launches instead of six; each mode's
// blocks compute what launch_stats / launch_reduce_parts / launch_normal_wishart compute, with
// the same keyed draws, so the result is the same bit for bit.
struct PriorPair {
  const void* U[2];
  long long N[2];
  long long rows_per_block[2];
  int nblocks[2];
  double* partials[2];
  double* final_[2];
  const double* mu0[2];
  double kappa[2];
  const double* T0[2];
  int nu[2];
  double* mu[2];
  double* Lambda[2];
};
void launch_prior_pair(const PriorPair& pp, bool f32, int K, int stride, Ctl* ctl,
                       unsigned long long seed, cudaStream_t s);
void launch_lambda_beta(const double* bb_partials, int nparts, int K, long long nfeat,
                        const double* Lambda, double nu, double mu, const Ctl* ctl,
                        unsigned long long seed, int mode, double* lambda_beta, cudaStream_t s);
int eval_blocks(long long ntest);
void launch_eval(const int* trow, const int* tcol, const double* tval, long long ntest,
                 const void* U, const void* V, bool f32, int K, int stride, double mean,
                 int n_fixed, const Ctl* ctl, double* pred, double* pvar, double* partials,
                 int nblocks, double* rmse, cudaStream_t s);
// Row index of every entry of a CSR (nnz entries, nrows rows).
void launch_entry_rows(const long long* ptr, long long nrows, long long nnz, int* erow,
                       cudaStream_t s);
// AdaptiveGaussianNoise::update: squared residuals of the nnz training entries (erow / col /
// val) under the latents U (rows) and V (columns), summed through `partials` (nblocks =
// eval_blocks(nnz) doubles), then the capped Gamma draw of the precision into ctl->alpha.
void launch_noise_update(const int* erow, const int* col, const double* val, long long nnz,
                         const void* U, const void* V, bool f32, int K, int stride, double mean,
                         double var_total, double alpha_max, double* partials, int nblocks,
                         Ctl* ctl, unsigned long long seed, cudaStream_t s);
// Batched problems: per problem p (rows row0[p] .. row0[p + 1] - 1 of U, stride 32, K = Kp[p]),
// the statistics into partials + 1056 p, then the Normal-Wishart draw into mu + 32 p and
// Lambda + 1024 p (K x K), keyed with seed[p]; LamF + 1024 p receives Lambda in FP32 (32 x 32,
// zero beyond K) and lmu + 32 p Lambda mu.
void launch_prior_batch(const float* U, const int* row0, const int* Kp,
                        const unsigned long long* seed, int P, double* partials, Ctl* ctl, int mode,
                        double* mu, double* Lambda, float* LamF, double* lmu, cudaStream_t s);
void launch_set_sweep(Ctl* ctl, uint32_t sweep, int burnin, cudaStream_t s);
void launch_advance(Ctl* ctl, cudaStream_t s);

// ---- side information / block-CG (cg_kernels.cu) ----
struct DevCsr {
  const long long* ptr = nullptr;
  const int* idx = nullptr;
  const double* val = nullptr;  // null = binary
  const float* valf = nullptr;  // FP32 copy of val (mixed CG), null = binary
  long long nrow = 0;
  long long ncol = 0;
  long long nnz = 0;
  // optional work split of the SpMMs over this CSR (built by make_spmm_split): rows sorted by
  // length, rows longer than the threshold in parts whose FP64 partial rows go to `parts`
  // (64 doubles per slot) and are summed in part order by the last part to finish
  const RowTask* tasks = nullptr;
  int ntasks = 0;
  unsigned* split_cnt = nullptr;  // arrival counters of split rows (zero between launches)
  double* parts = nullptr;
};

// out[r, :ncomp] = sum_{e in row r} val_e * src[idx_e, :]   (csr_A_mul_Bn / A_mul_Bx<N>)
void launch_spmm(const DevCsr& A, const void* src, int src_stride, void* dst, int dst_stride,
                 int ncomp, bool f32, cudaStream_t s);

// Univariate prior (univariate_kernels.cu): MacauOnePrior::sample_beta over Ft (the columns of
// F as CSR rows) with the feature levels lvl_ptr / lvl_feat (lvl_range: each listed feature's
// entry range in Ft; lvl_warp: one warp per feature in that level), Z (N x zstride doubles) and draws
// (nfeat x bstride doubles) as workspace; and sample_lambda_beta into lambda_beta[0 .. K).
void launch_beta_one(const DevCsr& Ft, const double* colsq, const int* lvl_ptr,
                     const int* lvl_feat, const longlong2* lvl_range, const int* lvl_warp,
                     int nlevels, const void* U, bool f32, int ustride,
                     const double* mu, const double* uhat, int hstride, const double* Lambda,
                     const double* lambda_beta, int K, long long N, double* beta, int bstride,
                     double* Z, int zstride, double* draws, const Ctl* ctl,
                     unsigned long long seed, int mode, cudaStream_t s);
void launch_lambda_beta_one(const double* beta, int bstride, long long nfeat, int K, double a0,
                            double b0, const Ctl* ctl, unsigned long long seed, int mode,
                            double* lambda_beta, cudaStream_t s);

// sample_beta pieces (latentprior.cpp:273-293)
//   tmp[n] = U[n] + chol(Lambda)^{-T} z_n - mu      (n < N; z keyed (kMvnN, n))
void launch_beta_rhs_tmp(const void* U, bool f32, int ustride, long long N, int K,
                         const double* Lchol, const double* mu, const Ctl* ctl,
                         unsigned long long seed, int mode, double* tmp, int tstride,
                         cudaStream_t s);
//   B[f] = sum_{n in Ft row f} tmp[n] + sqrt(lambda_beta) chol(Lambda)^{-T} z_f
void launch_beta_rhs_b(const DevCsr& Ft, const double* tmp, int tstride, int K,
                       const double* Lchol, const double* lambda_beta, const Ctl* ctl,
                       unsigned long long seed, int mode, double* B, int bstride,
                       cudaStream_t s);
// one-CTA Cholesky of a K x K matrix into L (lower, zero upper); status on failure
void launch_small_chol(const double* A, int K, double* L, Ctl* ctl, cudaStream_t s);

class BlockCg {
 public:
  // Workspace for nfeat features, F with `nrow` rows, up to 64 right-hand sides.
  void reserve(long long nrow, long long nfeat, int max_rhs, bool f32);
  void release();
  // Solves (F^T F + reg I) X = B for the nrhs columns of B (nfeat x stride, row f = the nrhs
  // values of feature f) with the blocked wrapper (blocks of 32, +8 excess).  reg is a host
  // value or, when reg_dev != null, read on the device.  Returns the summed iteration count.
  int solve(const DevCsr& F, const DevCsr& Ft, double reg, const double* reg_dev,
            const double* B, int bstride, int nrhs, double tol, double* X, int xstride,
            Ctl* ctl, cudaStream_t s, bool f32);
  // Iteration cap of each block's solve (default 100,000 like the reference, linop.h:279); a
  // block that reaches it keeps its last iterate and solve() reports converged() == false.
  void set_max_iter(int n) { max_iter_ = n; }
  int max_iter() const { return max_iter_; }
  bool converged() const { return converged_; }
  ~BlockCg() { release(); }

 private:
  int core(const DevCsr& F, const DevCsr& Ft, double reg, const double* reg_dev,
           const double* B, int bstride, int nrhs, double tol, double* X, int xstride, Ctl* ctl,
           cudaStream_t s, bool f32);
  long long nrow_ = 0, nfeat_ = 0;
  int maxr_ = 0;
  int max_iter_ = 100000;
  bool converged_ = true, last_converged_ = true;
  bool f32_ = false;
  void *R_ = nullptr, *P_ = nullptr, *KP_ = nullptr, *inner_ = nullptr;
  double *Xd_ = nullptr, *Bn_ = nullptr, *KX_ = nullptr, *innerd_ = nullptr;
  double *small_ = nullptr, *partials_ = nullptr, *norms_ = nullptr;
  int *flag_host_ = nullptr;
};

}  // namespace mg
