// Host side of the library: the C ABI of include/macau_b200.h over a C++ context that owns the
// device data of one Gibbs sampler (the B200 counterpart of MacauX<MatrixData,
// FixedGaussianNoise> with BPMFPrior / MacauPrior<SparseDoubleFeat>, macau.h:56-81,
// latentprior.h:53-125).
//
// Device data layout
//   * Ratings: one CSR per mode (mode 0 = rows of Y, mode 1 = columns), int64 row pointers,
//     int32 indices sorted ascending, duplicates summed (Eigen setFromTriplets semantics).
//     Mixed mode adds a packed (index, (y - mean) * alpha as FP32) pair per entry, and at
//     K <= 32 a second copy for the tensor-core sampler in which every row starts on a
//     16-entry (128-byte) boundary and is padded to a multiple of 16 entries with
//     (N_other, 0) sentinels, so each k-block of a row is one aligned bulk copy.
//   * Latents: N x KP, row n = the K-vector of entity n, zero padded to KP in {8,..,128}.
//     FP64 mode keeps FP64; mixed mode keeps an FP32 master plus a BF16 copy that the other
//     mode's sampler gathers; the BF16 copy has one extra all-zero row N, the target of the
//     padding sentinels (the tensor-core sampler's gathers read it as a zero vector).
//   * Hyperparameters (mu, Lambda, lambda_beta) and the Macau link matrix stay on the device;
//     a sweep needs no host round trip except the block-CG convergence check.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <memory>
#include <numeric>
#include <string>
#include <vector>

#include "common.cuh"
#include "host_util.h"
#include "tune.h"
#include "kernels.h"

namespace mg {

// Host<->device byte counters of the current process (reported through mg_stats).
long long g_h2d_bytes = 0;
long long g_d2h_bytes = 0;

namespace {

struct HostCsr {
  std::vector<long long> ptr;
  std::vector<int> idx;
  std::vector<double> val;
};

// COO -> CSR over `nrow` rows with indices sorted ascending and duplicates summed.
HostCsr coo_to_csr(const int* r, const int* c, const double* v, long long nnz, long long nrow,
                   long long ncol) {
  // counting sort by column, then stable counting sort by row => (row, col) order
  std::vector<long long> cnt(std::max(nrow, ncol) + 1, 0);
  std::vector<long long> ord(nnz), ord2(nnz);
  for (long long e = 0; e < nnz; e++) cnt[c[e] + 1]++;
  for (long long i = 0; i < ncol; i++) cnt[i + 1] += cnt[i];
  for (long long e = 0; e < nnz; e++) ord[cnt[c[e]]++] = e;
  std::fill(cnt.begin(), cnt.end(), 0);
  for (long long e = 0; e < nnz; e++) cnt[r[e] + 1]++;
  for (long long i = 0; i < nrow; i++) cnt[i + 1] += cnt[i];
  for (long long q = 0; q < nnz; q++) {
    const long long e = ord[q];
    ord2[cnt[r[e]]++] = e;
  }
  HostCsr out;
  out.ptr.assign(nrow + 1, 0);
  out.idx.reserve(nnz);
  out.val.reserve(nnz);
  long long prev_r = -1, prev_c = -1;
  for (long long q = 0; q < nnz; q++) {
    const long long e = ord2[q];
    if (r[e] == prev_r && c[e] == prev_c) {
      out.val.back() += v ? v[e] : 1.0;
      continue;
    }
    out.idx.push_back(c[e]);
    out.val.push_back(v ? v[e] : 1.0);
    out.ptr[r[e] + 1]++;
    prev_r = r[e];
    prev_c = c[e];
  }
  for (long long i = 0; i < nrow; i++) out.ptr[i + 1] += out.ptr[i];
  return out;
}

// Transpose of a CSR (rows sorted within each output row because input rows are scanned in
// order).
HostCsr transpose(const HostCsr& a, long long nrow, long long ncol) {
  HostCsr t;
  const long long nnz = (long long)a.idx.size();
  t.ptr.assign(ncol + 1, 0);
  t.idx.resize(nnz);
  t.val.resize(nnz);
  for (long long e = 0; e < nnz; e++) t.ptr[a.idx[e] + 1]++;
  for (long long i = 0; i < ncol; i++) t.ptr[i + 1] += t.ptr[i];
  std::vector<long long> pos(t.ptr.begin(), t.ptr.end() - 1);
  for (long long r = 0; r < nrow; r++)
    for (long long e = a.ptr[r]; e < a.ptr[r + 1]; e++) {
      const long long q = pos[a.idx[e]]++;
      t.idx[q] = (int)r;
      t.val[q] = a.val[e];
    }
  return t;
}

struct ModeData {
  long long N = 0, nnz = 0;
  DBuf<long long> ptr;
  DBuf<int> idx;
  DBuf<double> val;
  DBuf<uint2> packed;
  DBuf<RowTask> tasks;
  DBuf<unsigned> split_cnt;
  int ntasks = 0, nsplit = 0, nslots = 0;
  long long max_len = 0;
  // tensor-core sampler (mixed, KP = 32): 16-entry padded packed CSR and its task list, whose
  // begin / len are positions in the padded array (len a multiple of 16)
  DBuf<uint2> packed_tc;
  DBuf<long long> pptr_tc;  // row pointers of the padded copy
  DBuf<RowTask> tasks_tc;
  DBuf<float> gram_tc;     // N Gram records (32 x 32 + 32 floats) written by k_gram_tc
  DBuf<int4> split_tc;     // split rows {row, parts, scratch slot of part 0, 0}
  int ntasks_tc = 0, nsplit_tc = 0, nslots_tc = 0;
  // host copy of the row pointers (task lists are rebuilt from it by the autotuner), the split
  // threshold of the current task lists, the CUDA-core sampler's CTA shape (0: default) and the
  // autotuner's record for this mode
  std::vector<long long> hptr;
  long long thr = 0;
  int groups = 0;
  TuneChoice tune;
  int tune_state = 0;  // 0 not tuned, 1 timed here, 2 taken from the cache
};

// Work split of a CSR for the side-information SpMMs (k_spmm_split): rows longer than
// max(256, nnz / (64 warps per SM)) entries are cut into parts, so the long feature columns of a
// Zipf-distributed F do not serialise on one warp.
struct SpmmSplit {
  DBuf<RowTask> tasks;
  DBuf<unsigned> cnt;
  DBuf<double> parts;
  void build(const std::vector<long long>& ptr, int num_sms, cudaStream_t s, DevCsr& A) {
    const long long nnz = ptr.empty() ? 0 : ptr.back();
    const long long thr = std::max(256LL, nnz / ((long long)num_sms * 64));
    int nsplit = 0, nslots = 0;
    std::vector<RowTask> t = make_tasks(ptr, thr, 1, nsplit, nslots);
    tasks.upload(t.data(), t.size(), s);
    cnt.alloc_zero(std::max(1, nsplit), s);
    parts.alloc((size_t)std::max(1, nslots) * 64);
    A.tasks = tasks.p;
    A.ntasks = (int)t.size();
    A.split_cnt = cnt.p;
    A.parts = parts.p;
  }
};

struct Prior {
  bool macau = false;
  DBuf<double> mu, Lambda, WI, mu0;
  double b0 = 2.0;
  int df = 0;
  // side information (MacauPrior<SparseDoubleFeat>)
  long long nfeat = 0;
  DBuf<long long> fptr, tptr;
  DBuf<int> fidx, tidx;
  DBuf<double> fval, tval;
  DBuf<float> fvalf, tvalf;
  DevCsr F, Ft;
  SpmmSplit fsplit, tsplit;
  DBuf<double> beta, uhat, tmp, B, Lchol, lambda_beta, bb_partials, bb_final;
  double lambda_beta0 = 5.0, tol = 1e-6;
  double lb_mu0 = 1.0, lb_nu0 = 1e-3;
  BlockCg cg;
  int cg_iters = 0;
  // univariate prior (MacauOnePrior, macauoneprior.h:8-51): squared column norms of F, the
  // per-dimension lambda_beta, and the feature levels of its link sampler (features sorted by
  // level, lvl_ptr[l] .. lvl_ptr[l + 1] the features of level l)
  bool one = false;
  DBuf<double> colsq, lb_one;
  DBuf<int> lvl_ptr, lvl_feat, lvl_warp;
  DBuf<longlong2> lvl_range;
  int nlevels = 0;
  double lb_a0 = 0.1, lb_b0 = 0.1;
  bool side() const { return macau || one; }
};

}  // namespace

class Context {
 public:
  explicit Context(const mg_config& c) : cfg_(c) {
    if (c.num_latent < 1 || c.num_latent > 128)
      throw MgError(MG_ERR_ARG, "num_latent must be in [1, 128]");
    K_ = c.num_latent;
    KP_ = kpad(K_);
    CP_ = K_ <= 32 ? 32 : 64;
    mixed_ = c.compute == MG_COMPUTE_MIXED;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
      throw MgError(MG_ERR_NOGPU, "no CUDA device");
    dev_ = c.device;
    MG_CUDA(cudaSetDevice(dev_));
    int major = 0;
    MG_CUDA(cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev_));
    if (major < 10) {
      cudaDeviceProp prop;
      MG_CUDA(cudaGetDeviceProperties(&prop, dev_));
      throw MgError(MG_ERR_NOGPU, std::string("sm_100a device required, found ") + prop.name);
    }
    MG_CUDA(cudaDeviceGetAttribute(&num_sms_, cudaDevAttrMultiProcessorCount, dev_));
    MG_CUDA(cudaStreamCreateWithFlags(&s_, cudaStreamNonBlocking));
    ctl_.alloc_zero(1, s_);
    for (int m = 0; m < 2; m++) prior_[m].df = K_;
    MG_CUDA(cudaEventCreate(&ev0_));
    MG_CUDA(cudaEventCreate(&ev1_));
  }

  ~Context() {
    drop_graphs();
    if (ev0_) cudaEventDestroy(ev0_);
    if (ev1_) cudaEventDestroy(ev1_);
    if (s_) cudaStreamDestroy(s_);
  }

  void set_train(const int32_t* idx, int nmodes, const double* vals, long long nnz,
                 const int32_t* dims) {
    if (nmodes != 2) throw MgError(MG_ERR_ARG, "MatrixData: tensor training input not supported.");
    set_train(idx, idx + nnz, vals, nnz, dims[0], dims[1]);
  }
  // The same from separate row and column index arrays (MatrixData::setTrain(rows, cols, ...)).
  void set_train(const int32_t* r, const int32_t* c, const double* vals, long long nnz,
                 int nrows, int ncols) {
    if (nnz < 1) throw MgError(MG_ERR_ARG, "training data is empty");
    dims_[0] = nrows;
    dims_[1] = ncols;
    // CSR of the rows and of the columns, built on the device (build_kernels.cu), which also
    // checks the indices; a rejected set leaves the context without training data.
    have_data_ = false;
    initialised_ = false;
    drop_graphs();
    long long nu = 0;
    {
      DBuf<int> dr, dc;
      DBuf<double> dv;
      dr.upload(r, (size_t)nnz, s_);
      dc.upload(c, (size_t)nnz, s_);
      dv.upload(vals, (size_t)nnz, s_);
      for (int m = 0; m < 2; m++) {
        md_[m].ptr.alloc((size_t)dims_[m] + 1);
        md_[m].idx.alloc((size_t)nnz);
        md_[m].val.alloc((size_t)nnz);
      }
      nu = build_csr_pair(dr.p, dc.p, dv.p, nnz, dims_[0], dims_[1], md_[0].ptr.p, md_[0].idx.p,
                          md_[0].val.p, md_[1].ptr.p, md_[1].idx.p, md_[1].val.p, s_);
    }
    // mean_value = Y.sum() / Y.nonZeros() over the column-major storage (sparsetensor.cpp:82),
    // and AdaptiveGaussianNoise::init's var_total (noisemodels.cpp:14-33), summed on the device
    std::vector<long long> p0((size_t)dims_[0] + 1), p1((size_t)dims_[1] + 1);
    MG_CUDA(cudaMemcpyAsync(p0.data(), md_[0].ptr.p, sizeof(long long) * p0.size(),
                            cudaMemcpyDeviceToHost, s_));
    MG_CUDA(cudaMemcpyAsync(p1.data(), md_[1].ptr.p, sizeof(long long) * p1.size(),
                            cudaMemcpyDeviceToHost, s_));
    g_d2h_bytes += (long long)(sizeof(long long) * (p0.size() + p1.size()) + 16);
    ntrain_ = nu;
    mean_ = value_moment(md_[1].val.p, nu, 0.0, false, s_) / (double)ntrain_;
    var_total_ = value_moment(md_[1].val.p, nu, mean_, true, s_) / (double)ntrain_;
    if (var_total_ <= 0.0 || std::isnan(var_total_)) var_total_ = 1.0;
    upload_mode(0, p0, nu);
    upload_mode(1, p1, nu);
    drop_graphs();
    have_data_ = true;
    initialised_ = false;
  }

  void set_test(const int32_t* idx, int nmodes, const double* vals, long long nnz,
                const int32_t* dims) {
    if (nmodes != 2) throw MgError(MG_ERR_ARG, "MatrixData: tensor test input not supported.");
    set_test(idx, idx + nnz, vals, nnz, dims);
  }
  // The same from separate row and column index arrays (MatrixData::setTest(rows, cols, ...)).
  void set_test(const int32_t* r, const int32_t* c, const double* vals, long long nnz,
                const int32_t* dims) {
    // Ytest in CSC order (sparseFromIJV -> column-major storage): entries sorted by (column,
    // row), duplicates summed in input order, built and index-checked on the device.
    ntest_ = 0;
    drop_graphs();
    if (nnz > 0) {
      DBuf<int> dr, dc;
      DBuf<double> dv;
      dr.upload(r, (size_t)nnz, s_);
      dc.upload(c, (size_t)nnz, s_);
      dv.upload(vals, (size_t)nnz, s_);
      trow_.alloc((size_t)nnz);
      tcol_.alloc((size_t)nnz);
      tval_.alloc((size_t)nnz);
      ntest_ = build_coo_sorted(dc.p, dr.p, dv.p, nnz, dims[1], dims[0], "test index out of range",
                                tcol_.p, trow_.p, tval_.p, s_);
    }
    pred_.alloc_zero(ntest_, s_);
    pvar_.alloc_zero(ntest_, s_);
    eval_partials_.alloc(2 * (size_t)eval_blocks(ntest_));
    rmse_.alloc(2);
    const double nan2[2] = {NAN, NAN};
    MG_CUDA(cudaMemcpyAsync(rmse_.p, nan2, sizeof(nan2), cudaMemcpyHostToDevice, s_));
    MG_CUDA(cudaStreamSynchronize(s_));
  }

  // univariate = false: MacauPrior<SparseDoubleFeat> (block-CG link solve); true: MacauOnePrior
  // (macauoneprior.cpp:16-39), whose link sampler visits the features level by level.
  void set_side(int mode, const int32_t* rows, const int32_t* cols, const double* vals,
                long long nnz, int nrows, int nfeat, double lambda_beta, double tol,
                bool univariate = false) {
    if (mode < 0 || mode > 1) throw MgError(MG_ERR_ARG, "mode must be 0 or 1");
    if (!have_data_) throw MgError(MG_ERR_STATE, "set the training data before side info");
    if (nrows != dims_[mode])
      throw MgError(MG_ERR_ARG, "side information rows must equal the mode's dimension");
    if (K_ > 64) throw MgError(MG_ERR_ARG, "side information supports num_latent <= 64");
    for (long long e = 0; e < nnz; e++)
      if (rows[e] < 0 || rows[e] >= nrows || cols[e] < 0 || cols[e] >= nfeat)
        throw MgError(MG_ERR_ARG, "side information index out of range");
    Prior& p = prior_[mode];
    HostCsr f = coo_to_csr(rows, cols, vals, nnz, nrows, nfeat);
    HostCsr t = transpose(f, nrows, nfeat);
    bool binary = true;
    for (double v : f.val) binary = binary && (v == 1.0);
    p.macau = !univariate;
    p.one = univariate;
    p.nfeat = nfeat;
    p.fptr.upload(f.ptr.data(), f.ptr.size(), s_);
    p.fidx.upload(f.idx.data(), f.idx.size(), s_);
    p.tptr.upload(t.ptr.data(), t.ptr.size(), s_);
    p.tidx.upload(t.idx.data(), t.idx.size(), s_);
    p.F = DevCsr{};
    p.Ft = DevCsr{};
    if (!binary) {
      p.fval.upload(f.val.data(), f.val.size(), s_);
      p.tval.upload(t.val.data(), t.val.size(), s_);
      std::vector<float> ff(f.val.begin(), f.val.end()), tf(t.val.begin(), t.val.end());
      p.fvalf.upload(ff.data(), ff.size(), s_);
      p.tvalf.upload(tf.data(), tf.size(), s_);
      p.F.val = p.fval.p;
      p.F.valf = p.fvalf.p;
      p.Ft.val = p.tval.p;
      p.Ft.valf = p.tvalf.p;
    }
    p.F.ptr = p.fptr.p;
    p.F.idx = p.fidx.p;
    p.F.nrow = nrows;
    p.F.ncol = nfeat;
    p.F.nnz = (long long)f.idx.size();
    p.Ft.ptr = p.tptr.p;
    p.Ft.idx = p.tidx.p;
    p.Ft.nrow = nfeat;
    p.Ft.ncol = nrows;
    p.Ft.nnz = p.F.nnz;
    p.fsplit.build(f.ptr, num_sms_, s_, p.F);
    p.tsplit.build(t.ptr, num_sms_, s_, p.Ft);
    p.lambda_beta0 = lambda_beta;
    p.tol = tol;
    if (univariate) {
      // col_square_sum (linop.cpp:374-401) and the feature levels: level(f) = 1 + the highest
      // level of an earlier feature sharing a row with f (0 when none)
      std::vector<double> cs(nfeat, 0.0);
      std::vector<int> level(nfeat, 0), last(nrows, -1);
      int nl = 0;
      for (int f = 0; f < nfeat; f++) {
        int lv = 0;
        for (long long e = t.ptr[f]; e < t.ptr[f + 1]; e++) {
          cs[f] += binary ? 1.0 : t.val[e] * t.val[e];
          lv = std::max(lv, last[t.idx[e]] + 1);
        }
        for (long long e = t.ptr[f]; e < t.ptr[f + 1]; e++) last[t.idx[e]] = lv;
        level[f] = lv;
        nl = std::max(nl, lv + 1);
      }
      std::vector<int> lptr(nl + 1, 0), order(nfeat);
      for (int f = 0; f < nfeat; f++) lptr[level[f] + 1]++;
      for (int l = 0; l < nl; l++) lptr[l + 1] += lptr[l];
      std::vector<int> fill(lptr.begin(), lptr.end() - 1);
      for (int f = 0; f < nfeat; f++) order[fill[level[f]]++] = f;
      // a level runs one warp per feature when it has many features or only short ones
      std::vector<int> lwarp(nl, 1);
      for (int l = 0; l < nl; l++) {
        long long longest = 0;
        for (int q = lptr[l]; q < lptr[l + 1]; q++)
          longest = std::max(longest, t.ptr[order[q] + 1] - t.ptr[order[q]]);
        lwarp[l] = (lptr[l + 1] - lptr[l] >= 8 || longest <= 1024) ? 1 : 0;
      }
      p.colsq.upload(cs.data(), cs.size(), s_);
      p.lvl_warp.upload(lwarp.data(), lwarp.size(), s_);
      p.lvl_ptr.upload(lptr.data(), lptr.size(), s_);
      p.lvl_feat.upload(order.data(), order.size(), s_);
      std::vector<longlong2> range(nfeat);
      for (int q = 0; q < nfeat; q++)
        range[q] = make_longlong2(t.ptr[order[q]], t.ptr[order[q] + 1]);
      p.lvl_range.upload(range.data(), range.size(), s_);
      p.nlevels = nl;
    }
    MG_CUDA(cudaStreamSynchronize(s_));
    drop_graphs();
    initialised_ = false;
  }

  void set_samples(int burnin, int nsamples) {
    burnin_ = burnin;
    nsamples_ = nsamples;
  }

  // MacauX::init (macau.cpp:72-86) + prior init (latentprior.cpp:84-99, 181-216)
  void init() {
    if (!have_data_) throw MgError(MG_ERR_STATE, "no training data");
    for (int m = 0; m < 2; m++) {
      size_gram_records(m);  // the prior kind decides whether the mode keeps per-row records
      const size_t n = (size_t)dims_[m] * KP_;
      if (mixed_) {
        lat32_[m].alloc_zero(n, s_);
        lat16_[m].alloc_zero(n + KP_, s_);  // + the zero row N
        lat64_[m].reset();
      } else {
        lat64_[m].alloc_zero(n, s_);
        lat32_[m].reset();
        lat16_[m].reset();
      }
      Prior& p = prior_[m];
      std::vector<double> eye((size_t)K_ * K_, 0.0), lam((size_t)K_ * K_, 0.0), z(K_, 0.0);
      for (int i = 0; i < K_; i++) {
        eye[i + (size_t)i * K_] = 1.0;
        lam[i + (size_t)i * K_] = 10.0;
      }
      p.mu.upload(z.data(), K_, s_);
      p.mu0.upload(z.data(), K_, s_);
      p.Lambda.upload(lam.data(), lam.size(), s_);
      p.WI.upload(eye.data(), eye.size(), s_);
      p.b0 = 2.0;
      p.df = K_;
      if (p.macau) {
        p.beta.alloc_zero((size_t)p.nfeat * CP_, s_);
        p.uhat.alloc_zero((size_t)dims_[m] * KP_, s_);
        p.tmp.alloc_zero((size_t)dims_[m] * CP_, s_);
        p.B.alloc_zero((size_t)p.nfeat * CP_, s_);
        p.Lchol.alloc_zero((size_t)K_ * K_, s_);
        p.lambda_beta.upload(&p.lambda_beta0, 1, s_);
        p.bb_partials.alloc((size_t)stats_blocks(p.nfeat) * (K_ + K_ * K_));
        p.bb_final.alloc((size_t)(K_ + K_ * K_));
        p.cg.reserve(p.F.nrow, p.nfeat, 64, cg_f32_);
      }
      if (p.one) {  // MacauOnePrior::init (macauoneprior.cpp:16-39) + setLambdaBeta
        p.beta.alloc_zero((size_t)p.nfeat * CP_, s_);
        p.uhat.alloc_zero((size_t)dims_[m] * KP_, s_);
        p.tmp.alloc_zero((size_t)dims_[m] * CP_, s_);
        p.B.alloc_zero((size_t)p.nfeat * CP_, s_);  // the link sampler's draws
        std::vector<double> lb(K_, p.lambda_beta0);
        p.lb_one.upload(lb.data(), lb.size(), s_);
      }
    }
    const long long maxN = std::max(dims_[0], dims_[1]);
    stat_partials_.alloc((size_t)stats_blocks(maxN) * (K_ + K_ * K_));
    stat_final_.alloc((size_t)(K_ + K_ * K_));
    if (pair_priors()) {  // mode 1's own work of the two-mode prior update
      stat_partials1_.alloc((size_t)stats_blocks(dims_[1]) * (K_ + K_ * K_));
      stat_final1_.alloc((size_t)(K_ + K_ * K_));
    }
    nwbuf_.alloc(3 * (size_t)K_ + 4 * (size_t)K_ * K_);
    nw_.vec = nwbuf_.p;
    nw_.m0 = nwbuf_.p + 3 * K_;
    nw_.m1 = nw_.m0 + K_ * K_;
    nw_.m2 = nw_.m1 + K_ * K_;
    nw_.m3 = nw_.m2 + K_ * K_;
    if (ntest_ > 0) {
      MG_CUDA(cudaMemsetAsync(pred_.p, 0, ntest_ * sizeof(double), s_));
      MG_CUDA(cudaMemsetAsync(pvar_.p, 0, ntest_ * sizeof(double), s_));
    }
    Ctl zero{};
    zero.bad_row = -1;
    // AdaptiveGaussianNoise::init: alpha = (sn_init + 1) / var_total, alpha_max likewise
    alpha_max_ = (sn_max_ + 1.0) / var_total_;
    zero.alpha = adaptive_ ? (sn_init_ + 1.0) / var_total_ : cfg_.precision;
    if (adaptive_) {
      erow_.alloc((size_t)md_[0].nnz);
      launch_entry_rows(md_[0].ptr.p, md_[0].N, md_[0].nnz, erow_.p, s_);
      noise_partials_.alloc((size_t)eval_blocks(md_[0].nnz));
    }
    MG_CUDA(cudaMemcpyAsync(ctl_.p, &zero, sizeof(Ctl), cudaMemcpyHostToDevice, s_));
    MG_CUDA(cudaStreamSynchronize(s_));
    retries_[0] = retries_[1] = 0;
    rows_[0] = rows_[1] = 0;
    sweeps_done_ = 0;
    launches_ = 0;
    t_sample_ = t_prior_ = t_eval_ = 0.0;
    drop_graphs();
    initialised_ = true;
    if (autotune_) autotune(autotune_ == 1);
  }


  // ---- phases ----
  void sample(int mode, const double* znoise_dev, bool reset_queue = true,
              cudaEvent_t mid = nullptr) {
    launches_ += 1;
    ModeData& md = md_[mode];
    Prior& p = prior_[mode];
    const int other = 1 - mode;
    if (reset_queue) MG_CUDA(cudaMemsetAsync(&ctl_.p->queue[0], 0, 8 * sizeof(uint32_t), s_));
    SampleParams sp{};
    sp.tasks = md.tasks.p;
    sp.ntasks = md.ntasks;
    sp.nrows = (int)md.N;
    sp.nother = (int)dims_[other];
    sp.K = K_;
    sp.rowptr = md.ptr.p;
    sp.colidx = md.idx.p;
    sp.vals = md.val.p;
    sp.packed = md.packed.p;
    sp.mean = mean_;
    sp.alpha = cfg_.precision;
    sp.alpha_dev = adaptive_ ? &ctl_.p->alpha : nullptr;
    sp.other = !mixed_ ? (const void*)lat64_[other].p
               : gram_ == 2 ? (const void*)lat32_[other].p   // TF32: rounded from the master
                            : (const void*)lat16_[other].p;
    sp.half_copy = mixed_ && gram_ == 1 ? 1 : 0;
    sp.Lambda = p.Lambda.p;
    sp.mu = p.mu.p;
    sp.uhat = p.side() ? p.uhat.p : nullptr;
    sp.one = p.one ? 1 : 0;
    sp.out_f64 = lat64_[mode].p;
    sp.out_f32 = lat32_[mode].p;
    sp.out_bf16 = lat16_[mode].p;
    sp.scratch = scratch_.p;
    sp.retry_work = retry_work_.p;
    sp.split_cnt = md.split_cnt.p;
    sp.ctl = ctl_.p;
    sp.qslot = mode;
    sp.mode = mode;
    sp.seed = cfg_.seed;
    sp.znoise = znoise_dev;
    sp.wait_cycles = tc_wait_cycles_;
    sp.wait_test = tc_wait_test_ ? 1 : 0;
    if (range_hi_[mode] >= 0 && uses_tc(mode) && (!fused_ || p.one))
      throw MgError(MG_ERR_STATE, "a row range needs the fused tensor-core sampler or the "
                                  "CUDA-core sampler (its record-based finish covers all rows)");
    if (mixed_ && use_tc_ && gram_ == 0 && KP_ == 32) {
      SampleParams tp = sp;
      tp.tasks = md.tasks_tc.p;
      tp.ntasks = md.ntasks_tc;
      tp.packed = md.packed_tc.p;
      if (launch_sample_tc(tp, md.gram_tc.p, md.split_tc.p, md.nsplit_tc, KP_, s_, num_sms_,
                           mid, fused_)) {
        // k_gram_tc (+ k_sum_parts) + k_finish_tc; fused: k_gram_tc (+ k_sum_parts + k_finish_tc)
        if (fused_ && !p.one)
          launches_ += md.nsplit_tc > 0 ? 2 : 0;
        else
          launches_ += 1 + (md.nsplit_tc > 0 ? 1 : 0);
        return;
      }
    }
    launch_sample(sp, KP_, mixed_, gram_, s_, num_sms_, md.groups);
  }

  // Sampler kind of mode m in the autotuner's keys.
  const char* tune_kind(int m) const {
    if (uses_tc(m)) return "tc";
    if (!mixed_) return "fp64";
    return gram_ == 0 ? "bf16" : gram_ == 1 ? "fp16" : "tf32";
  }

  // True when mode m's latents are drawn by the tensor-core sampler.
  bool uses_tc(int m) const {
    return mixed_ && use_tc_ && gram_ == 0 && KP_ == 32 && md_[m].packed_tc.p != nullptr;
  }

  // Autotuner (tune.h): for each mode, the split threshold of the task lists (divisors 1, 2, 4,
  // 8, 16 of nnz per row group) and, for the CUDA-core sampler, its CTA shape, each timed as
  // one warm-up and three timed half-sweeps (CUDA events, the fastest kept) on the current
  // state.  The latents, the control block and the counters are restored afterwards, so the
  // chain continues as if untuned; only the summation order of split rows can differ.
  void autotune(bool use_cache) {
    if (!initialised_) throw MgError(MG_ERR_STATE, "call mg_init before autotuning");
    drop_graphs();
    const long long saved_launches = launches_;
    const double saved_ts = t_sample_;
    const long long saved_retries[2] = {retries_[0], retries_[1]};
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    try {
      DeviceBackup ctl_backup(s_);  // the control block (sweep, queues, retry counts, alpha)
      ctl_backup.save(ctl_.p, sizeof(Ctl));
      MG_CUDA(cudaEventCreate(&e0));
      MG_CUDA(cudaEventCreate(&e1));
      for (int m = 0; m < 2; m++) {
        ModeData& md = md_[m];
        const bool tc = uses_tc(m);
        const std::string key = tune_key(tune_kind(m), K_, num_sms_, md.hptr);
        TuneChoice c;
        if (use_cache && TuneCache::get().find(key, &c)) {
          if (md.thr != c.thr || md.groups != c.groups) {
            md.groups = c.groups;
            build_tasks(m, c.thr);
          }
          md.tune = c;
          md.tune_state = 2;
          continue;
        }
        // the latents this mode's timing runs overwrite, put back before the next mode (whose
        // sampler reads them) or when a run throws
        DeviceBackup lat_backup(s_);
        const size_t n = (size_t)dims_[m] * KP_;
        if (lat64_[m].p) lat_backup.save(lat64_[m].p, n * sizeof(double));
        if (lat32_[m].p) lat_backup.save(lat32_[m].p, n * sizeof(float));
        if (lat16_[m].p) lat_backup.save(lat16_[m].p, lat16_[m].n * sizeof(__nv_bfloat16));
        std::vector<long long> thrs;
        for (int div : {2, 1, 4, 8, 16}) {
          const long long t = split_divisor_thr(m, div);
          if (std::find(thrs.begin(), thrs.end(), t) == thrs.end()) thrs.push_back(t);
        }
        const std::vector<int> shapes =
            tc ? std::vector<int>{0} : sample_group_options(KP_, mixed_, gram_);
        TuneChoice best;
        best.ms = 1e30;
        int tried = 0;
        for (int g : shapes)
          for (long long t : thrs) {
            md.groups = g;
            build_tasks(m, t);
            float best_ms = 1e30f;
            for (int rep = 0; rep < 4; rep++) {
              MG_CUDA(cudaEventRecord(e0, s_));
              sample(m, nullptr);
              MG_CUDA(cudaEventRecord(e1, s_));
              MG_CUDA(cudaEventSynchronize(e1));
              float ms = 0.f;
              MG_CUDA(cudaEventElapsedTime(&ms, e0, e1));
              if (rep > 0) best_ms = std::min(best_ms, ms);
            }
            check_status();
            tried++;
            if (tried == 1) best.ms_default = best_ms;
            if (best_ms < best.ms) {
              best.ms = best_ms;
              best.thr = t;
              best.groups = g;
            }
          }
        best.candidates = tried;
        md.groups = best.groups;
        build_tasks(m, best.thr);
        md.tune = best;
        md.tune_state = 1;
        TuneCache::get().put(key, best);
      }
    } catch (...) {
      if (e0) cudaEventDestroy(e0);
      if (e1) cudaEventDestroy(e1);
      launches_ = saved_launches;
      t_sample_ = saved_ts;
      retries_[0] = saved_retries[0];
      retries_[1] = saved_retries[1];
      throw;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    MG_CUDA(cudaStreamSynchronize(s_));
    launches_ = saved_launches;
    t_sample_ = saved_ts;
    retries_[0] = saved_retries[0];
    retries_[1] = saved_retries[1];
    drop_graphs();
  }

  void get_tuning(int mode, mg_tuning* out) const {
    if (mode < 0 || mode > 1) throw MgError(MG_ERR_ARG, "mode must be 0 or 1");
    const ModeData& md = md_[mode];
    out->split_threshold = md.thr;
    out->cta_groups = uses_tc(mode) ? 0 : (md.groups ? md.groups : sample_default_groups(KP_));
    out->tensor_core = uses_tc(mode) ? 1 : 0;
    out->state = md.tune_state;
    out->candidates = md.tune_state ? md.tune.candidates : 0;
    out->ms_best = md.tune_state ? md.tune.ms : 0.0;
    out->ms_default = md.tune_state ? md.tune.ms_default : 0.0;
    out->finish_ctas_per_sm = 0;
  }

  const void* latents(int mode) const {
    return mixed_ ? (const void*)lat32_[mode].p : (const void*)lat64_[mode].p;
  }

  // Both modes have the plain BPMF prior at K <= 32: the sweep updates them together
  // (launch_prior_pair: three launches instead of six, the same result bit for bit).  The
  // phase-timed sweeps keep one mode after the other, so each mode's prior is timed alone.
  bool pair_priors() const {
    return K_ <= 32 && !prior_[0].macau && !prior_[0].one && !prior_[1].macau && !prior_[1].one;
  }
  void update_priors_pair() {
    PriorPair pp{};
    for (int m = 0; m < 2; m++) {
      const Prior& p = prior_[m];
      pp.U[m] = latents(m);
      pp.N[m] = dims_[m];
      pp.nblocks[m] = stats_blocks(dims_[m]);
      pp.rows_per_block[m] = (dims_[m] + pp.nblocks[m] - 1) / pp.nblocks[m];
      pp.partials[m] = m ? stat_partials1_.p : stat_partials_.p;
      pp.final_[m] = m ? stat_final1_.p : stat_final_.p;
      pp.mu0[m] = p.mu0.p;
      pp.kappa[m] = p.b0;
      pp.T0[m] = p.WI.p;
      pp.nu[m] = p.df;
      pp.mu[m] = p.mu.p;
      pp.Lambda[m] = p.Lambda.p;
    }
    launch_prior_pair(pp, mixed_, K_, KP_, ctl_.p, cfg_.seed, s_);
    launches_ += 3;
  }

  void update_prior(int mode) {
    Prior& p = prior_[mode];
    const long long N = dims_[mode];
    launches_ += p.macau ? 0 : 3;  // Macau launches are counted by kernels_in_cg below
    const int nb = stats_blocks(N);
    const int rec = K_ + K_ * K_;
    launch_stats(latents(mode), mixed_, p.side() ? p.uhat.p : nullptr, N, K_, KP_, KP_,
                 stat_partials_.p, nb, s_);
    launch_reduce_parts(stat_partials_.p, nb, rec, stat_final_.p, s_);
    if (p.one) {
      // MacauOnePrior::update_prior (macauoneprior.cpp:189-194): sample_mu_lambda (Normal-Wishart
      // of U - Uhat with mu0 = 0, kappa = 2, W0 = I, nu = K, the BPMF defaults), sample_beta,
      // compute_uhat, sample_lambda_beta
      launch_normal_wishart(stat_final_.p, 1, N, K_, p.mu0.p, p.b0, p.WI.p, p.df, nullptr, 0,
                            nullptr, nw_, ctl_.p, cfg_.seed, mode, p.mu.p, p.Lambda.p, s_);
      launch_beta_one(p.Ft, p.colsq.p, p.lvl_ptr.p, p.lvl_feat.p, p.lvl_range.p, p.lvl_warp.p,
                      p.nlevels,
                      latents(mode),
                      mixed_, KP_, p.mu.p, p.uhat.p, KP_, p.Lambda.p, p.lb_one.p, K_, N, p.beta.p,
                      CP_, p.tmp.p, CP_, p.B.p, ctl_.p, cfg_.seed, mode, s_);
      launch_spmm(p.F, p.beta.p, CP_, p.uhat.p, KP_, K_, false, s_);
      launch_lambda_beta_one(p.beta.p, CP_, p.nfeat, K_, p.lb_a0, p.lb_b0, ctl_.p, cfg_.seed,
                             mode, p.lb_one.p, s_);
      launches_ += 4;  // draws, beta, spmm, lambda_beta (after the 3 of stats / reduce / NW)
      return;
    }
    if (!p.macau) {  // BPMFPrior::update_prior (latentprior.cpp:79-81)
      launch_normal_wishart(stat_final_.p, 1, N, K_, p.mu0.p, p.b0, p.WI.p, p.df, nullptr, 0,
                            nullptr, nw_, ctl_.p, cfg_.seed, mode, p.mu.p, p.Lambda.p, s_);
      return;
    }
    // MacauPrior::update_prior (latentprior.cpp:255-264)
    const int nbb = stats_blocks(p.nfeat);
    launch_stats(p.beta.p, false, nullptr, p.nfeat, K_, CP_, 0, p.bb_partials.p, nbb, s_);
    launch_reduce_parts(p.bb_partials.p, nbb, rec, p.bb_final.p, s_);
    launch_normal_wishart(stat_final_.p, 1, N, K_, p.mu0.p, p.b0, p.WI.p, p.df + (int)p.nfeat,
                          p.bb_final.p, 1, p.lambda_beta.p, nw_, ctl_.p, cfg_.seed, mode, p.mu.p,
                          p.Lambda.p, s_);
    // sample_beta (latentprior.cpp:273-293)
    launch_small_chol(p.Lambda.p, K_, p.Lchol.p, ctl_.p, s_);
    launch_beta_rhs_tmp(latents(mode), mixed_, KP_, N, K_, p.Lchol.p, p.mu.p, ctl_.p, cfg_.seed,
                        mode, p.tmp.p, CP_, s_);
    launch_beta_rhs_b(p.Ft, p.tmp.p, CP_, K_, p.Lchol.p, p.lambda_beta.p, ctl_.p, cfg_.seed,
                      mode, p.B.p, CP_, s_);
    p.cg.set_max_iter(cg_max_iter_);
    p.cg_iters = p.cg.solve(p.F, p.Ft, 0.0, p.lambda_beta.p, p.B.p, CP_, K_, p.tol, p.beta.p,
                            CP_, ctl_.p, s_, cg_f32_);
    // a solve that reached its cap keeps its last iterate; the update completes and the
    // status check after it reports MG_ERR_CG
    if (!p.cg.converged()) cg_noconv_ = true;
    // stats x3 (+ reductions), NW, chol, tmp, spmm, noise, uhat spmm, lambda_beta + the CG's
    // (set-up, then 10 per iteration)
    launches_ += 12 + 6 + 10LL * p.cg_iters;
    // compute_uhat (linop.h:196-198): Uhat = beta F^T, one K-vector per row of F
    launch_spmm(p.F, p.beta.p, CP_, p.uhat.p, KP_, K_, false, s_);
    // sample_lambda_beta with the new beta and Lambda (latentprior.cpp:263)
    launch_stats(p.beta.p, false, nullptr, p.nfeat, K_, CP_, 0, p.bb_partials.p, nbb, s_);
    launch_reduce_parts(p.bb_partials.p, nbb, rec, p.bb_final.p, s_);
    launch_lambda_beta(p.bb_final.p, 1, K_, p.nfeat, p.Lambda.p, p.lb_nu0, p.lb_mu0, ctl_.p,
                       cfg_.seed, mode, p.lambda_beta.p, s_);
  }

  void eval(int n_fixed) {
    if (ntest_ == 0) return;
    launches_ += 2;
    launch_eval(trow_.p, tcol_.p, tval_.p, ntest_, latents(0), latents(1), mixed_, K_, KP_,
                mean_, n_fixed, ctl_.p, pred_.p, pvar_.p, eval_partials_.p,
                eval_blocks(ntest_), rmse_.p, s_);
  }

  // AdaptiveGaussianNoise::update (noisemodels.cpp:55-81); nothing under fixed noise.
  void update_noise() {
    if (!adaptive_) return;
    launches_ += 2;
    const ModeData& md = md_[0];
    launch_noise_update(erow_.p, md.idx.p, md.val.p, md.nnz, latents(0), latents(1), mixed_, K_,
                        KP_, mean_, var_total_, alpha_max_, noise_partials_.p,
                        eval_blocks(md.nnz), ctl_.p, cfg_.seed, s_);
  }

  // Noise model before its first sweep: AdaptiveGaussianNoise(sn_init, sn_max) in place of
  // FixedGaussianNoise(precision) (make_macau_adaptive, macau.cpp:222-228).
  void set_noise_adaptive(double sn_init, double sn_max) {
    if (!(sn_init >= 0.0) || !(sn_max >= 0.0) || !std::isfinite(sn_init) || !std::isfinite(sn_max))
      throw MgError(MG_ERR_ARG, "sn_init and sn_max must be finite and non-negative");
    adaptive_ = true;
    sn_init_ = sn_init;
    sn_max_ = sn_max;
    if (have_data_) {
      pack_mode(0);
      pack_mode(1);
      MG_CUDA(cudaStreamSynchronize(s_));
    }
    drop_graphs();
    initialised_ = false;
  }

  // out[0] = current precision, out[1] = its cap (adaptive noise), out[2] = var_total
  void get_noise(double* out) {
    double a = cfg_.precision;
    if (initialised_) {
      Ctl h;
      MG_CUDA(cudaMemcpyAsync(&h, ctl_.p, sizeof(Ctl), cudaMemcpyDeviceToHost, s_));
      MG_CUDA(cudaStreamSynchronize(s_));
      g_d2h_bytes += sizeof(Ctl);
      a = h.alpha;
    }
    out[0] = a;
    out[1] = adaptive_ ? (sn_max_ + 1.0) / var_total_ : cfg_.precision;
    out[2] = var_total_;
  }
  bool adaptive() const { return adaptive_; }

  bool graphable() const { return !prior_[0].macau && !prior_[1].macau; }

  // One sweep; ev (optional, 8 events) brackets: sample 0 | sample 1 | prior 0 | prior 1 |
  // noise update + eval + advance; ev[6], ev[7] end the tensor-core Gram kernel of mode 0, 1 (recorded only
  // when that sampler runs).
  void sweep_body(bool do_eval, cudaEvent_t* ev = nullptr) {
    MG_CUDA(cudaMemsetAsync(&ctl_.p->queue[0], 0, 8 * sizeof(uint32_t), s_));
    if (ev) MG_CUDA(cudaEventRecord(ev[0], s_));
    sample(0, nullptr, false, ev ? ev[6] : nullptr);
    if (ev) MG_CUDA(cudaEventRecord(ev[1], s_));
    sample(1, nullptr, false, ev ? ev[7] : nullptr);
    if (ev) MG_CUDA(cudaEventRecord(ev[2], s_));
    if (!ev && pair_priors()) {
      update_priors_pair();
    } else {
      update_prior(0);
      if (ev) MG_CUDA(cudaEventRecord(ev[3], s_));
      update_prior(1);
    }
    if (ev) MG_CUDA(cudaEventRecord(ev[4], s_));
    update_noise();  // noise.update between the priors and the evaluation (macau.cpp:130-132)
    if (do_eval) eval(-1);
    launch_advance(ctl_.p, s_);
    launches_ += 1;
    if (ev) MG_CUDA(cudaEventRecord(ev[5], s_));
  }

  // Device time of `count` sweeps: total between two events on the library stream; with
  // phase_events the sweeps run un-captured with events between phases and phase[0..4]
  // receives the summed seconds of sample 0, sample 1, prior 0, prior 1, eval.
  void time_sweeps(int first_iter, int count, bool do_eval, bool phase_events, double* total,
                   double* phase) {
    if (!initialised_) throw MgError(MG_ERR_STATE, "call mg_init first");
    if (count < 1) {
      if (total) *total = 0.0;
      if (phase)
        for (int q = 0; q < 7; q++) phase[q] = 0.0;
      return;
    }
    if (!phase_events) {
      // make sure the graph exists before the timed region
      if (graphable() && use_graph_ && !graph_[do_eval ? 1 : 0]) {
        sweeps(first_iter, 1, do_eval, true);
        first_iter++;
        count--;
      }
      MG_CUDA(cudaStreamSynchronize(s_));
      MG_CUDA(cudaEventRecord(ev0_, s_));
      sweeps(first_iter, count, do_eval, false);
      MG_CUDA(cudaEventRecord(ev1_, s_));
      MG_CUDA(cudaEventSynchronize(ev1_));
      float ms = 0.f;
      MG_CUDA(cudaEventElapsedTime(&ms, ev0_, ev1_));
      if (total) *total = ms * 1e-3;
      check_status();
      return;
    }
    std::vector<cudaEvent_t> ev((size_t)count * 8);
    for (auto& e : ev) MG_CUDA(cudaEventCreate(&e));
    try {
      launch_set_sweep(ctl_.p, (uint32_t)first_iter, burnin_, s_);
      for (int i = 0; i < count; i++) sweep_body(do_eval, ev.data() + 8 * (size_t)i);
      rows_[0] += md_[0].N * count;
      rows_[1] += md_[1].N * count;
      sweeps_done_ += count;
      const bool tc = mixed_ && use_tc_ && KP_ == 32;
      MG_CUDA(cudaEventSynchronize(ev[8 * (size_t)(count - 1) + 5]));
      double ph[7] = {0, 0, 0, 0, 0, 0, 0};
      for (int i = 0; i < count; i++) {
        const cudaEvent_t* e = ev.data() + 8 * (size_t)i;
        for (int q = 0; q < 5; q++) {
          float ms = 0.f;
          MG_CUDA(cudaEventElapsedTime(&ms, e[q], e[q + 1]));
          ph[q] += ms * 1e-3;
        }
        for (int m = 0; tc && m < 2; m++) {
          float ms = 0.f;
          MG_CUDA(cudaEventElapsedTime(&ms, e[m], e[6 + m]));
          ph[5 + m] += ms * 1e-3;
        }
      }
      float ms = 0.f;
      MG_CUDA(cudaEventElapsedTime(&ms, ev[0], ev[8 * (size_t)(count - 1) + 5]));
      if (total) *total = ms * 1e-3;
      if (phase)
        for (int q = 0; q < 7; q++) phase[q] = ph[q];
    } catch (...) {
      for (auto& e : ev) cudaEventDestroy(e);
      throw;
    }
    for (auto& e : ev) cudaEventDestroy(e);
    check_status();
  }

  void check_status() {
    Ctl h;
    MG_CUDA(cudaMemcpyAsync(&h, ctl_.p, sizeof(Ctl), cudaMemcpyDeviceToHost, s_));
    g_d2h_bytes += sizeof(Ctl);
    MG_CUDA(cudaStreamSynchronize(s_));
    retries_[0] = h.retries[0];
    retries_[1] = h.retries[1];
    // a timed-out launch left its work unfinished, so its status comes before what followed
    if (h.status & kStatTimeout) throw MgError(MG_ERR_TIMEOUT, "device wait timed out");
    if (cg_noconv_) {
      cg_noconv_ = false;
      throw MgError(MG_ERR_CG, "block-CG did not converge within " + std::to_string(cg_max_iter_) +
                                   " iterations");
    }
    if (h.status & kStatCholFail)
      throw MgError(MG_ERR_CHOL, "Cholesky Decomposition failed!");
    if (h.status & kStatHyperFail)
      throw MgError(MG_ERR_CHOL, "Cholesky Decomposition failed! (hyperprior)");
    if (h.status & kStatCgFail) throw MgError(MG_ERR_CG, "block-CG breakdown");
  }

  void sweeps(int first_iter, int count, bool do_eval, bool sync = true) {
    if (!initialised_) throw MgError(MG_ERR_STATE, "call mg_init first");
    launch_set_sweep(ctl_.p, (uint32_t)first_iter, burnin_, s_);
    rows_[0] += md_[0].N * count;
    rows_[1] += md_[1].N * count;
    sweeps_done_ += count;
    if (graphable() && use_graph_) {
      cudaGraphExec_t& ge = graph_[do_eval ? 1 : 0];
      if (!ge && count > 0) {
        // first sweep runs eagerly (one-time kernel attribute set-up happens outside capture)
        sweep_body(do_eval);
        count--;
        cudaGraph_t g = nullptr;
        MG_CUDA(cudaStreamBeginCapture(s_, cudaStreamCaptureModeThreadLocal));
        const long long before = launches_;
        try {
          sweep_body(do_eval);
          graph_kernels_[do_eval ? 1 : 0] = launches_ - before;
          launches_ = before;
        } catch (...) {
          cudaStreamEndCapture(s_, &g);
          if (g) cudaGraphDestroy(g);
          throw;
        }
        MG_CUDA(cudaStreamEndCapture(s_, &g));
        MG_CUDA(cudaGraphInstantiate(&ge, g, 0));
        cudaGraphDestroy(g);
      }
      for (int i = 0; i < count; i++) MG_CUDA(cudaGraphLaunch(ge, s_));
      launches_ += graph_kernels_[do_eval ? 1 : 0] * count;
    } else {
      for (int i = 0; i < count; i++) sweep_body(do_eval);
    }
    if (sync) check_status();
  }

  void run() {
    init();
    if (cfg_.verbose) {
      if (adaptive_)  // AdaptiveGaussianNoise::getInitStatus (noisemodels.h:75)
        printf("Noise precision: adaptive (with max precision of %f)\nSampling\n",
               (sn_max_ + 1.0) / var_total_);
      else
        printf("Noise precision: %f (fixed)\nSampling\n", cfg_.precision);
      fflush(stdout);
    }
    const int total = burnin_ + nsamples_;
    for (int i = 0; i < total; i++) {
      const auto t0 = std::chrono::steady_clock::now();
      if (cfg_.verbose && i == burnin_)
        printf(" ====== Burn-in complete, averaging samples ====== \n");
      sweeps(i, 1, true, true);
      if (cfg_.verbose) {
        double r[2];
        get_rmse(r);
        const double took =
            std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        // AdaptiveGaussianNoise::getStatus (noisemodels.h:77-79): "Prec:" + alpha to 2 digits
        char prec[48] = "";
        if (adaptive_) {
          double nz[3];
          get_noise(nz);
          snprintf(prec, sizeof prec, "Prec:%.2g", nz[0]);
        }
        // NoiseModel::getEvalString (noisemodels.h:46): to_string_with_precision(rmse, 5), an
        // ostream at precision 5 in its default float format, which is printf's %.5g
        printf("Iter %3d: RMSE: %.5g (1samp: %.5g)  U:[%1.2e, %1.2e]\tSide:[%s, %s]%s [took %0.1fs]\n",
               i, r[0], r[1], latent_norm(0), latent_norm(1), link_norm_str(0).c_str(),
               link_norm_str(1).c_str(), prec, took);
        fflush(stdout);
      }
    }
  }

  double latent_norm(int mode) {
    std::vector<double> u((size_t)dims_[mode] * K_);
    get_latents(mode, u.data());
    double s = 0.0;
    for (double x : u) s += x * x;
    return std::sqrt(s);
  }
  std::string link_norm_str(int mode) {
    if (!prior_[mode].side()) return "nan";
    std::vector<double> b((size_t)prior_[mode].nfeat * K_);
    get_beta(mode, b.data());
    double s = 0.0;
    for (double x : b) s += x * x;
    char buf[32];
    snprintf(buf, sizeof buf, "%1.2e", std::sqrt(s));
    return buf;
  }

  // ---- state access ----
  void get_latents(int mode, double* out) {
    const long long N = dims_[mode];
    if (mixed_) {
      std::vector<float> h((size_t)N * KP_);
      MG_CUDA(cudaMemcpyAsync(h.data(), lat32_[mode].p, h.size() * 4, cudaMemcpyDeviceToHost, s_));
      g_d2h_bytes += (long long)h.size() * 4;
      MG_CUDA(cudaStreamSynchronize(s_));
      for (long long n = 0; n < N; n++)
        for (int k = 0; k < K_; k++) out[n * K_ + k] = h[n * KP_ + k];
    } else {
      MG_CUDA(cudaMemcpy2DAsync(out, K_ * 8, lat64_[mode].p, KP_ * 8, K_ * 8, N,
                                cudaMemcpyDeviceToHost, s_));
      g_d2h_bytes += (long long)N * K_ * 8;
      MG_CUDA(cudaStreamSynchronize(s_));
    }
  }
  void set_latents(int mode, const double* in) {
    const long long N = dims_[mode];
    if (mixed_) {
      std::vector<float> h((size_t)N * KP_, 0.f);
      for (long long n = 0; n < N; n++)
        for (int k = 0; k < K_; k++) h[n * KP_ + k] = (float)in[n * K_ + k];
      MG_CUDA(cudaMemcpyAsync(lat32_[mode].p, h.data(), h.size() * 4, cudaMemcpyHostToDevice, s_));
      // the 16-bit gather copy (BF16, or FP16 under that Gram precision), rounded on the device
      launch_copy16(lat32_[mode].p, lat16_[mode].p, (long long)N * KP_, gram_ == 1, s_);
    } else {
      MG_CUDA(cudaMemcpy2DAsync(lat64_[mode].p, KP_ * 8, in, K_ * 8, K_ * 8, N,
                                cudaMemcpyHostToDevice, s_));
    }
    MG_CUDA(cudaStreamSynchronize(s_));
  }
  void get_hyper(int mode, double* mu, double* Lambda, double* lb) {
    Prior& p = prior_[mode];
    if (mu) MG_CUDA(cudaMemcpyAsync(mu, p.mu.p, K_ * 8, cudaMemcpyDeviceToHost, s_));
    if (Lambda)
      MG_CUDA(cudaMemcpyAsync(Lambda, p.Lambda.p, (size_t)K_ * K_ * 8, cudaMemcpyDeviceToHost, s_));
    std::vector<double> lbv;
    if (lb) {
      if (p.macau) {
        MG_CUDA(cudaMemcpyAsync(lb, p.lambda_beta.p, 8, cudaMemcpyDeviceToHost, s_));
      } else if (p.one && p.lb_one.p) {
        lbv.resize(K_);
        MG_CUDA(cudaMemcpyAsync(lbv.data(), p.lb_one.p, K_ * 8, cudaMemcpyDeviceToHost, s_));
      } else {
        *lb = NAN;
      }
    }
    MG_CUDA(cudaStreamSynchronize(s_));
    // a univariate prior reports the mean over dimensions, like getLinkLambda (macauoneprior.h:46)
    if (!lbv.empty()) *lb = std::accumulate(lbv.begin(), lbv.end(), 0.0) / K_;
  }
  // lambda_beta of each dimension of a univariate prior (K values)
  void get_lambda_beta_one(int mode, double* out) {
    Prior& p = prior_[mode];
    if (!p.one) throw MgError(MG_ERR_STATE, "mode has no univariate prior");
    if (!initialised_) throw MgError(MG_ERR_STATE, "call mg_init first");
    MG_CUDA(cudaMemcpyAsync(out, p.lb_one.p, K_ * 8, cudaMemcpyDeviceToHost, s_));
    MG_CUDA(cudaStreamSynchronize(s_));
  }
  void set_hyper(int mode, const double* mu, const double* Lambda, const double* lb) {
    Prior& p = prior_[mode];
    if (mu) MG_CUDA(cudaMemcpyAsync(p.mu.p, mu, K_ * 8, cudaMemcpyHostToDevice, s_));
    if (Lambda)
      MG_CUDA(cudaMemcpyAsync(p.Lambda.p, Lambda, (size_t)K_ * K_ * 8, cudaMemcpyHostToDevice, s_));
    if (lb && p.macau) MG_CUDA(cudaMemcpyAsync(p.lambda_beta.p, lb, 8, cudaMemcpyHostToDevice, s_));
    std::vector<double> lbv(lb && p.one ? K_ : 0, lb ? *lb : 0.0);  // setLambdaBeta: every dim
    if (!lbv.empty() && p.lb_one.p)
      MG_CUDA(cudaMemcpyAsync(p.lb_one.p, lbv.data(), K_ * 8, cudaMemcpyHostToDevice, s_));
    MG_CUDA(cudaStreamSynchronize(s_));
  }
  void get_beta(int mode, double* out) {
    Prior& p = prior_[mode];
    if (!p.side()) throw MgError(MG_ERR_STATE, "mode has no side information");
    MG_CUDA(cudaMemcpy2DAsync(out, K_ * 8, p.beta.p, CP_ * 8, K_ * 8, p.nfeat,
                              cudaMemcpyDeviceToHost, s_));
    MG_CUDA(cudaStreamSynchronize(s_));
  }
  void get_uhat(int mode, double* out) {
    Prior& p = prior_[mode];
    if (!p.side()) throw MgError(MG_ERR_STATE, "mode has no side information");
    MG_CUDA(cudaMemcpy2DAsync(out, K_ * 8, p.uhat.p, KP_ * 8, K_ * 8, dims_[mode],
                              cudaMemcpyDeviceToHost, s_));
    MG_CUDA(cudaStreamSynchronize(s_));
  }
  void get_rmse(double* r) {
    if (ntest_ == 0) {
      r[0] = r[1] = NAN;
      return;
    }
    MG_CUDA(cudaMemcpyAsync(r, rmse_.p, 16, cudaMemcpyDeviceToHost, s_));
    g_d2h_bytes += 16;
    MG_CUDA(cudaStreamSynchronize(s_));
  }
  void get_predictions(double* out) {
    if (ntest_ == 0) return;
    MG_CUDA(cudaMemcpyAsync(out, pred_.p, ntest_ * 8, cudaMemcpyDeviceToHost, s_));
    g_d2h_bytes += ntest_ * 8;
    MG_CUDA(cudaStreamSynchronize(s_));
  }
  // MacauX::getStds (macau.cpp:175-188)
  void get_stds(double* out) {
    if (ntest_ == 0) return;
    if (nsamples_ <= 1) {
      for (long long i = 0; i < ntest_; i++) out[i] = NAN;
      return;
    }
    MG_CUDA(cudaMemcpyAsync(out, pvar_.p, ntest_ * 8, cudaMemcpyDeviceToHost, s_));
    g_d2h_bytes += ntest_ * 8;
    MG_CUDA(cudaStreamSynchronize(s_));
    const double inorm = 1.0 / (nsamples_ - 1);
    for (long long i = 0; i < ntest_; i++) out[i] = std::sqrt(out[i] * inorm);
  }
  void get_test_data(double* out) {
    if (ntest_ == 0) return;
    std::vector<int> r((size_t)ntest_), c((size_t)ntest_);
    MG_CUDA(cudaMemcpyAsync(r.data(), trow_.p, ntest_ * 4, cudaMemcpyDeviceToHost, s_));
    MG_CUDA(cudaMemcpyAsync(c.data(), tcol_.p, ntest_ * 4, cudaMemcpyDeviceToHost, s_));
    MG_CUDA(cudaMemcpyAsync(out + 2 * ntest_, tval_.p, ntest_ * 8, cudaMemcpyDeviceToHost, s_));
    g_d2h_bytes += ntest_ * 16;
    MG_CUDA(cudaStreamSynchronize(s_));
    for (long long i = 0; i < ntest_; i++) {
      out[i] = r[i];
      out[i + ntest_] = c[i];
    }
  }
  void get_stats(mg_stats* st) {
    Ctl h;
    MG_CUDA(cudaMemcpyAsync(&h, ctl_.p, sizeof(Ctl), cudaMemcpyDeviceToHost, s_));
    MG_CUDA(cudaStreamSynchronize(s_));
    std::memset(st, 0, sizeof(*st));
    st->sweeps = (double)sweeps_done_;
    st->seconds_sample = t_sample_;
    st->seconds_prior = t_prior_;
    st->seconds_eval = t_eval_;
    st->retries[0] = h.retries[0];
    st->retries[1] = h.retries[1];
    st->rows_sampled[0] = rows_[0];
    st->rows_sampled[1] = rows_[1];
    st->cg_iters[0] = prior_[0].cg_iters;
    st->cg_iters[1] = prior_[1].cg_iters;
    st->graph_captured = (graph_[0] || graph_[1]) ? 1 : 0;
    st->kernel_launches = launches_;
    st->h2d_bytes = g_h2d_bytes;
    st->d2h_bytes = g_d2h_bytes;
    st->ntasks[0] = md_[0].ntasks;
    st->ntasks[1] = md_[1].ntasks;
    st->nnz[0] = md_[0].nnz;
    st->nnz[1] = md_[1].nnz;
  }
  void dims(int64_t* nrow, int64_t* ncol, int64_t* ntrain, int64_t* ntest, double* mean) {
    if (nrow) *nrow = dims_[0];
    if (ncol) *ncol = dims_[1];
    if (ntrain) *ntrain = ntrain_;
    if (ntest) *ntest = ntest_;
    if (mean) *mean = mean_;
  }

  void count_rows(int mode) { rows_[mode] += md_[mode].N; }
  cudaStream_t stream() const { return s_; }
  Ctl* ctl() const { return ctl_.p; }
  int K() const { return K_; }
  int KP() const { return KP_; }
  long long dim(int m) const { return dims_[m]; }
  bool initialised() const { return initialised_; }
  void set_use_graph(bool b) { use_graph_ = b; drop_graphs(); }
  void set_use_tc(bool b) { use_tc_ = b; drop_graphs(); }
  void set_row_range(int mode, long long lo, long long hi) {
    if (mode < 0 || mode > 1) throw MgError(MG_ERR_ARG, "mode must be 0 or 1");
    if (!have_data_) throw MgError(MG_ERR_STATE, "set the training data before a row range");
    if (lo < 0 || hi < lo || hi > dims_[mode])
      throw MgError(MG_ERR_ARG, "row range must satisfy 0 <= lo <= hi <= rows of the mode");
    if (prior_[mode].one)
      throw MgError(MG_ERR_ARG, "row ranges are not supported with the univariate prior");
    range_lo_[mode] = lo;
    range_hi_[mode] = hi;
    drop_graphs();
    build_tasks(mode, md_[mode].thr);
    MG_CUDA(cudaStreamSynchronize(s_));
  }
  // Device buffer of a mode's latents as the samplers write them: N rows of KP values, FP64
  // (FP64 mode) or the FP32 master (mixed mode).
  void latents_device(int mode, void** ptr, int* row_stride, int* elem_bytes) const {
    if (!initialised_) throw MgError(MG_ERR_STATE, "call mg_init first");
    if (ptr) *ptr = mixed_ ? (void*)lat32_[mode].p : (void*)lat64_[mode].p;
    if (row_stride) *row_stride = KP_;
    if (elem_bytes) *elem_bytes = mixed_ ? 4 : 8;
  }
  // Rows of the buffer above were written from outside (an exchange between ranks): refresh
  // what the samplers derive from it (mixed mode: the 16-bit gather copy).  Ordered on the
  // context's stream.
  void latents_changed(int mode) {
    if (!initialised_) throw MgError(MG_ERR_STATE, "call mg_init first");
    if (mixed_)
      launch_copy16(lat32_[mode].p, lat16_[mode].p, dims_[mode] * (long long)KP_, gram_ == 1, s_);
  }
  void set_tc_wait(int us) {
    if (us < 0) throw MgError(MG_ERR_ARG, "tc_wait_us must be >= 0");
    tc_wait_cycles_ = 2000LL * us;
    drop_graphs();
  }
  void set_cg_max_iter(int n) {
    if (n < 1) throw MgError(MG_ERR_ARG, "cg_max_iter must be >= 1");
    cg_max_iter_ = n;
  }
  void set_tc_wait_test(bool b) {
    tc_wait_test_ = b;
    drop_graphs();
  }
  void set_fused(bool b) {
    fused_ = b;
    drop_graphs();
    if (have_data_)
      for (int m = 0; m < 2; m++) size_gram_records(m);
  }
  void set_cg_f32(bool b) { cg_f32_ = b && mixed_; }
  // A fixed work split / CTA shape for both modes' row samplers (the autotuner's knobs).
  void set_split_threshold(int t) {
    if (!have_data_) throw MgError(MG_ERR_STATE, "set the training data before split_threshold");
    if (t < 256 || t > 16384) throw MgError(MG_ERR_ARG, "split_threshold must be in [256, 16384]");
    drop_graphs();
    for (int m = 0; m < 2; m++) {
      build_tasks(m, t);
      md_[m].tune_state = 0;
    }
    MG_CUDA(cudaStreamSynchronize(s_));
  }
  // Order of the tensor-core sampler's row groups: 0 = by descending length, n > 0 = long and
  // short groups interleaved with a finished row counted as n k-blocks (interleave_groups).
  void set_group_mix(int v) {
    if (v < 0 || v > 64) throw MgError(MG_ERR_ARG, "group_mix must be in [0, 64]");
    group_mix_ = v;
    if (!have_data_) return;
    drop_graphs();
    for (int m = 0; m < 2; m++) build_tasks(m, md_[m].thr);
    MG_CUDA(cudaStreamSynchronize(s_));
  }
  void set_cta_groups(int g) {
    const std::vector<int> opts = sample_group_options(KP_, mixed_, gram_);
    if (g != 0 && std::find(opts.begin(), opts.end(), g) == opts.end())
      throw MgError(MG_ERR_ARG, "cta_groups not offered for this K and precision");
    drop_graphs();
    for (int m = 0; m < 2; m++) {
      md_[m].groups = g;
      md_[m].tune_state = 0;
    }
  }
  void set_autotune(int v) {
    if (v < 0 || v > 2) throw MgError(MG_ERR_ARG, "autotune must be 0, 1 or 2");
    autotune_ = v;
  }
  void set_gram(int g) {
    if (g < 0 || g > 2) throw MgError(MG_ERR_ARG, "gram_precision must be 0 (BF16), 1 (FP16) or 2 (TF32)");
    if (!mixed_ && g != 0) throw MgError(MG_ERR_ARG, "gram_precision applies to mixed mode");
    gram_ = g;
    drop_graphs();
    initialised_ = false;
  }

  std::string err;

 private:
  void drop_graphs() {
    for (auto& g : graph_)
      if (g) {
        cudaGraphExecDestroy(g);
        g = nullptr;
      }
  }

  // Derived layouts of mode m from its device CSR (md.ptr / idx / val, nnz entries) and a host
  // copy of its row pointers: packed entries, task lists, the padded copy.
  void upload_mode(int m, const std::vector<long long>& hptr, long long nnz) {
    ModeData& md = md_[m];
    md.N = dims_[m];
    md.nnz = nnz;
    md.hptr = hptr;
    if (mixed_) md.packed.alloc((size_t)std::max(1LL, nnz));
    md.max_len = 0;
    for (long long r = 0; r < md.N; r++) md.max_len = std::max(md.max_len, hptr[r + 1] - hptr[r]);
    if (mixed_ && KP_ == 32) {
      // padded copy for the tensor-core sampler: rows at 16-entry boundaries, sentinel padding
      std::vector<long long> pptr(md.N + 1, 0);
      for (long long r = 0; r < md.N; r++)
        pptr[r + 1] = pptr[r] + (hptr[r + 1] - hptr[r] + 15) / 16 * 16;
      md.pptr_tc.upload(pptr.data(), pptr.size(), s_);
      md.packed_tc.alloc((size_t)std::max(1LL, pptr[md.N]));
    }
    md.groups = 0;
    md.tune_state = 0;
    long long thr = split_divisor_thr(m, 2);
    if (autotune_ == 1) {  // a cached choice for this data: build its task lists right away
      TuneChoice c;
      if (TuneCache::get().find(tune_key(tune_kind(m), K_, num_sms_, md.hptr), &c)) {
        thr = c.thr;
        md.groups = c.groups;
        md.tune = c;
        md.tune_state = 2;
      }
    }
    build_tasks(m, thr);
    pack_mode(m);
    MG_CUDA(cudaStreamSynchronize(s_));
  }

  // Split threshold nnz / (div * row groups), row groups = 16 per SM, clamped to [256, 16384]:
  // div = 2 is the default; the autotuner tries 1 to 16.
  long long split_divisor_thr(int m, int div) const {
    const long long groups = (long long)num_sms_ * 16;
    return std::max(256LL, std::min(16384LL, md_[m].nnz / (div * groups)));
  }

  // Task lists of mode m at split threshold thr: rows sorted by descending length, rows above
  // the threshold cut into near-equal parts so that no task is much longer than the average
  // work per row group (the CUDA-core list; for the tensor-core sampler the 16-entry aligned
  // list over the padded copy, with its split-row table); split counters and the shared
  // split-part scratch sized to match.
  void build_tasks(int m, long long thr) {
    ModeData& md = md_[m];
    const std::vector<long long>& hptr = md.hptr;
    md.thr = thr;
    int nsplit = 0, nslots = 0;
    std::vector<RowTask> tasks = make_tasks(hptr, thr, 1, nsplit, nslots, range_lo_[m],
                                            range_hi_[m]);
    md.ntasks = (int)tasks.size();
    md.nsplit = nsplit;
    md.nslots = nslots;
    md.tasks.upload(tasks.data(), tasks.size(), s_);
    if (mixed_ && KP_ == 32) {
      std::vector<long long> pptr(md.N + 1, 0);
      for (long long r = 0; r < md.N; r++)
        pptr[r + 1] = pptr[r] + (hptr[r + 1] - hptr[r] + 15) / 16 * 16;
      const long long thr16 = (thr + 15) / 16 * 16;
      int ns = 0, nsl = 0;
      std::vector<RowTask> tt = make_tasks(pptr, thr16, 16, ns, nsl, range_lo_[m], range_hi_[m]);
      if (group_mix_ > 0) interleave_groups(tt, (double)group_mix_);
      md.ntasks_tc = (int)tt.size();
      md.nsplit_tc = ns;
      md.nslots_tc = nsl;
      md.tasks_tc.upload(tt.data(), tt.size(), s_);
      std::vector<int4> sr;
      for (const RowTask& t : tt)
        if (t.nparts > 1 && t.part == 0) sr.push_back(make_int4(t.row, t.nparts, t.slot, 0));
      std::sort(sr.begin(), sr.end(), [](const int4& a, const int4& b) { return a.x < b.x; });
      md.split_tc.upload(sr.data(), sr.size(), s_);
      size_gram_records(m);
    }
    md.split_cnt.alloc_zero(std::max(1, nsplit), s_);
    const size_t need =
        (size_t)std::max(std::max(md_[0].nslots, md_[1].nslots),
                         std::max(md_[0].nslots_tc, md_[1].nslots_tc)) *
        (KP_ * KP_ + KP_);
    if (need > scratch_.n) scratch_.alloc(need);
    if (mixed_ && KP_ == 32 && retry_work_.n == 0) retry_work_.alloc(tc_retry_work_doubles(num_sms_));
  }

  // Gram records of the tensor-core sampler of mode m: one per split row when the fused kernel
  // finishes the mode's rows, one per row when a separate finish kernel reads them (option
  // "fused_finish" = 0, or the univariate prior).  Kept when large enough.
  void size_gram_records(int m) {
    ModeData& md = md_[m];
    if (!(mixed_ && KP_ == 32) || md.N == 0) return;
    const bool per_row = !fused_ || prior_[m].one;
    const size_t need = (size_t)std::max(1LL, per_row ? md.N : (long long)md.nsplit_tc) *
                        (32 * 32 + 32);
    if (md.gram_tc.n < need) md.gram_tc.alloc(need);
  }

  // Mixed mode: the packed (index, weight) entries of mode m and their padded copy.  The weights
  // are (y - mean) * alpha under fixed noise and (y - mean) under adaptive noise, whose precision
  // the samplers apply from the device as they read them.
  void pack_mode(int m) {
    ModeData& md = md_[m];
    if (!mixed_) return;
    launch_pack(md.idx.p, md.val.p, md.nnz, mean_, adaptive_ ? 1.0 : cfg_.precision,
                md.packed.p, s_);
    if (KP_ == 32)
      launch_pad(md.ptr.p, md.pptr_tc.p, md.N, md.packed.p, (unsigned)dims_[1 - m],
                 md.packed_tc.p, s_);
  }

  mg_config cfg_;
  int K_ = 0, KP_ = 0, CP_ = 32;
  bool mixed_ = false;
  int dev_ = 0, num_sms_ = 148;
  cudaStream_t s_ = nullptr;
  cudaEvent_t ev0_ = nullptr, ev1_ = nullptr;
  long long dims_[2] = {0, 0};
  long long ntrain_ = 0, ntest_ = 0;
  double mean_ = 0.0;
  // AdaptiveGaussianNoise (noisemodels.h:50-86): var_total of the training values, the cap of
  // the precision, and sn_init / sn_max; the current precision lives in Ctl::alpha
  bool adaptive_ = false;
  double sn_init_ = 1.0, sn_max_ = 10.0, var_total_ = 1.0, alpha_max_ = 0.0;
  DBuf<int> erow_;                // row of each mode-0 entry (residual sum of the noise update)
  DBuf<double> noise_partials_;
  bool have_data_ = false, initialised_ = false;
  bool use_graph_ = true, use_tc_ = true;
  // Rows of each mode this context samples (mg_set_row_range): [lo, hi), hi < 0 = all rows.
  // The split threshold is the one of the whole mode, so a row's arithmetic does not depend on
  // the range.
  long long range_lo_[2] = {0, 0}, range_hi_[2] = {-1, -1};
  // The tensor-core sampler finishes rows in its Gram kernel's epilogue (option "fused_finish",
  // default on); off: Gram records in HBM and a separate finish kernel.
  bool fused_ = true;
  // Row-group order of the tensor-core sampler (option "group_mix", set_group_mix).
  int group_mix_ = 16;
  // Clock budget of each barrier wait of the tensor-core sampler (option "tc_wait_us", in
  // microseconds at 2 GHz; 0 = the kernel's default of about 2 s).  Tests shorten it to make a
  // wait run out.
  long long tc_wait_cycles_ = 0;
  // Option "tc_wait_test" (tests only): the tensor-core sampler's MMA warp first waits on a
  // barrier that nothing arrives on, so that the wait runs out and the launch aborts.
  bool tc_wait_test_ = false;
  // Block-CG in FP32 with FP64 residual replacement (mixed mode, option "cg_fp32").  Off by
  // default: at tol 1e-6 the FP32 iteration needs about 1.5x the iterations of FP64, which
  // costs more than its halved gather traffic saves.
  bool cg_f32_ = false;
  // Block-CG iteration cap per solve (option "cg_max_iter"; the reference's 100,000,
  // linop.h:279) and whether a solve since the last status check reached it.
  int cg_max_iter_ = 100000;
  bool cg_noconv_ = false;
  // Autotuning at mg_init (option "autotune"): 0 off, 1 on with the choice cache, 2 on and
  // always timed
  int autotune_ = 0;
  // Gram precision of the mixed samplers (option "gram_precision"): 0 BF16 gathers (the
  // tensor-core sampler at K = 32), 1 FP16 gathers, 2 FP32 master rounded to TF32 as gathered;
  // 1 and 2 run the CUDA-core sampler at every K
  int gram_ = 0;
  int burnin_ = 50, nsamples_ = 400;
  ModeData md_[2];
  Prior prior_[2];
  DBuf<double> lat64_[2];
  DBuf<float> lat32_[2];
  DBuf<__nv_bfloat16> lat16_[2];
  DBuf<double> scratch_, stat_partials_, stat_final_, nwbuf_;
  DBuf<double> stat_partials1_, stat_final1_;  // mode 1's work of update_priors_pair
  DBuf<double> retry_work_;  // the fused tensor-core sampler's FP64-redo work areas
  NwWork nw_{};
  DBuf<Ctl> ctl_;
  DBuf<int> trow_, tcol_;
  DBuf<double> tval_, pred_, pvar_, eval_partials_, rmse_;
  cudaGraphExec_t graph_[2] = {nullptr, nullptr};
  long long retries_[2] = {0, 0}, rows_[2] = {0, 0};
  long long sweeps_done_ = 0;
  long long launches_ = 0;
  long long graph_kernels_[2] = {0, 0};
  double t_sample_ = 0, t_prior_ = 0, t_eval_ = 0;
};

}  // namespace mg

// ============================== C ABI ==============================
struct mg_ctx {
  std::unique_ptr<mg::Context> c;
  std::string err;
};

namespace {
thread_local std::string g_create_error;

template <typename F>
int guarded(mg_ctx* ctx, F&& f) {
  if (!ctx || !ctx->c) return MG_ERR_ARG;
  try {
    f(*ctx->c);
    ctx->err.clear();
    return MG_OK;
  } catch (const mg::MgError& e) {
    ctx->err = e.what();
    return e.code;
  } catch (const mg::CudaError& e) {
    ctx->err = e.what();
    return MG_ERR_CUDA;
  } catch (const std::exception& e) {
    ctx->err = e.what();
    return MG_ERR_ARG;
  }
}
}  // namespace

extern "C" {

int mg_create(mg_ctx** out, const mg_config* cfg) {
  if (!out || !cfg) return MG_ERR_ARG;
  *out = nullptr;
  try {
    auto* h = new mg_ctx();
    h->c.reset(new mg::Context(*cfg));
    *out = h;
    return MG_OK;
  } catch (const mg::MgError& e) {
    g_create_error = e.what();
    return e.code;
  } catch (const std::exception& e) {
    g_create_error = e.what();
    return MG_ERR_CUDA;
  }
}

void mg_destroy(mg_ctx* ctx) { delete ctx; }

const char* mg_last_error(const mg_ctx* ctx) {
  if (!ctx) return g_create_error.c_str();
  return ctx->err.c_str();
}

int mg_set_relation_data(mg_ctx* ctx, const int32_t* idx, int nmodes, const double* values,
                         int64_t nnz, const int32_t* dims) {
  if (!idx || !values || !dims) return MG_ERR_ARG;
  return guarded(ctx, [&](mg::Context& c) { c.set_train(idx, nmodes, values, nnz, dims); });
}

int mg_set_relation_data_test(mg_ctx* ctx, const int32_t* idx, int nmodes,
                              const double* values, int64_t nnz, const int32_t* dims) {
  if ((nnz > 0 && (!idx || !values)) || !dims) return MG_ERR_ARG;
  return guarded(ctx, [&](mg::Context& c) { c.set_test(idx, nmodes, values, nnz, dims); });
}

int mg_set_relation_data_rc(mg_ctx* ctx, const int32_t* rows, const int32_t* cols,
                            const double* values, int64_t nnz, int nrows, int ncols) {
  if (!rows || !cols || !values || nrows < 1 || ncols < 1) return MG_ERR_ARG;
  return guarded(ctx, [&](mg::Context& c) { c.set_train(rows, cols, values, nnz, nrows, ncols); });
}

int mg_set_relation_data_test_rc(mg_ctx* ctx, const int32_t* rows, const int32_t* cols,
                                 const double* values, int64_t nnz, int nrows, int ncols) {
  if ((nnz > 0 && (!rows || !cols || !values)) || nrows < 1 || ncols < 1) return MG_ERR_ARG;
  const int32_t dims[2] = {nrows, ncols};
  return guarded(ctx, [&](mg::Context& c) { c.set_test(rows, cols, values, nnz, dims); });
}

int mg_set_side(mg_ctx* ctx, int mode, const int32_t* rows, const int32_t* cols,
                const double* vals, int64_t nnz, int nrows, int nfeat, double lambda_beta,
                double tol) {
  if ((nnz > 0 && (!rows || !cols)) || nfeat < 1) return MG_ERR_ARG;
  return guarded(ctx, [&](mg::Context& c) {
    c.set_side(mode, rows, cols, vals, nnz, nrows, nfeat, lambda_beta, tol);
  });
}

int mg_set_side_univariate(mg_ctx* ctx, int mode, const int32_t* rows, const int32_t* cols,
                           const double* vals, int64_t nnz, int nrows, int nfeat,
                           double lambda_beta) {
  if ((nnz > 0 && (!rows || !cols)) || nfeat < 1) return MG_ERR_ARG;
  return guarded(ctx, [&](mg::Context& c) {
    c.set_side(mode, rows, cols, vals, nnz, nrows, nfeat, lambda_beta, 1e-6, true);
  });
}

int mg_get_lambda_beta_univariate(mg_ctx* ctx, int mode, double* out) {
  if (mode < 0 || mode > 1 || !out) return MG_ERR_ARG;
  return guarded(ctx, [&](mg::Context& c) { c.get_lambda_beta_one(mode, out); });
}

int mg_set_samples(mg_ctx* ctx, int burnin, int nsamples) {
  if (burnin < 0 || nsamples < 0) return MG_ERR_ARG;
  return guarded(ctx, [&](mg::Context& c) { c.set_samples(burnin, nsamples); });
}

int mg_init(mg_ctx* ctx) {
  return guarded(ctx, [&](mg::Context& c) { c.init(); });
}

int mg_sweep(mg_ctx* ctx, int iter, int eval) {
  return guarded(ctx, [&](mg::Context& c) { c.sweeps(iter, 1, eval != 0, true); });
}

int mg_sweeps(mg_ctx* ctx, int first_iter, int count, int eval) {
  if (count < 0) return MG_ERR_ARG;
  return guarded(ctx, [&](mg::Context& c) { c.sweeps(first_iter, count, eval != 0, true); });
}

int mg_time_sweeps(mg_ctx* ctx, int first_iter, int count, int eval, int phase_events,
                   double* total_seconds, double* phase_seconds) {
  if (count < 1) return MG_ERR_ARG;
  return guarded(ctx, [&](mg::Context& c) {
    c.time_sweeps(first_iter, count, eval != 0, phase_events != 0, total_seconds, phase_seconds);
  });
}

int mg_run(mg_ctx* ctx) {
  return guarded(ctx, [&](mg::Context& c) { c.run(); });
}

int mg_sample_latents(mg_ctx* ctx, int mode, int iter, const double* z) {
  if (mode < 0 || mode > 1) return MG_ERR_ARG;
  return guarded(ctx, [&](mg::Context& c) {
    if (!c.initialised()) throw mg::MgError(MG_ERR_STATE, "call mg_init first");
    mg::launch_set_sweep(c.ctl(), (uint32_t)iter, 0, c.stream());
    double* zd = nullptr;
    const size_t bytes = (size_t)c.dim(mode) * c.K() * sizeof(double);
    if (z) {
      MG_CUDA(cudaMalloc(&zd, bytes));
      MG_CUDA(cudaMemcpyAsync(zd, z, bytes, cudaMemcpyHostToDevice, c.stream()));
    }
    try {
      c.sample(mode, zd);
      c.count_rows(mode);
      c.check_status();
    } catch (...) {
      if (zd) cudaFree(zd);
      throw;
    }
    if (zd) {
      MG_CUDA(cudaStreamSynchronize(c.stream()));
      cudaFree(zd);
    }
  });
}

int mg_update_prior(mg_ctx* ctx, int mode, int iter) {
  if (mode < 0 || mode > 1) return MG_ERR_ARG;
  return guarded(ctx, [&](mg::Context& c) {
    if (!c.initialised()) throw mg::MgError(MG_ERR_STATE, "call mg_init first");
    mg::launch_set_sweep(c.ctl(), (uint32_t)iter, 0, c.stream());
    c.update_prior(mode);
    c.check_status();
  });
}

int mg_set_noise_adaptive(mg_ctx* ctx, double sn_init, double sn_max) {
  return guarded(ctx, [&](mg::Context& c) { c.set_noise_adaptive(sn_init, sn_max); });
}

int mg_update_noise(mg_ctx* ctx, int iter) {
  return guarded(ctx, [&](mg::Context& c) {
    if (!c.initialised()) throw mg::MgError(MG_ERR_STATE, "call mg_init first");
    mg::launch_set_sweep(c.ctl(), (uint32_t)iter, 0, c.stream());
    c.update_noise();
    c.check_status();
  });
}

int mg_get_noise(mg_ctx* ctx, double* out) {
  if (!out) return MG_ERR_ARG;
  return guarded(ctx, [&](mg::Context& c) { c.get_noise(out); });
}

int mg_eval(mg_ctx* ctx, int n) {
  if (n < 0) return MG_ERR_ARG;
  return guarded(ctx, [&](mg::Context& c) {
    c.eval(n);
    c.check_status();
  });
}

int mg_get_latents(mg_ctx* ctx, int mode, double* out) {
  if (mode < 0 || mode > 1 || !out) return MG_ERR_ARG;
  return guarded(ctx, [&](mg::Context& c) { c.get_latents(mode, out); });
}
int mg_set_row_range(mg_ctx* ctx, int mode, int64_t lo, int64_t hi) {
  return guarded(ctx, [&](mg::Context& c) { c.set_row_range(mode, lo, hi); });
}

int mg_latents_device(mg_ctx* ctx, int mode, void** ptr, int* row_stride, int* elem_bytes) {
  if (mode < 0 || mode > 1) return MG_ERR_ARG;
  return guarded(ctx, [&](mg::Context& c) { c.latents_device(mode, ptr, row_stride, elem_bytes); });
}

int mg_latents_changed(mg_ctx* ctx, int mode) {
  if (mode < 0 || mode > 1) return MG_ERR_ARG;
  return guarded(ctx, [&](mg::Context& c) { c.latents_changed(mode); });
}

int mg_get_stream(mg_ctx* ctx, void** stream) {
  if (!stream) return MG_ERR_ARG;
  return guarded(ctx, [&](mg::Context& c) { *stream = (void*)c.stream(); });
}

int mg_set_latents(mg_ctx* ctx, int mode, const double* in) {
  if (mode < 0 || mode > 1 || !in) return MG_ERR_ARG;
  return guarded(ctx, [&](mg::Context& c) {
    if (!c.initialised()) throw mg::MgError(MG_ERR_STATE, "call mg_init first");
    c.set_latents(mode, in);
  });
}
int mg_get_hyper(mg_ctx* ctx, int mode, double* mu, double* Lambda, double* lambda_beta) {
  if (mode < 0 || mode > 1) return MG_ERR_ARG;
  return guarded(ctx, [&](mg::Context& c) { c.get_hyper(mode, mu, Lambda, lambda_beta); });
}
int mg_set_hyper(mg_ctx* ctx, int mode, const double* mu, const double* Lambda,
                 const double* lambda_beta) {
  if (mode < 0 || mode > 1) return MG_ERR_ARG;
  return guarded(ctx, [&](mg::Context& c) { c.set_hyper(mode, mu, Lambda, lambda_beta); });
}
int mg_get_beta(mg_ctx* ctx, int mode, double* beta) {
  if (mode < 0 || mode > 1 || !beta) return MG_ERR_ARG;
  return guarded(ctx, [&](mg::Context& c) { c.get_beta(mode, beta); });
}
int mg_get_uhat(mg_ctx* ctx, int mode, double* uhat) {
  if (mode < 0 || mode > 1 || !uhat) return MG_ERR_ARG;
  return guarded(ctx, [&](mg::Context& c) { c.get_uhat(mode, uhat); });
}
int mg_get_dims(mg_ctx* ctx, int64_t* nrow, int64_t* ncol, int64_t* ntrain, int64_t* ntest,
                double* mean_value) {
  return guarded(ctx, [&](mg::Context& c) { c.dims(nrow, ncol, ntrain, ntest, mean_value); });
}
int mg_get_rmse(mg_ctx* ctx, double* rmse) {
  if (!rmse) return MG_ERR_ARG;
  return guarded(ctx, [&](mg::Context& c) { c.get_rmse(rmse); });
}
int mg_get_predictions(mg_ctx* ctx, double* out) {
  return guarded(ctx, [&](mg::Context& c) { c.get_predictions(out); });
}
int mg_get_stds(mg_ctx* ctx, double* out) {
  return guarded(ctx, [&](mg::Context& c) { c.get_stds(out); });
}
int mg_get_test_data(mg_ctx* ctx, double* out) {
  return guarded(ctx, [&](mg::Context& c) { c.get_test_data(out); });
}
int mg_get_stats(mg_ctx* ctx, mg_stats* out) {
  if (!out) return MG_ERR_ARG;
  return guarded(ctx, [&](mg::Context& c) { c.get_stats(out); });
}

int mg_set_option(mg_ctx* ctx, const char* name, int value) {
  if (!name) return MG_ERR_ARG;
  return guarded(ctx, [&](mg::Context& c) {
    const std::string n(name);
    if (n == "graph") c.set_use_graph(value != 0);
    else if (n == "tensor_core_gram") c.set_use_tc(value != 0);
    else if (n == "fused_finish") c.set_fused(value != 0);
    else if (n == "tc_wait_us") c.set_tc_wait(value);
    else if (n == "tc_wait_test") c.set_tc_wait_test(value != 0);
    else if (n == "cg_fp32") c.set_cg_f32(value != 0);
    else if (n == "cg_max_iter") c.set_cg_max_iter(value);
    else if (n == "gram_precision") c.set_gram(value);
    else if (n == "autotune") c.set_autotune(value);
    else if (n == "split_threshold") c.set_split_threshold(value);
    else if (n == "cta_groups") c.set_cta_groups(value);
    else if (n == "group_mix") c.set_group_mix(value);
    else throw mg::MgError(MG_ERR_ARG, "unknown option " + n);
  });
}

int mg_autotune(mg_ctx* ctx, int use_cache) {
  return guarded(ctx, [&](mg::Context& c) { c.autotune(use_cache != 0); });
}

int mg_get_tuning(mg_ctx* ctx, int mode, mg_tuning* out) {
  if (!out) return MG_ERR_ARG;
  return guarded(ctx, [&](mg::Context& c) { c.get_tuning(mode, out); });
}

int mg_blockcg(const int32_t* rows, const int32_t* cols, const double* vals, int64_t nnz,
               int nrows, int nfeat, const double* B, int nrhs, double reg, double tol,
               int compute, double* X, int* niter, double* seconds) {
  if (!rows || !cols || !B || !X || nrhs < 1 || nfeat < 1 || nrows < 1) return MG_ERR_ARG;
  try {
    for (int64_t e = 0; e < nnz; e++)
      if (rows[e] < 0 || rows[e] >= nrows || cols[e] < 0 || cols[e] >= nfeat) return MG_ERR_ARG;
    int dev = 0;
    MG_CUDA(cudaGetDevice(&dev));
    cudaStream_t s;
    MG_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    mg::HostCsr f = mg::coo_to_csr(rows, cols, vals, nnz, nrows, nfeat);
    mg::HostCsr t = mg::transpose(f, nrows, nfeat);
    mg::DBuf<long long> fp, tp;
    mg::DBuf<int> fi, ti;
    mg::DBuf<double> fv, tv, Bd, Xd;
    mg::DBuf<float> fvf, tvf;
    mg::DBuf<mg::Ctl> ctl;
    fp.upload(f.ptr.data(), f.ptr.size(), s);
    fi.upload(f.idx.data(), f.idx.size(), s);
    tp.upload(t.ptr.data(), t.ptr.size(), s);
    ti.upload(t.idx.data(), t.idx.size(), s);
    mg::DevCsr F, Ft;
    F.ptr = fp.p; F.idx = fi.p; F.nrow = nrows; F.ncol = nfeat; F.nnz = (long long)f.idx.size();
    Ft.ptr = tp.p; Ft.idx = ti.p; Ft.nrow = nfeat; Ft.ncol = nrows; Ft.nnz = F.nnz;
    int nsm = 148;
    MG_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    mg::SpmmSplit fs, ts;
    fs.build(f.ptr, nsm, s, F);
    ts.build(t.ptr, nsm, s, Ft);
    if (vals) {
      fv.upload(f.val.data(), f.val.size(), s);
      tv.upload(t.val.data(), t.val.size(), s);
      std::vector<float> a(f.val.begin(), f.val.end()), b(t.val.begin(), t.val.end());
      fvf.upload(a.data(), a.size(), s);
      tvf.upload(b.data(), b.size(), s);
      F.val = fv.p; F.valf = fvf.p; Ft.val = tv.p; Ft.valf = tvf.p;
    }
    // B is nrhs x nfeat column-major == nfeat rows of nrhs values
    Bd.upload(B, (size_t)nrhs * nfeat, s);
    Xd.alloc_zero((size_t)nrhs * nfeat, s);
    ctl.alloc_zero(1, s);
    mg::BlockCg cg;
    cudaEvent_t e0, e1;
    MG_CUDA(cudaEventCreate(&e0));
    MG_CUDA(cudaEventCreate(&e1));
    MG_CUDA(cudaEventRecord(e0, s));
    const int it = cg.solve(F, Ft, reg, nullptr, Bd.p, nrhs, nrhs, tol, Xd.p, nrhs, ctl.p, s,
                            compute == MG_COMPUTE_MIXED);
    MG_CUDA(cudaEventRecord(e1, s));
    MG_CUDA(cudaMemcpyAsync(X, Xd.p, sizeof(double) * nrhs * nfeat, cudaMemcpyDeviceToHost, s));
    mg::Ctl h;
    MG_CUDA(cudaMemcpyAsync(&h, ctl.p, sizeof(h), cudaMemcpyDeviceToHost, s));
    MG_CUDA(cudaStreamSynchronize(s));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaStreamDestroy(s);
    if (niter) *niter = it;
    if (seconds) *seconds = ms * 1e-3;
    if (h.status & mg::kStatCgFail) {
      g_create_error = "block-CG breakdown";
      return MG_ERR_CG;
    }
    if (!cg.converged()) {  // X holds the last iterate
      g_create_error = "block-CG did not converge within " + std::to_string(cg.max_iter()) +
                       " iterations";
      return MG_ERR_CG;
    }
    return MG_OK;
  } catch (const mg::MgError& e) {
    g_create_error = e.what();
    return e.code;
  } catch (const std::exception& e) {
    g_create_error = e.what();
    return MG_ERR_CUDA;
  }
}

}  // extern "C"
