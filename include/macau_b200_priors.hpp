// Adapters that put the sm_100a library behind the reference's own C++ interfaces, so that a C++
// host written against jaak-s/macau switches to the GPU by constructing different objects:
//
//   GpuBPMFPrior   implements ILatentPrior (lib/macau-cpp/latentprior.h:17-49) for a mode without
//                  side information, in place of BPMFPrior (latentprior.h:53-79);
//   GpuMacauPrior  implements ILatentPrior for a mode with sparse side information, in place of
//                  MacauPrior<SparseDoubleFeat> (latentprior.h:82-125; F given as COO arrays, NULL
//                  values = binary, like make_prior in macau.pyx:154-192);
//   MacauGpuX      implements Macau (lib/macau-cpp/macau.h:11-54) for a 2-mode matrix with fixed
//                  Gaussian noise, in place of MacauX<MatrixData, FixedGaussianNoise> built by
//                  make_macau_fixed(2, K, precision) (macau.cpp:214-220).
//
// This header does not include the reference's headers itself: include "latentprior.h" and
// "macau.h" (which bring Eigen) before it.
//
// Who owns what.  One GpuSession (one mg_ctx, one CUDA stream) holds the training data, the test
// data, every mode's latents on the device and the device copy of every prior's hyperparameters
// (mu, Lambda; beta, Uhat and lambda_beta for side information).  Two ways of running a chain:
//
//   1. MacauGpuX::run() owns the run: the whole Gibbs loop runs on the device (mg_sweep per
//      iteration, a replayed CUDA graph when possible), and the host copies are refreshed at the
//      end -- `samples` (K x N latents per mode), `predictions`, `predictions_var`, `rmse_test`
//      and each prior's public mu / Lambda (+ beta, Uhat, lambda_beta).  With setSaveModel(true)
//      the latents and hyperparameters are also read back after every post-burn-in iteration to
//      write the reference's model files (macau.cpp:191-205, latentprior.cpp:307-315).
//   2. A host that drives its own loop (like MacauX::run, macau.cpp:110-147) calls the priors'
//      sample_latents / update_prior with host Eigen matrices, exactly as it calls the CPU
//      priors.  The host owns U, V, mu and Lambda then: sample_latents uploads the other mode's
//      latents and this prior's mu / Lambda, samples the mode on the device and downloads the
//      new latents into U; update_prior uploads U, draws the hyperparameters on the device and
//      downloads them into the prior's public members.  Every call copies K x N values over
//      PCIe, which is the price of keeping the reference's calling convention.
//
// The sparse matrix passed to sample_latents must be the training matrix given to the session
// (its transpose for mode 0, as in ILatentPrior::sample_latents, latentprior.cpp:30-37); only its
// shape is checked, the device keeps its own CSR.  `alpha` must equal the session's fixed
// precision.  Draws are keyed by (seed, iteration, mode): each prior counts its update_prior
// calls as the iteration index, which is the sweep index when the host follows MacauX::run's
// order (sample every mode, then update every prior).
//
// Probit noise and tensor (more than 2 mode) data are not supported by the GPU sampler; their
// overloads throw std::runtime_error.  Errors of the library throw std::runtime_error with its
// message ("Cholesky Decomposition failed!" for a failed factorisation, latentprior.cpp:375).
#pragma once

#include <cmath>
#include <cstdint>
#include <cstdio>
#include <fstream>
#include <iomanip>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "macau_b200.h"

namespace macau_b200 {

// writeToCSVfile (bpmfutils.h:169-173): one line per matrix row, values joined by ',', six
// significant digits, no trailing newline.  Works for any column-major matrix type with rows(),
// cols() and operator()(i, j).
template <typename M>
inline void write_csv(const std::string& path, const M& m) {
  std::ofstream f(path.c_str());
  f << std::setprecision(6);
  for (long i = 0; i < (long)m.rows(); i++) {
    if (i) f << "\n";
    for (long j = 0; j < (long)m.cols(); j++) {
      if (j) f << ",";
      f << m(i, j);
    }
  }
}

inline void check_code(const mg_ctx* ctx, int code) {
  if (code == MG_OK) return;
  const char* m = mg_last_error(ctx);
  throw std::runtime_error(m && *m ? m : "macau_b200 error " + std::to_string(code));
}

// Side information registered by a GpuMacauPrior, applied to the context at initialisation.
struct SideInfo {
  int mode;
  std::vector<int32_t> rows, cols;
  std::vector<double> vals;  // empty: binary
  int nrows, nfeat;
  double lambda_beta, tol;
};

// One device context shared by the priors and the Macau object of a run.
class GpuSession {
 public:
  GpuSession(int num_latent, double precision, int compute = MG_COMPUTE_FP64, uint64_t seed = 0,
             int device = 0, bool verbose = false)
      : num_latent(num_latent), precision(precision) {
    mg_config cfg{};
    cfg.num_latent = num_latent;
    cfg.precision = precision;
    cfg.seed = seed;
    cfg.compute = compute;
    cfg.verbose = verbose ? 1 : 0;
    cfg.device = device;
    const int code = mg_create(&ctx_, &cfg);
    if (code != MG_OK) {
      const char* m = mg_last_error(nullptr);
      const std::string msg = m && *m ? m : "mg_create failed";
      if (ctx_) mg_destroy(ctx_);
      ctx_ = nullptr;
      throw std::runtime_error(msg);
    }
  }
  GpuSession(const GpuSession&) = delete;
  GpuSession& operator=(const GpuSession&) = delete;
  ~GpuSession() {
    if (ctx_) mg_destroy(ctx_);
  }

  mg_ctx* ctx() const { return ctx_; }
  void check(int code) const { check_code(ctx_, code); }

  // Training / test data: idx is nnz x 2 column-major (rows, then columns).
  void set_train(const int32_t* idx, const double* vals, int64_t nnz, const int32_t* dims) {
    check(mg_set_relation_data(ctx_, idx, 2, vals, nnz, dims));
    dims_[0] = dims[0];
    dims_[1] = dims[1];
    initialised_ = false;
  }
  void set_test(const int32_t* idx, const double* vals, int64_t nnz, const int32_t* dims) {
    check(mg_set_relation_data_test(ctx_, idx, 2, vals, nnz, dims));
    initialised_ = false;
  }
  void add_side(SideInfo s) {
    sides_.push_back(std::move(s));
    initialised_ = false;
  }
  int64_t dim(int mode) const { return dims_[mode]; }

  // mg_set_side for every registered side, then mg_init (latents zero, initial hyperparameters).
  void init() {
    for (const SideInfo& s : sides_)
      check(mg_set_side(ctx_, s.mode, s.rows.data(), s.cols.data(),
                        s.vals.empty() ? nullptr : s.vals.data(), (int64_t)s.rows.size(),
                        s.nrows, s.nfeat, s.lambda_beta, s.tol));
    check(mg_init(ctx_));
    initialised_ = true;
  }
  void ensure_init() {
    if (!initialised_) init();
  }
  bool initialised() const { return initialised_; }

  const int num_latent;
  const double precision;

 private:
  mg_ctx* ctx_ = nullptr;
  int64_t dims_[2] = {0, 0};
  bool initialised_ = false;
  std::vector<SideInfo> sides_;
};

// Common part of the two adapter priors: the session, the mode and the host mirrors of the
// hyperparameters (public like BPMFPrior's members).
class GpuLatentPrior : public ILatentPrior {
 public:
  Eigen::VectorXd mu;
  Eigen::MatrixXd Lambda;

  GpuLatentPrior(std::shared_ptr<GpuSession> session, int mode)
      : session_(std::move(session)), mode_(mode) {
    if (mode_ != 0 && mode_ != 1) throw std::runtime_error("macau_b200: mode must be 0 or 1");
    const int K = session_->num_latent;
    // BPMFPrior::init / MacauPrior::init (latentprior.cpp:84-99, 181-216): mu = 0, Lambda = 10 I
    mu = Eigen::VectorXd::Zero(K);
    Lambda = Eigen::MatrixXd::Identity(K, K) * 10.0;
  }

  int mode() const { return mode_; }
  GpuSession& session() const { return *session_; }
  const std::shared_ptr<GpuSession>& session_ptr() const { return session_; }

  // ILatentPrior::sample_latents with host matrices: U (K x N_mode) receives the new latents,
  // `samples` is the other mode's K x N_other latents.
  void sample_latents(Eigen::MatrixXd& U, const Eigen::SparseMatrix<double>& mat,
                      double mean_value, const Eigen::MatrixXd& samples, double alpha,
                      const int num_latent) override {
    GpuSession& s = *session_;
    const int K = s.num_latent;
    if (num_latent != K) throw std::runtime_error("macau_b200: num_latent differs from the session");
    if (alpha != s.precision)
      throw std::runtime_error("macau_b200: alpha differs from the session's fixed precision");
    const int other = 1 - mode_;
    if ((int64_t)U.rows() != K || (int64_t)U.cols() != s.dim(mode_) ||
        (int64_t)samples.rows() != K || (int64_t)samples.cols() != s.dim(other) ||
        (int64_t)mat.cols() != s.dim(mode_) || (int64_t)mat.rows() != s.dim(other))
      throw std::runtime_error("macau_b200: matrix shapes differ from the session's data");
    (void)mean_value;  // the device computed the same mean from the training data
    s.ensure_init();
    s.check(mg_set_latents(s.ctx(), other, samples.data()));
    upload_hyper();
    s.check(mg_sample_latents(s.ctx(), mode_, (int)iter_, nullptr));
    s.check(mg_get_latents(s.ctx(), mode_, U.data()));
  }
  void sample_latents(ProbitNoise&, Eigen::MatrixXd&, const Eigen::SparseMatrix<double>&, double,
                      const Eigen::MatrixXd&, const int) override {
    throw std::runtime_error("macau_b200: probit noise is not supported by the GPU sampler");
  }
  void sample_latents(ProbitNoise&, TensorData&, std::vector<std::unique_ptr<Eigen::MatrixXd>>&,
                      int, const int) override {
    throw std::runtime_error("macau_b200: tensor data is not supported by the GPU sampler");
  }
  void sample_latents(double, TensorData&, std::vector<std::unique_ptr<Eigen::MatrixXd>>&, int,
                      const int) override {
    throw std::runtime_error("macau_b200: tensor data is not supported by the GPU sampler");
  }

  // ILatentPrior::update_prior: the hyperparameters (and, with side information, beta, Uhat and
  // lambda_beta) are drawn on the device from U and copied into the public members.
  void update_prior(const Eigen::MatrixXd& U) override {
    GpuSession& s = *session_;
    if ((int64_t)U.rows() != s.num_latent || (int64_t)U.cols() != s.dim(mode_))
      throw std::runtime_error("macau_b200: matrix shapes differ from the session's data");
    s.ensure_init();
    s.check(mg_set_latents(s.ctx(), mode_, U.data()));
    upload_hyper();
    s.check(mg_update_prior(s.ctx(), mode_, (int)iter_));
    download_hyper();
    iter_++;
  }

  // Refreshes the host mirrors from the device (after a device-driven run).
  virtual void download_hyper() {
    double lb = 0.0;
    session_->check(mg_get_hyper(session_->ctx(), mode_, mu.data(), Lambda.data(), &lb));
  }

  void saveModel(std::string prefix) override { write_csv(prefix + "-latentmean.csv", mu); }

 protected:
  virtual void upload_hyper() {
    session_->check(mg_set_hyper(session_->ctx(), mode_, mu.data(), Lambda.data(), nullptr));
  }

  std::shared_ptr<GpuSession> session_;
  int mode_;
  uint32_t iter_ = 0;
};

// BPMFPrior on the GPU.
class GpuBPMFPrior : public GpuLatentPrior {
 public:
  GpuBPMFPrior(std::shared_ptr<GpuSession> session, int mode)
      : GpuLatentPrior(std::move(session), mode) {}
};

// MacauPrior<SparseDoubleFeat> on the GPU: F is nrows x nfeat, given as COO (vals NULL for a
// binary matrix); the device solves for beta with block-CG (solve_blockcg, linop.h:207-343).
class GpuMacauPrior : public GpuLatentPrior {
 public:
  Eigen::MatrixXd beta;  // K x nfeat link matrix (host mirror)
  Eigen::MatrixXd Uhat;  // K x N, beta F^T (host mirror)
  double lambda_beta = 5.0;
  double tol = 1e-6;

  GpuMacauPrior(std::shared_ptr<GpuSession> session, int mode, const int32_t* rows,
                const int32_t* cols, const double* vals, int64_t nnz, int nrows, int nfeat)
      : GpuLatentPrior(std::move(session), mode), nrows_(nrows), nfeat_(nfeat) {
    rows_.assign(rows, rows + nnz);
    cols_.assign(cols, cols + nnz);
    if (vals) vals_.assign(vals, vals + nnz);
    beta = Eigen::MatrixXd::Zero(session_->num_latent, nfeat);
    Uhat = Eigen::MatrixXd::Zero(session_->num_latent, nrows);
  }

  // MacauPrior::setLambdaBeta / setTol (latentprior.h:120-121); take effect at initialisation.
  void setLambdaBeta(double lb) { lambda_beta = lb; }
  void setTol(double t) { tol = t; }
  double getLinkLambda() override { return lambda_beta; }
  // MacauPrior::getLinkNorm (latentprior.cpp:296-298): Frobenius norm of beta.
  double getLinkNorm() override { return beta.norm(); }

  // Registers F with the session (done by MacauGpuX::addPrior, or by hand before the first
  // sample_latents of a host-driven loop).
  void register_side() {
    if (registered_) return;
    SideInfo s{mode_, rows_, cols_, vals_, nrows_, nfeat_, lambda_beta, tol};
    session_->add_side(std::move(s));
    registered_ = true;
  }

  void download_hyper() override {
    GpuSession& s = *session_;
    s.check(mg_get_hyper(s.ctx(), mode_, mu.data(), Lambda.data(), &lambda_beta));
    s.check(mg_get_beta(s.ctx(), mode_, beta.data()));
    s.check(mg_get_uhat(s.ctx(), mode_, Uhat.data()));
  }

  void saveModel(std::string prefix) override {
    write_csv(prefix + "-latentmean.csv", mu);
    write_csv(prefix + "-link.csv", beta);
  }

 protected:
  void upload_hyper() override {
    session_->check(mg_set_hyper(session_->ctx(), mode_, mu.data(), Lambda.data(), &lambda_beta));
  }

 private:
  std::vector<int32_t> rows_, cols_;
  std::vector<double> vals_;
  int nrows_, nfeat_;
  bool registered_ = false;
};

// MacauX<MatrixData, FixedGaussianNoise> on the GPU.  addPrior takes GpuBPMFPrior /
// GpuMacauPrior objects of this object's session, in mode order.
class MacauGpuX : public Macau {
 public:
  MacauGpuX(std::shared_ptr<GpuSession> session) : session_(std::move(session)) {
    num_latent = session_->num_latent;
  }
  // make_macau_fixed(2, K, precision) with the GPU's compute mode and seed.
  MacauGpuX(int K, double precision, int compute = MG_COMPUTE_FP64, uint64_t seed = 0)
      : MacauGpuX(std::make_shared<GpuSession>(K, precision, compute, seed)) {}

  const std::shared_ptr<GpuSession>& session() const { return session_; }

  void addPrior(std::unique_ptr<ILatentPrior>& prior) override {
    auto* g = dynamic_cast<GpuLatentPrior*>(prior.get());
    if (!g || g->session_ptr() != session_)
      throw std::runtime_error("macau_b200: addPrior needs a GPU prior of this object's session");
    if (g->mode() != (int)priors.size())
      throw std::runtime_error("macau_b200: priors must be added in mode order");
    if (auto* m = dynamic_cast<GpuMacauPrior*>(g)) m->register_side();
    priors.push_back(std::move(prior));
  }
  void setSamples(int b, int n) override {
    burnin = b;
    nsamples = n;
    session_->check(mg_set_samples(session_->ctx(), b, n));
  }
  void setRelationData(int* rows, int* cols, double* values, int nnz, int nrows,
                       int ncols) override {
    std::vector<int32_t> idx = stack(rows, cols, nnz);
    const int32_t dims[2] = {nrows, ncols};
    session_->set_train(idx.data(), values, nnz, dims);
  }
  void setRelationDataTest(int* rows, int* cols, double* values, int nnz, int nrows,
                           int ncols) override {
    std::vector<int32_t> idx = stack(rows, cols, nnz);
    const int32_t dims[2] = {nrows, ncols};
    session_->set_test(idx.data(), values, nnz, dims);
  }
  void setRelationData(int* idx, int nmodes, double* values, int nnz, int* dims) override {
    if (nmodes != 2) throw std::runtime_error("macau_b200: tensor data is not supported");
    session_->set_train(idx, values, nnz, dims);
  }
  void setRelationDataTest(int* idx, int nmodes, double* values, int nnz, int* dims) override {
    if (nmodes != 2) throw std::runtime_error("macau_b200: tensor data is not supported");
    session_->set_test(idx, values, nnz, dims);
  }

  // MacauX::init (macau.cpp:72-86): needs both priors; latents start at zero.
  void init() override {
    if (priors.size() < 2) throw std::runtime_error("Less 2 priors are not supported.");
    session_->init();
    samples.clear();
    for (int m = 0; m < 2; m++)
      samples.push_back(std::unique_ptr<Eigen::MatrixXd>(
          new Eigen::MatrixXd(Eigen::MatrixXd::Zero(num_latent, session_->dim(m)))));
  }

  // MacauX::run (macau.cpp:94-148) with every iteration on the device.
  void run() override {
    init();
    mg_ctx* c = session_->ctx();
    int64_t ntest = 0;
    double mean = 0.0;
    session_->check(mg_get_dims(c, nullptr, nullptr, nullptr, &ntest, &mean));
    if (save_model) saveGlobalParams();
    if (!save_model && !verbose) {
      session_->check(mg_sweeps(c, 0, burnin + nsamples, 1));
    } else {
      for (int i = 0; i < burnin + nsamples; i++) {
        session_->check(mg_sweep(c, i, 1));
        if (save_model && i >= burnin) {
          refresh();
          saveModel(i - burnin + 1);
        }
        if (verbose) {
          double r[2] = {0.0, 0.0};
          session_->check(mg_get_rmse(c, r));
          std::printf("Iter %3d: RMSE: %.4f (1samp: %.4f)\n", i, r[0], r[1]);
        }
      }
    }
    refresh();
    predictions = Eigen::VectorXd::Zero(ntest);
    predictions_var = Eigen::VectorXd::Zero(ntest);
    if (ntest > 0) {
      session_->check(mg_get_predictions(c, predictions.data()));
      Eigen::VectorXd sd = getStds();
      for (int64_t i = 0; i < ntest; i++)
        predictions_var[i] = nsamples > 1 ? sd[i] * sd[i] * (nsamples - 1) : 0.0;
    }
    double r[2] = {0.0, 0.0};
    session_->check(mg_get_rmse(c, r));
    rmse_test = r[0];
  }

  void printStatus(int i, double elapsedi, double samples_per_sec) override {
    (void)samples_per_sec;
    double r[2] = {0.0, 0.0};
    session_->check(mg_get_rmse(session_->ctx(), r));
    std::printf("Iter %3d: RMSE: %.4f (1samp: %.4f) [took %0.1fs]\n", i, r[0], r[1], elapsedi);
  }
  void setVerbose(bool v) override { verbose = v; }
  double getRmseTest() override { return rmse_test; }
  Eigen::VectorXd getPredictions() override { return predictions; }
  // MacauX::getStds (macau.cpp:174-188): NaN when nsamples <= 1.
  Eigen::VectorXd getStds() override {
    int64_t ntest = 0;
    session_->check(mg_get_dims(session_->ctx(), nullptr, nullptr, nullptr, &ntest, nullptr));
    Eigen::VectorXd sd(ntest);
    if (ntest > 0) session_->check(mg_get_stds(session_->ctx(), sd.data()));
    return sd;
  }
  void setSaveModel(bool save) override { save_model = save; }
  void setSavePrefix(std::string pref) override { save_prefix = pref; }
  // MacauX::saveModel (macau.cpp:191-198).
  void saveModel(int isample) override {
    const std::string fp = save_prefix + "-sample" + std::to_string(isample) + "-";
    for (size_t i = 0; i < samples.size(); i++) {
      write_csv(fp + "U" + std::to_string(i + 1) + "-latents.csv", *samples[i]);
      priors[i]->saveModel(fp + "U" + std::to_string(i + 1));
    }
  }
  // MatrixData::getTestData (sparsetensor.cpp:63-76): ntest x 3 (row, col, value).
  Eigen::MatrixXd getTestData() override {
    int64_t ntest = 0;
    session_->check(mg_get_dims(session_->ctx(), nullptr, nullptr, nullptr, &ntest, nullptr));
    Eigen::MatrixXd t(ntest, 3);
    if (ntest > 0) session_->check(mg_get_test_data(session_->ctx(), t.data()));
    return t;
  }
  // MacauX::saveGlobalParams (macau.cpp:200-205).
  void saveGlobalParams() override {
    double mean = 0.0;
    session_->check(mg_get_dims(session_->ctx(), nullptr, nullptr, nullptr, nullptr, &mean));
    Eigen::VectorXd means(1);
    means[0] = mean;
    write_csv(save_prefix + "-meanvalue.csv", means);
  }

 private:
  // Host copies of the device state: latents of both modes and every prior's hyperparameters.
  void refresh() {
    for (int m = 0; m < 2; m++) {
      session_->check(mg_get_latents(session_->ctx(), m, samples[m]->data()));
      static_cast<GpuLatentPrior*>(priors[m].get())->download_hyper();
    }
  }
  static std::vector<int32_t> stack(const int* rows, const int* cols, int nnz) {
    std::vector<int32_t> idx(2 * (size_t)(nnz > 0 ? nnz : 0));
    for (int e = 0; e < nnz; e++) {
      idx[e] = rows[e];
      idx[(size_t)nnz + e] = cols[e];
    }
    return idx;
  }
  std::shared_ptr<GpuSession> session_;
};

}  // namespace macau_b200
