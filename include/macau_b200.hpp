// C++ host class over the C ABI of macau_b200.h, shaped like the reference's `Macau` /
// `MacauX<MatrixData, FixedGaussianNoise>` (lib/macau-cpp/macau.h:11-81, built by
// make_macau_fixed / make_macau_adaptive, macau.cpp:214-228), so that a C++ host written against
// that class switches to the GPU sampler by changing the type it constructs.
//
// Differences from the reference class, all forced by dropping Eigen from the interface:
//   * results are std::vector<double> instead of Eigen::VectorXd / MatrixXd (getTestData is
//     ntest x 3 column-major, like MatrixData::getTestData, sparsetensor.cpp:63-76);
//   * priors are not ILatentPrior objects: a mode without side information is BPMF, and
//     addSide / addSideUnivariate stand in for addPrior(MacauPrior / MacauOnePrior);
//   * verbose output is chosen at construction (printStatus runs inside the library).
// Errors throw std::runtime_error with the library's message; a failed Cholesky keeps the
// reference's text "Cholesky Decomposition failed!" (latentprior.cpp:375).
#pragma once

#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

#include "macau_b200.h"

namespace macau_b200 {

class MacauGpu {
 public:
  MacauGpu(int num_latent, double precision, int compute = MG_COMPUTE_FP64, uint64_t seed = 0,
           bool verbose = false, int device = 0)
      : num_latent(num_latent) {
    mg_config cfg{};
    cfg.num_latent = num_latent;
    cfg.precision = precision;
    cfg.seed = seed;
    cfg.compute = compute;
    cfg.verbose = verbose ? 1 : 0;
    cfg.device = device;
    const int code = mg_create(&ctx_, &cfg);
    if (code != 0) {
      const std::string msg = mg_last_error(nullptr) ? mg_last_error(nullptr) : "mg_create failed";
      if (ctx_) mg_destroy(ctx_);
      ctx_ = nullptr;
      throw std::runtime_error(msg);
    }
  }
  MacauGpu(const MacauGpu&) = delete;
  MacauGpu& operator=(const MacauGpu&) = delete;
  ~MacauGpu() {
    if (ctx_) mg_destroy(ctx_);
  }

  // make_macau_adaptive(2, K, sn_init, sn_max): adaptive Gaussian noise (before init / run).
  void setAdaptiveNoise(double sn_init, double sn_max) {
    check(mg_set_noise_adaptive(ctx_, sn_init, sn_max));
  }
  void setSamples(int burnin_, int nsamples_) {
    burnin = burnin_;
    nsamples = nsamples_;
    check(mg_set_samples(ctx_, burnin_, nsamples_));
  }
  void setRelationData(int* rows, int* cols, double* values, int nnz, int nrows, int ncols) {
    check(mg_set_relation_data_rc(ctx_, rows, cols, values, nnz, nrows, ncols));
  }
  void setRelationData(int* idx, int nmodes, double* values, int nnz, int* dims) {
    check(mg_set_relation_data(ctx_, idx, nmodes, values, nnz, dims));
  }
  void setRelationDataTest(int* rows, int* cols, double* values, int nnz, int nrows, int ncols) {
    check(mg_set_relation_data_test_rc(ctx_, rows, cols, values, nnz, nrows, ncols));
  }
  void setRelationDataTest(int* idx, int nmodes, double* values, int nnz, int* dims) {
    check(mg_set_relation_data_test(ctx_, idx, nmodes, values, nnz, dims));
  }
  // addPrior(MacauPrior<SparseDoubleFeat>) for `mode`: F is nrows x nfeat COO, vals NULL for a
  // binary matrix (make_prior, macau.pyx:154-192).
  void addSide(int mode, const int* rows, const int* cols, const double* vals, int64_t nnz,
               int nrows, int nfeat, double lambda_beta = 5.0, double tol = 1e-6) {
    check(mg_set_side(ctx_, mode, rows, cols, vals, nnz, nrows, nfeat, lambda_beta, tol));
  }
  // addPrior(MacauOnePrior) for `mode` (make_one_prior, macau.pyx:194-214).
  void addSideUnivariate(int mode, const int* rows, const int* cols, const double* vals,
                         int64_t nnz, int nrows, int nfeat, double lambda_beta = 5.0) {
    check(mg_set_side_univariate(ctx_, mode, rows, cols, vals, nnz, nrows, nfeat, lambda_beta));
  }
  void init() { check(mg_init(ctx_)); }
  void run() { check(mg_run(ctx_)); }
  double getRmseTest() {
    double r[2] = {0.0, 0.0};
    check(mg_get_rmse(ctx_, r));
    return r[0];
  }
  std::vector<double> getPredictions() { return per_test(mg_get_predictions, 1); }
  std::vector<double> getStds() { return per_test(mg_get_stds, 1); }
  std::vector<double> getTestData() { return per_test(mg_get_test_data, 3); }

  // The underlying context, for the phase-level entry points of macau_b200.h.
  mg_ctx* context() const { return ctx_; }

  int num_latent;
  int burnin = 50, nsamples = 100;  // Macau's defaults (macau.h:17-18)

 private:
  std::vector<double> per_test(int (*get)(mg_ctx*, double*), int width) {
    int64_t ntest = 0;
    check(mg_get_dims(ctx_, nullptr, nullptr, nullptr, &ntest, nullptr));
    std::vector<double> out((size_t)ntest * width);
    if (ntest > 0) check(get(ctx_, out.data()));
    return out;
  }
  void check(int code) {
    if (code == 0) return;
    const char* m = mg_last_error(ctx_);
    throw std::runtime_error(m && *m ? m : "macau_b200 error " + std::to_string(code));
  }
  mg_ctx* ctx_ = nullptr;
};

}  // namespace macau_b200
