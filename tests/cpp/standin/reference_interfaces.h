// Test stand-in for the two reference interfaces the adapters of include/macau_b200_priors.hpp
// implement, so that the adapters compile and run without the reference's sources and Eigen:
//   * a few Eigen types, reduced to what the adapters and this test use (column-major dense
//     storage; a sparse matrix that only knows its shape);
//   * ILatentPrior with the virtual member signatures of lib/macau-cpp/latentprior.h:17-49 that
//     a prior must override (the noise-dispatching overloads of the real class are left out);
//   * Macau with the pure virtual members of lib/macau-cpp/macau.h:11-54.
#pragma once

#include <cmath>
#include <memory>
#include <string>
#include <vector>

namespace Eigen {

class MatrixXd {
 public:
  MatrixXd() = default;
  MatrixXd(long r, long c) : r_(r), c_(c), v_((size_t)(r * c), 0.0) {}
  static MatrixXd Zero(long r, long c) { return MatrixXd(r, c); }
  static MatrixXd Identity(long r, long c) {
    MatrixXd m(r, c);
    for (long i = 0; i < r && i < c; i++) m(i, i) = 1.0;
    return m;
  }
  MatrixXd operator*(double s) const {
    MatrixXd m = *this;
    for (double& x : m.v_) x *= s;
    return m;
  }
  long rows() const { return r_; }
  long cols() const { return c_; }
  double* data() { return v_.data(); }
  const double* data() const { return v_.data(); }
  double& operator()(long i, long j) { return v_[(size_t)(i + j * r_)]; }
  double operator()(long i, long j) const { return v_[(size_t)(i + j * r_)]; }
  double norm() const {
    double s = 0.0;
    for (double x : v_) s += x * x;
    return std::sqrt(s);
  }

 protected:
  long r_ = 0, c_ = 0;
  std::vector<double> v_;
};

class VectorXd : public MatrixXd {
 public:
  VectorXd() = default;
  explicit VectorXd(long n) : MatrixXd(n, 1) {}
  static VectorXd Zero(long n) { return VectorXd(n); }
  long size() const { return r_; }
  double& operator[](long i) { return v_[(size_t)i]; }
  double operator[](long i) const { return v_[(size_t)i]; }
};

template <typename T>
class SparseMatrix {
 public:
  SparseMatrix(long r, long c) : r_(r), c_(c) {}
  long rows() const { return r_; }
  long cols() const { return c_; }

 private:
  long r_, c_;
};

}  // namespace Eigen

class ProbitNoise;
class TensorData;

class ILatentPrior {
 public:
  virtual void sample_latents(Eigen::MatrixXd& U, const Eigen::SparseMatrix<double>& mat,
                              double mean_value, const Eigen::MatrixXd& samples, double alpha,
                              const int num_latent) = 0;
  virtual void sample_latents(ProbitNoise& noise, Eigen::MatrixXd& U,
                              const Eigen::SparseMatrix<double>& mat, double mean_value,
                              const Eigen::MatrixXd& samples, const int num_latent) = 0;
  virtual void sample_latents(ProbitNoise& noiseModel, TensorData& data,
                              std::vector<std::unique_ptr<Eigen::MatrixXd>>& samples, int mode,
                              const int num_latent) = 0;
  virtual void sample_latents(double noisePrecision, TensorData& data,
                              std::vector<std::unique_ptr<Eigen::MatrixXd>>& samples, int mode,
                              const int num_latent) = 0;
  virtual void update_prior(const Eigen::MatrixXd& /*U*/) {}
  virtual double getLinkNorm() { return NAN; }
  virtual double getLinkLambda() { return NAN; }
  virtual void saveModel(std::string /*prefix*/) {}
  virtual ~ILatentPrior() {}
};

class Macau {
 public:
  int num_latent;
  int nsamples = 100;
  int burnin = 50;
  Eigen::VectorXd predictions;
  Eigen::VectorXd predictions_var;
  double rmse_test = .0;
  double rmse_train = .0;
  std::vector<std::unique_ptr<ILatentPrior>> priors;
  std::vector<std::unique_ptr<Eigen::MatrixXd>> samples;
  bool verbose = true;
  bool save_model = false;
  std::string save_prefix = "model";

  virtual void addPrior(std::unique_ptr<ILatentPrior>& prior) = 0;
  virtual void setSamples(int burnin, int nsamples) = 0;
  virtual void setRelationData(int* rows, int* cols, double* values, int nnz, int nrows,
                               int ncols) = 0;
  virtual void setRelationDataTest(int* rows, int* cols, double* values, int nnz, int nrows,
                                   int ncols) = 0;
  virtual void setRelationData(int* idx, int nmodes, double* values, int nnz, int* dims) = 0;
  virtual void setRelationDataTest(int* idx, int nmodes, double* values, int nnz,
                                   int* dims) = 0;
  virtual void init() = 0;
  virtual void run() = 0;
  virtual void printStatus(int i, double elapsedi, double samples_per_sec) = 0;
  virtual void setVerbose(bool v) = 0;
  virtual double getRmseTest() = 0;
  virtual Eigen::VectorXd getPredictions() = 0;
  virtual Eigen::VectorXd getStds() = 0;
  virtual void setSaveModel(bool save) = 0;
  virtual void setSavePrefix(std::string pref) = 0;
  virtual void saveModel(int isample) = 0;
  virtual Eigen::MatrixXd getTestData() = 0;
  virtual void saveGlobalParams() = 0;
  virtual ~Macau() {}
};
