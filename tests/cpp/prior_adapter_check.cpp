// Drives the adapters of include/macau_b200_priors.hpp through the reference's interfaces
// (ILatentPrior, Macau; here the test stand-ins of tests/cpp/standin/reference_interfaces.h):
//   device  MacauGpuX::run() with two adapter priors added by addPrior;
//   host    the loop of MacauX::run (macau.cpp:110-147) written against ILatentPrior:
//           sample_latents on host Eigen matrices for modes 0 and 1, then update_prior for both.
// Input: a binary file of int32 {nrow, ncol, ntrain, ntest, K, burnin, nsamples}, train rows,
// cols (int32), values (double), the same for the test set, then int32 {nnzF, nfeat} and the
// rows and cols (int32) of a binary side matrix for mode 0 (nnzF = 0: BPMF on both modes).
// Prints the device run's RMSE, the largest difference between the two runs' latents and the
// results of the interface checks, or "ERROR <message>" with exit code 2 when the library
// reports an error (e.g. no GPU).
#include <cmath>
#include <cstdio>
#include <stdexcept>
#include <vector>

#include "standin/reference_interfaces.h"
#include "macau_b200_priors.hpp"

using macau_b200::GpuBPMFPrior;
using macau_b200::GpuLatentPrior;
using macau_b200::GpuMacauPrior;
using macau_b200::GpuSession;
using macau_b200::MacauGpuX;

template <typename T>
static bool read(FILE* f, std::vector<T>& v, size_t n) {
  v.resize(n);
  return n == 0 || std::fread(v.data(), sizeof(T), n, f) == n;
}

struct Data {
  std::vector<int> hdr, r, c, tr, tc, fr, fc, side;
  std::vector<double> v, tv;
};

static std::unique_ptr<ILatentPrior> make_prior(const std::shared_ptr<GpuSession>& s, int mode,
                                                Data& d) {
  if (mode == 0 && d.side[0] > 0) {
    auto* p = new GpuMacauPrior(s, 0, d.fr.data(), d.fc.data(), nullptr, d.side[0], d.hdr[0],
                                d.side[1]);
    p->setLambdaBeta(5.0);
    p->setTol(1e-6);
    return std::unique_ptr<ILatentPrior>(p);
  }
  return std::unique_ptr<ILatentPrior>(new GpuBPMFPrior(s, mode));
}

int main(int argc, char** argv) {
  if (argc != 3) {
    std::printf("usage: prior_adapter_check <data> <seed>\n");
    return 1;
  }
  FILE* f = std::fopen(argv[1], "rb");
  if (!f) return 1;
  Data d;
  bool ok = read(f, d.hdr, 7);
  ok = ok && read(f, d.r, d.hdr[2]) && read(f, d.c, d.hdr[2]) && read(f, d.v, d.hdr[2]);
  ok = ok && read(f, d.tr, d.hdr[3]) && read(f, d.tc, d.hdr[3]) && read(f, d.tv, d.hdr[3]);
  ok = ok && read(f, d.side, 2) && read(f, d.fr, d.side[0]) && read(f, d.fc, d.side[0]);
  std::fclose(f);
  if (!ok) return 1;
  const int nrow = d.hdr[0], ncol = d.hdr[1], K = d.hdr[4], burnin = d.hdr[5],
            nsamples = d.hdr[6];
  const double alpha = 2.0;
  const unsigned long long seed = std::stoull(argv[2]);
  try {
    // ---- device-driven run ----
    MacauGpuX m(K, alpha, MG_COMPUTE_FP64, seed);
    std::unique_ptr<ILatentPrior> p0 = make_prior(m.session(), 0, d);
    std::unique_ptr<ILatentPrior> p1 = make_prior(m.session(), 1, d);
    m.addPrior(p0);
    m.addPrior(p1);
    m.setRelationData(d.r.data(), d.c.data(), d.v.data(), d.hdr[2], nrow, ncol);
    m.setRelationDataTest(d.tr.data(), d.tc.data(), d.tv.data(), d.hdr[3], nrow, ncol);
    m.setSamples(burnin, nsamples);
    m.setVerbose(false);
    m.run();
    std::printf("RMSE %.17g\n", m.getRmseTest());
    double sp = 0.0;
    for (long i = 0; i < m.getPredictions().size(); i++) sp += m.getPredictions()[i];
    std::printf("PRED %.17g\n", sp);
    std::printf("LINKNORM %.17g\n", m.priors[0]->getLinkNorm());

    // ---- host-driven loop through ILatentPrior ----
    auto s = std::make_shared<GpuSession>(K, alpha, MG_COMPUTE_FP64, seed);
    std::vector<int32_t> idx(2 * (size_t)d.hdr[2]);
    for (int e = 0; e < d.hdr[2]; e++) {
      idx[e] = d.r[e];
      idx[(size_t)d.hdr[2] + e] = d.c[e];
    }
    const int32_t dims[2] = {nrow, ncol};
    s->set_train(idx.data(), d.v.data(), d.hdr[2], dims);
    std::unique_ptr<ILatentPrior> q[2] = {make_prior(s, 0, d), make_prior(s, 1, d)};
    if (auto* mp = dynamic_cast<GpuMacauPrior*>(q[0].get())) mp->register_side();
    std::vector<std::unique_ptr<Eigen::MatrixXd>> samples;
    samples.emplace_back(new Eigen::MatrixXd(Eigen::MatrixXd::Zero(K, nrow)));
    samples.emplace_back(new Eigen::MatrixXd(Eigen::MatrixXd::Zero(K, ncol)));
    const Eigen::SparseMatrix<double> Y(nrow, ncol), Yt(ncol, nrow);
    for (int i = 0; i < burnin + nsamples; i++) {
      q[0]->sample_latents(*samples[0], Yt, 0.0, *samples[1], alpha, K);
      q[1]->sample_latents(*samples[1], Y, 0.0, *samples[0], alpha, K);
      q[0]->update_prior(*samples[0]);
      q[1]->update_prior(*samples[1]);
    }
    double du = 0.0, dl = 0.0;
    for (int mode = 0; mode < 2; mode++) {
      const Eigen::MatrixXd& a = *m.samples[mode];
      const Eigen::MatrixXd& b = *samples[mode];
      for (long j = 0; j < a.cols(); j++)
        for (long k = 0; k < K; k++) du = std::fmax(du, std::fabs(a(k, j) - b(k, j)));
      const auto* ga = static_cast<GpuLatentPrior*>(m.priors[mode].get());
      const auto* gb = static_cast<GpuLatentPrior*>(q[mode].get());
      for (long j = 0; j < K; j++)
        for (long k = 0; k < K; k++)
          dl = std::fmax(dl, std::fabs(ga->Lambda(k, j) - gb->Lambda(k, j)));
    }
    std::printf("LATENT_DIFF %.17g\nLAMBDA_DIFF %.17g\n", du, dl);

    // ---- interface checks ----
    int checks = 0;
    try {  // a prior of another session
      std::unique_ptr<ILatentPrior> foreign(new GpuBPMFPrior(s, 0));
      MacauGpuX other(K, alpha);
      other.addPrior(foreign);
    } catch (const std::runtime_error&) {
      checks++;
    }
    try {  // a different alpha than the session's fixed precision
      q[0]->sample_latents(*samples[0], Yt, 0.0, *samples[1], alpha + 1.0, K);
    } catch (const std::runtime_error&) {
      checks++;
    }
    try {  // fewer than two priors
      MacauGpuX lone(K, alpha);
      lone.init();
    } catch (const std::runtime_error& e) {
      if (std::string(e.what()) == "Less 2 priors are not supported.") checks++;
    }
    std::printf("CHECKS %d\n", checks);
  } catch (const std::exception& e) {
    std::printf("ERROR %s\n", e.what());
    return 2;
  }
  return 0;
}
