// A C++ host driving the GPU sampler through include/macau_b200.hpp the way a host of the
// reference drives MacauX (set data, setSamples, run, getRmseTest / getPredictions / getStds /
// getTestData).  Input: a binary file of int32 {nrow, ncol, ntrain, ntest, K, burnin, nsamples},
// then train rows, cols (int32), values (double), then the same for the test set.  Prints the
// posterior-mean RMSE and sums of the predictions, stds and test data, or "ERROR <message>" with
// exit code 2 when the library reports an error (e.g. no GPU).
#include <cstdio>
#include <stdexcept>
#include <vector>

#include "macau_b200.hpp"

template <typename T>
static bool read(FILE* f, std::vector<T>& v, size_t n) {
  v.resize(n);
  return n == 0 || std::fread(v.data(), sizeof(T), n, f) == n;
}

int main(int argc, char** argv) {
  if (argc != 3) {
    std::printf("usage: macau_cpp_host <data> <seed>\n");
    return 1;
  }
  FILE* f = std::fopen(argv[1], "rb");
  if (!f) return 1;
  std::vector<int> hdr, r, c, tr, tc;
  std::vector<double> v, tv;
  bool ok = read(f, hdr, 7);
  ok = ok && read(f, r, hdr[2]) && read(f, c, hdr[2]) && read(f, v, hdr[2]);
  ok = ok && read(f, tr, hdr[3]) && read(f, tc, hdr[3]) && read(f, tv, hdr[3]);
  std::fclose(f);
  if (!ok) return 1;
  try {
    macau_b200::MacauGpu m(hdr[4], 2.0, MG_COMPUTE_FP64, std::stoull(argv[2]));
    m.setRelationData(r.data(), c.data(), v.data(), hdr[2], hdr[0], hdr[1]);
    m.setRelationDataTest(tr.data(), tc.data(), tv.data(), hdr[3], hdr[0], hdr[1]);
    m.setSamples(hdr[5], hdr[6]);
    m.run();
    double sp = 0.0, ss = 0.0, st = 0.0;
    for (double x : m.getPredictions()) sp += x;
    for (double x : m.getStds()) ss += x;
    for (double x : m.getTestData()) st += x;
    std::printf("RMSE %.17g\nPRED %.17g\nSTDS %.17g\nTEST %.17g\n", m.getRmseTest(), sp, ss, st);
  } catch (const std::exception& e) {
    std::printf("ERROR %s\n", e.what());
    return 2;
  }
  return 0;
}
