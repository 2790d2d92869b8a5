// TEST INFRASTRUCTURE ONLY -- part of the CPU oracle. Nothing in the product links this file.
//
// Keyed random draws for the oracle.  The reference draws its N(0,1) and Gamma variates from
// thread-local, non-reproducible std::mt19937 streams (mvnormal.cpp:32-51, 81-102, 163-166,
// 217-228), so "the same draws" can only be defined by a keyed counter-based generator that the
// oracle and the CUDA path both implement:
//
//   * Philox-4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as easy as 1, 2, 3",
//     SC'11): 10 rounds of the 4x32 Philox S-box with the published multipliers and Weyl key
//     increments.  Checked against the published known-answer vectors in the tests.
//   * N(0,1): Box-Muller on two 53-bit uniforms in (0,1) built from one Philox block.
//   * Gamma(shape >= 1, scale 1): Marsaglia & Tsang, "A simple method for generating gamma
//     variables", ACM TOMS 26(3), 2000.  shape < 1 uses the same paper's boost
//     Gamma(a) = Gamma(a+1) * U^(1/a).
//
// Key and counter layout of one draw (identical in the CUDA library):
//   key     = {seed & 0xffffffff, seed >> 32}
//   counter = {block, index, (purpose << 8) | mode, sweep}
// where `block` is the pair index j/2 for normals and 2*attempt (+1 for the uniform) for gamma
// draws, and `index` is the row / feature / matrix-row the draw belongs to.
#pragma once
#include <cmath>
#include <cstdint>

namespace oracle {

enum Purpose : uint32_t {
  kRowNoise = 1,      // sample_latent_blas: randn0() per latent dim (latentprior.cpp:380-382)
  kMvnN = 2,          // sample_beta: MvNormal_prec_omp(Lambda, N) (latentprior.cpp:277)
  kMvnF = 3,          // sample_beta: MvNormal_prec_omp(Lambda, nfeat) (latentprior.cpp:278)
  kWishartOff = 4,    // WishartUnit off-diagonal N(0,1) (mvnormal.cpp:225-226)
  kWishartDiag = 5,   // WishartUnit chi via Gamma (mvnormal.cpp:223-224)
  kMuDraw = 6,        // NormalWishart: MvNormal_prec(kappa*Lambda, mu) (mvnormal.cpp:273)
  kLambdaBeta = 7,    // sample_lambda_beta: rgamma (latentprior.cpp:328-331)
  kNoiseAlpha = 8,    // AdaptiveGaussianNoise::update: rgamma(aN, 1/bN) (noisemodels.cpp:75-78)
  kBetaOne = 9,       // MacauOnePrior::sample_beta: bmrandn_single per feature (macauoneprior.cpp:241)
};

inline void philox4x32_10(const uint32_t ctr_in[4], const uint32_t key_in[2], uint32_t out[4]) {
  const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u;
  const uint32_t W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
  uint32_t c0 = ctr_in[0], c1 = ctr_in[1], c2 = ctr_in[2], c3 = ctr_in[3];
  uint32_t k0 = key_in[0], k1 = key_in[1];
  for (int r = 0; r < 10; r++) {
    if (r > 0) { k0 += W0; k1 += W1; }
    uint64_t p0 = (uint64_t)M0 * c0;
    uint64_t p1 = (uint64_t)M1 * c2;
    uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
    uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
    uint32_t n0 = hi1 ^ c1 ^ k0;
    uint32_t n2 = hi0 ^ c3 ^ k1;
    c0 = n0; c1 = lo1; c2 = n2; c3 = lo0;
  }
  out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

// 53-bit uniform strictly inside (0, 1).
inline double unit_open(uint32_t hi, uint32_t lo) {
  uint64_t x = (((uint64_t)hi << 32) | lo) >> 11;
  return ((double)x + 0.5) * (1.0 / 9007199254740992.0);
}

inline uint32_t stream_id(uint32_t purpose, uint32_t mode) { return (purpose << 8) | mode; }

inline void philox_block(uint64_t seed, uint32_t sweep, uint32_t stream, uint32_t index,
                         uint32_t block, uint32_t out[4]) {
  const uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
  const uint32_t ctr[4] = {block, index, stream, sweep};
  philox4x32_10(ctr, key, out);
}

// Draw j of the N(0,1) sequence at (seed, sweep, stream, index).
inline double normal_draw(uint64_t seed, uint32_t sweep, uint32_t stream, uint32_t index,
                          uint32_t j) {
  uint32_t r[4];
  philox_block(seed, sweep, stream, index, j >> 1, r);
  const double u1 = unit_open(r[0], r[1]);
  const double u2 = unit_open(r[2], r[3]);
  const double rad = std::sqrt(-2.0 * std::log(u1));
  const double th = 6.283185307179586 * u2;
  return (j & 1) ? rad * std::sin(th) : rad * std::cos(th);
}

// Gamma(shape, 1) by Marsaglia-Tsang with at most 64 attempts (the acceptance rate is above
// 0.95 for shape >= 1, so the cap is never reached in practice; if it is, the mode d is
// returned).
inline double gamma_draw(uint64_t seed, uint32_t sweep, uint32_t stream, uint32_t index,
                         double shape) {
  double boost = 1.0;
  if (shape < 1.0) {
    uint32_t r[4];
    philox_block(seed, sweep, stream, index, 1000u, r);
    boost = std::pow(unit_open(r[0], r[1]), 1.0 / shape);
    shape += 1.0;
  }
  const double d = shape - 1.0 / 3.0;
  const double c = 1.0 / std::sqrt(9.0 * d);
  for (uint32_t t = 0; t < 64; t++) {
    uint32_t r[4];
    philox_block(seed, sweep, stream, index, 2 * t, r);
    const double u1 = unit_open(r[0], r[1]);
    const double u2 = unit_open(r[2], r[3]);
    const double x = std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
    double v = 1.0 + c * x;
    if (v <= 0.0) continue;
    v = v * v * v;
    philox_block(seed, sweep, stream, index, 2 * t + 1, r);
    const double u = unit_open(r[0], r[1]);
    if (std::log(u) < 0.5 * x * x + d - d * v + d * std::log(v)) return d * v * boost;
  }
  return d * boost;
}

}  // namespace oracle
