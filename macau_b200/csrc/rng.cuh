// Keyed random draws used on the Gibbs-sweep path (host and device).
//
// The reference draws from thread-local std::mt19937 streams seeded by std::random_device and the
// wall clock (mvnormal.cpp:32-51, 59-79), so its draws cannot be reproduced.  This library keys
// every draw instead, so a run is reproducible and a CPU restatement can be fed the same draws:
//
//   Philox-4x32-10 (Salmon et al., SC'11)  ->  53-bit uniforms in (0,1)
//   N(0,1): Box-Muller on the two uniforms of one Philox block (draw j uses block j/2)
//   Gamma(shape, 1): Marsaglia & Tsang (ACM TOMS 2000), shape < 1 boosted by U^(1/shape)
//
// key     = {seed low 32 bits, seed high 32 bits}
// counter = {block, index, (purpose << 8) | mode, sweep}
#pragma once
#include <cstdint>

#ifdef __CUDACC__
#define MG_HD __host__ __device__ __forceinline__
#else
#define MG_HD inline
#include <cmath>
#endif

namespace mg {

enum Purpose : uint32_t {
  kRowNoise = 1,     // per-row noise of the latent sampler (latentprior.cpp:380-382)
  kMvnN = 2,         // MvNormal_prec_omp(Lambda, N) in sample_beta (latentprior.cpp:277)
  kMvnF = 3,         // MvNormal_prec_omp(Lambda, nfeat) in sample_beta (latentprior.cpp:278)
  kWishartOff = 4,   // Bartlett off-diagonal normals (mvnormal.cpp:225-226)
  kWishartDiag = 5,  // Bartlett diagonal chi draws (mvnormal.cpp:223-224)
  kMuDraw = 6,       // NormalWishart mean draw (mvnormal.cpp:273)
  kLambdaBeta = 7,   // lambda_beta Gamma draw (latentprior.cpp:328-331)
  kNoiseAlpha = 8,   // AdaptiveGaussianNoise precision Gamma draw (noisemodels.cpp:75-78)
  kBetaOne = 9,      // univariate link-matrix draws, one per (feature, dim) (macauoneprior.cpp:241)
};

MG_HD uint32_t stream_id(uint32_t purpose, uint32_t mode) { return (purpose << 8) | mode; }

MG_HD void philox(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3, uint32_t k0, uint32_t k1,
                  uint32_t out[4]) {
#pragma unroll
  for (int r = 0; r < 10; r++) {
    if (r > 0) {
      k0 += 0x9E3779B9u;
      k1 += 0xBB67AE85u;
    }
    const uint64_t p0 = (uint64_t)0xD2511F53u * c0;
    const uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
    const uint32_t n0 = (uint32_t)(p1 >> 32) ^ c1 ^ k0;
    const uint32_t n2 = (uint32_t)(p0 >> 32) ^ c3 ^ k1;
    c1 = (uint32_t)p1;
    c3 = (uint32_t)p0;
    c0 = n0;
    c2 = n2;
  }
  out[0] = c0;
  out[1] = c1;
  out[2] = c2;
  out[3] = c3;
}

MG_HD double unit_open(uint32_t hi, uint32_t lo) {
  const uint64_t x = (((uint64_t)hi << 32) | lo) >> 11;
  return ((double)x + 0.5) * (1.0 / 9007199254740992.0);
}

MG_HD void keyed_block(uint64_t seed, uint32_t sweep, uint32_t stream, uint32_t index,
                       uint32_t block, uint32_t out[4]) {
  philox(block, index, stream, sweep, (uint32_t)seed, (uint32_t)(seed >> 32), out);
}

// Both normals of block `pair` (draws 2*pair and 2*pair+1).
MG_HD void normal_pair(uint64_t seed, uint32_t sweep, uint32_t stream, uint32_t index,
                       uint32_t pair, double* z0, double* z1) {
  uint32_t r[4];
  keyed_block(seed, sweep, stream, index, pair, r);
  const double u1 = unit_open(r[0], r[1]);
  const double u2 = unit_open(r[2], r[3]);
  const double rad = sqrt(-2.0 * log(u1));
  const double th = 6.283185307179586 * u2;
  *z0 = rad * cos(th);
  *z1 = rad * sin(th);
}

#ifdef __CUDACC__
// normal_pair evaluated in FP32 from the same Philox block (the mixed-precision row samplers,
// whose draws are rounded to FP32 anyway): r = sqrt(-2 log u1) and the angle 2 pi u2 - pi, whose
// sine and cosine the SFU evaluates on [-pi, pi] (cos(a) = -cos(a - pi), sin(a) = -sin(a - pi)).
// The draws agree with normal_pair's to about 1e-6 relative; no branch of this code reaches a
// slow argument-reduction path.
__device__ __forceinline__ void normal_pair_f32(uint64_t seed, uint32_t sweep, uint32_t stream,
                                                uint32_t index, uint32_t pair, float* z0,
                                                float* z1) {
  uint32_t r[4];
  keyed_block(seed, sweep, stream, index, pair, r);
  const float u1 = (float)unit_open(r[0], r[1]);
  const float u2 = (float)unit_open(r[2], r[3]);
  const float rad = sqrtf(-2.f * logf(u1));
  const float th = 6.28318530717958648f * u2 - 3.14159265358979324f;
  *z0 = -rad * __cosf(th);
  *z1 = -rad * __sinf(th);
}
#endif

MG_HD double normal_draw(uint64_t seed, uint32_t sweep, uint32_t stream, uint32_t index,
                         uint32_t j) {
  double z0, z1;
  normal_pair(seed, sweep, stream, index, j >> 1, &z0, &z1);
  return (j & 1) ? z1 : z0;
}

MG_HD double gamma_draw(uint64_t seed, uint32_t sweep, uint32_t stream, uint32_t index,
                        double shape) {
  double boost = 1.0;
  uint32_t r[4];
  if (shape < 1.0) {
    keyed_block(seed, sweep, stream, index, 1000u, r);
    boost = pow(unit_open(r[0], r[1]), 1.0 / shape);
    shape += 1.0;
  }
  const double d = shape - 1.0 / 3.0;
  const double c = 1.0 / sqrt(9.0 * d);
  for (uint32_t t = 0; t < 64; t++) {
    keyed_block(seed, sweep, stream, index, 2 * t, r);
    const double u1 = unit_open(r[0], r[1]);
    const double u2 = unit_open(r[2], r[3]);
    const double x = sqrt(-2.0 * log(u1)) * cos(6.283185307179586 * u2);
    double v = 1.0 + c * x;
    if (v <= 0.0) continue;
    v = v * v * v;
    keyed_block(seed, sweep, stream, index, 2 * t + 1, r);
    const double u = unit_open(r[0], r[1]);
    if (log(u) < 0.5 * x * x + d - d * v + d * log(v)) return d * v * boost;
  }
  return d * boost;
}

}  // namespace mg
