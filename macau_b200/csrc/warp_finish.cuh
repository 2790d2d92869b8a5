// Warp-level finish of one sampler row (K <= 32): lane i holds row i of MM = Lambda + alpha*G,
// the warp factorises MM = L L^T, solves L y = rr, adds the row's N(0,1) draws and solves
// L^T x = y (sample_latent_blas, latentprior.cpp:373-384).  Shared by the CUDA-core sampler
// (sample_kernels.cu) and the tensor-core sampler (gram_tc.cu).
#pragma once
#include <cuda_bf16.h>

#include "common.cuh"
#include "rng.cuh"

namespace mg {

__device__ __forceinline__ float mfma(float a, float b, float c) { return fmaf(a, b, c); }
__device__ __forceinline__ double mfma(double a, double b, double c) { return fma(a, b, c); }
__device__ __forceinline__ float msqrt(float a) { return sqrtf(a); }
__device__ __forceinline__ double msqrt(double a) { return sqrt(a); }

__device__ __forceinline__ float wshfl(float v, int src) { return __shfl_sync(0xffffffffu, v, src); }
__device__ __forceinline__ double wshfl(double v, int src) { return __shfl_sync(0xffffffffu, v, src); }

__device__ __forceinline__ float mrsqrt(float a) { return rsqrtf(a); }
__device__ __forceinline__ double mrsqrt(double a) { return rsqrt(a); }

// Vector load of 4 consecutive values from shared memory (16-byte aligned for float).
template <typename F>
struct Vec4 {
  F v[4];
};
template <typename F>
__device__ __forceinline__ Vec4<F> lds4(const F* p) {
  Vec4<F> r;
  if constexpr (sizeof(F) == 4) {
    const float4 t = *reinterpret_cast<const float4*>(p);
    r.v[0] = t.x; r.v[1] = t.y; r.v[2] = t.z; r.v[3] = t.w;
  } else {
    const double2 t0 = *reinterpret_cast<const double2*>(p);
    const double2 t1 = *reinterpret_cast<const double2*>(p + 2);
    r.v[0] = t0.x; r.v[1] = t0.y; r.v[2] = t1.x; r.v[3] = t1.y;
  }
  return r;
}

// Warp Cholesky of the KP x KP matrix whose row i is held by lane i in a[] (lower triangle
// used; d0 = the lane's diagonal entry).  Right-looking over columns: entry (i, k) receives its
// updates in the order j = 0, 1, ... and is then scaled by 1/L(k, k).  The critical chain of a
// column step stays in registers and shuffles: each lane keeps its own diagonal in `diag`, the
// pivot lane forms 1/L(j, j) and shuffles it, and the next column's L(j+1, j) comes by
// shuffle; columns j+2 onwards read L(k, j) from shared memory (column j published as Lc row j,
// leading dimension ld, a multiple of 4) as 4-wide broadcasts, off the critical chain.  Every
// update is the same fma with the same operands as a plain right-looking loop, so the factor
// does not depend on this scheduling.  Entries above a lane's diagonal are never read for the
// factor or the solves, so the updates run unpredicated on every lane (the upper entries of a[]
// and a[lane] itself receive values that are discarded; a[lane] is overwritten by L(i, i) in
// its own step).  rinv receives the lane's 1/L(i, i).  A pivot that is not positive, or falls
// below rel_floor times the original diagonal d0, fails the whole warp.  On success Lc holds
// L^T (row j = column j of L; its entries above the diagonal are not meaningful).
template <typename F, int KP>
__device__ __forceinline__ bool warp_factor(F (&a)[KP], F& rinv, int lane, double rel_floor,
                                            F d0, F* Lc, int ld) {
  const F floor = (F)rel_floor * d0;
  F diag = d0;
  bool bad = false;
#pragma unroll
  for (int j = 0; j < KP; j++) {
    if (lane == j) bad = !(diag > (F)0) || !(diag > floor);
    const F r = wshfl(mrsqrt(diag), j);
    if (lane == j) rinv = r;
    a[j] = (lane == j ? diag : a[j]) * r;
    if (j + 1 < KP) {
      const F lnext = wshfl(a[j], j + 1);  // L(j+1, j)
      if (lane > j) diag = mfma(-a[j], a[j], diag);
      a[j + 1] = mfma(-a[j], lnext, a[j + 1]);
    }
    if (lane < KP) Lc[j * ld + lane] = a[j];
    __syncwarp();
#pragma unroll
    for (int q = (j + 2) / 4; q < KP / 4; q++) {
      const Vec4<F> c = lds4(Lc + j * ld + 4 * q);
#pragma unroll
      for (int u = 0; u < 4; u++) {
        const int k = 4 * q + u;
        if (k > j + 1) a[k] = mfma(-a[j], c.v[u], a[k]);
      }
    }
  }
  return !__any_sync(0xffffffffu, bad);
}

// y = L^{-1} rr (lane i holds rr_i and row i of L), rr += z, then x = L^{-T} rr with L^T read
// from Lc (row j = column j of L).  Returns x_i in lane i.
// The row's N(0,1) draw for component `lane` (0 beyond K): injected, or keyed by
// (seed, sweep, mode, row).  Computed before the factorisation so its latency overlaps it.
__device__ __forceinline__ double row_noise(const SampleParams& p, int row, int K, int lane,
                                            uint32_t sweep) {
  if (p.znoise) return lane < K ? p.znoise[(size_t)row * K + lane] : 0.0;
  double z0, z1;
  normal_pair(p.seed, sweep, stream_id(kRowNoise, (uint32_t)p.mode), (uint32_t)row,
              (uint32_t)(lane >> 1), &z0, &z1);
  return lane < K ? ((lane & 1) ? z1 : z0) : 0.0;
}

// Univariate finish of one row by a warp (MacauOnePrior::sample_latents,
// macauoneprior.cpp:41-95).  Lane d holds row d of the row's Gram G = sum_e v_e v_e^T (g), the
// rhs component c_d = sum_e w_e v_ed with w_e = alpha (y_e - mean), and the row's current value
// u_d (0 beyond K).  The coordinates are redrawn in order d = 0 .. K-1 with t = G u kept current:
//   L_d = lambda_d (mu_d + Uhat_d) + c_d - alpha (t_d - G_dd u_d),   Q_d = lambda_d + alpha G_dd,
//   u_d <- L_d / Q_d + z_d / sqrt(Q_d),   t += G[:, d] (u_d new - u_d old),
// lambda = diag(Lambda).  This is the reference's residual form with yhat_e = mean + v_e . u
// expanded through G: the same L_d and Q_d in exact arithmetic, O(K^2) per row after the Gram.
// Returns the new u for the lane.
template <int KP, typename GT>
__device__ __forceinline__ double one_gs_warp(const GT (&g)[KP], double c, double u,
                                              const SampleParams& p, int row, uint32_t sweep,
                                              int lane) {
  const int K = p.K;
  const double alpha = noise_alpha(p);
  const bool on = lane < K;
  const double lam = on ? p.Lambda[lane + lane * K] : 1.0;
  const double m =
      on ? lam * (p.mu[lane] + (p.uhat ? p.uhat[(size_t)row * KP + lane] : 0.0)) : 0.0;
  const double z = row_noise(p, row, K, lane, sweep);
  double t = 0.0;
#pragma unroll
  for (int j = 0; j < KP; j++) t = fma((double)g[j], __shfl_sync(0xffffffffu, u, j), t);
#pragma unroll
  for (int d = 0; d < KP; d++) {
    if (d >= K) break;
    double delta = 0.0;
    if (lane == d) {
      const double gdd = (double)g[d];
      const double L = m + c - alpha * (t - gdd * u);
      const double var = 1.0 / (lam + alpha * gdd);
      const double un = L * var + sqrt(var) * z;
      delta = un - u;
      u = un;
    }
    delta = __shfl_sync(0xffffffffu, delta, d);
    t = fma((double)g[d], delta, t);
  }
  return u;
}

template <typename F, int KP>
__device__ __forceinline__ F warp_solve(const F (&a)[KP], F rinv, F rr, int lane, const F* Lc,
                                        int ld, double z) {
#pragma unroll
  for (int j = 0; j < KP; j++) {
    if (lane == j) rr = rr * rinv;
    const F yj = wshfl(rr, j);
    if (lane > j) rr = mfma(-a[j], yj, rr);
  }
  rr += (F)z;
#pragma unroll
  for (int j = KP - 1; j >= 0; j--) {
    if (lane == j) rr = rr * rinv;
    const F xj = wshfl(rr, j);
    if (lane < j) rr = mfma(-Lc[lane * ld + j], xj, rr);
  }
  __syncwarp();
  return rr;
}

// ---- Two rows per warp (K <= 32, FP32): half-warp h factorises matrix h; lane l of the half holds
// rows l ("lo", columns 0..15, all a row l < 16 has in its lower triangle) and l + 16 ("hi",
// columns 0..31).  Every entry receives the same fma with the same operands, in the same
// order, as in warp_factor / warp_solve, so the results are identical; each column step's
// shuffles, rsqrt and barrier serve both matrices, and the short rows spend no instructions on
// the upper triangle.

__device__ __forceinline__ float hshfl(float v, int src) {
  return __shfl_sync(0xffffffffu, v, src, 16);
}

// The N(0,1) draw of component c (0 beyond K) of `row`: injected, or keyed by
// (seed, sweep, mode, row) exactly like row_noise.
__device__ __forceinline__ double comp_noise(const SampleParams& p, int row, int K, int c,
                                             uint32_t sweep) {
  if (p.znoise) return c < K ? p.znoise[(size_t)row * K + c] : 0.0;
  double z0, z1;
  normal_pair(p.seed, sweep, stream_id(kRowNoise, (uint32_t)p.mode), (uint32_t)row,
              (uint32_t)(c >> 1), &z0, &z1);
  return c < K ? ((c & 1) ? z1 : z0) : 0.0;
}

// Factorises this half's matrix; Lc (this half's, leading dimension ld, a multiple of 4)
// receives L^T.  Returns the half's verdict (pivot positive and above 2^-20 of its original
// diagonal, as warp_factor with rel_floor 2^-20).
__device__ __forceinline__ bool pair_factor(float (&lo)[16], float (&hi)[32], float& rinv_lo,
                                            float& rinv_hi, int l, float d0_lo, float d0_hi,
                                            float* Lc, int ld) {
  const float fl_lo = 0x1p-20f * d0_lo, fl_hi = 0x1p-20f * d0_hi;
  float dg_lo = d0_lo, dg_hi = d0_hi;
  bool bad = false;
#pragma unroll
  for (int j = 0; j < 32; j++) {
    const int o = j & 15;  // the lane of the half that owns row j
    const float dj = j < 16 ? dg_lo : dg_hi;
    if (l == o) bad |= !(dj > 0.f) || !(dj > (j < 16 ? fl_lo : fl_hi));
    const float r = hshfl(rsqrtf(dj), o);
    if (l == o) {
      if (j < 16) rinv_lo = r;
      else rinv_hi = r;
    }
    if (j < 16) lo[j] = (l == j ? dg_lo : lo[j]) * r;
    hi[j] = (l + 16 == j ? dg_hi : hi[j]) * r;
    if (j + 1 < 32) {
      const float ln = hshfl(j + 1 < 16 ? lo[j] : hi[j], (j + 1) & 15);  // L(j+1, j)
      if (j < 16 && l > j) dg_lo = fmaf(-lo[j], lo[j], dg_lo);
      if (l + 16 > j) dg_hi = fmaf(-hi[j], hi[j], dg_hi);
      if (j + 1 < 16) lo[j + 1] = fmaf(-lo[j], ln, lo[j + 1]);
      hi[j + 1] = fmaf(-hi[j], ln, hi[j + 1]);
    }
    if (j < 16) Lc[j * ld + l] = lo[j];
    Lc[j * ld + l + 16] = hi[j];
    __syncwarp();
#pragma unroll
    for (int q = (j + 2) / 4; q < 8; q++) {
      const Vec4<float> c = lds4(Lc + j * ld + 4 * q);
#pragma unroll
      for (int u = 0; u < 4; u++) {
        const int k = 4 * q + u;
        if (k > j + 1) {
          if (k < 16) lo[k] = fmaf(-lo[j], c.v[u], lo[k]);
          hi[k] = fmaf(-hi[j], c.v[u], hi[k]);
        }
      }
    }
  }
  const unsigned b = __ballot_sync(0xffffffffu, bad);
  return (b & (0xffffu << (16 * ((threadIdx.x & 31) >> 4)))) == 0u;
}

// y = L^{-1} b, y += z, x = L^{-T} y for this half's rows (r_lo, r_hi: b in, x out).
__device__ __forceinline__ void pair_solve(const float (&lo)[16], const float (&hi)[32],
                                           float rinv_lo, float rinv_hi, float& r_lo,
                                           float& r_hi, int l, const float* Lc, int ld,
                                           float z_lo, float z_hi) {
#pragma unroll
  for (int j = 0; j < 32; j++) {
    const int o = j & 15;
    if (l == o) {
      if (j < 16) r_lo = r_lo * rinv_lo;
      else r_hi = r_hi * rinv_hi;
    }
    const float yj = hshfl(j < 16 ? r_lo : r_hi, o);
    if (j < 16 && l > j) r_lo = fmaf(-lo[j], yj, r_lo);
    if (l + 16 > j) r_hi = fmaf(-hi[j], yj, r_hi);
  }
  r_lo += z_lo;
  r_hi += z_hi;
#pragma unroll
  for (int j = 31; j >= 0; j--) {
    const int o = j & 15;
    if (l == o) {
      if (j < 16) r_lo = r_lo * rinv_lo;
      else r_hi = r_hi * rinv_hi;
    }
    const float xj = hshfl(j < 16 ? r_lo : r_hi, o);
    if (l < j) r_lo = fmaf(-Lc[l * ld + j], xj, r_lo);
    if (l + 16 < j) r_hi = fmaf(-Lc[(l + 16) * ld + j], xj, r_hi);
  }
  __syncwarp();
}

// Row i of MM = Lambda + alpha * G for lane i (padded rows / columns of the identity), with G
// read from the Gram tile in shared memory (row-major, leading dimension ld).
template <typename F, typename GT, int KP>
__device__ __forceinline__ void warp_load_mm(F (&a)[KP], F& d0, const GT* Gs, int ld,
                                             const double* Lam_s, double alpha, int lane, int K) {
#pragma unroll
  for (int j = 0; j < KP; j++) {
    F v;
    if (lane < K && j < K) {
      if constexpr (sizeof(F) == 4)
        v = (float)Lam_s[lane * (KP + 1) + j] + (float)alpha * (float)Gs[lane * ld + j];
      else
        v = Lam_s[lane * (KP + 1) + j] + alpha * (double)Gs[lane * ld + j];
    } else {
      v = (lane == j) ? (F)1 : (F)0;
    }
    a[j] = v;
    if (j == lane) d0 = v;
  }
}

// FP64 finish of one row by one warp: MM = Lambda + alpha * G from the Gram tile Gs, Cholesky,
// solves and noise in FP64 (the FP64 path, and the retry of a row whose FP32 factor failed).
// Kept out of line so the FP32 path's register budget does not pay for it.  Writes the row and
// returns true, or returns false when the FP64 factor fails too.
template <int KP, typename GT>
__device__ __forceinline__ bool warp_finish_f64_body(const GT* Gs, int ld, const double* Lam_s,
                                             double rac_lm, const SampleParams& p, int row,
                                             uint32_t sweep, unsigned char* work) {
  const int lane = threadIdx.x & 31;
  const int K = p.K;
  double a[KP], d0 = 1.0, rinv = 1.0;
  const double z = row_noise(p, row, K, lane, sweep);
  warp_load_mm<double, GT, KP>(a, d0, Gs, ld, Lam_s, noise_alpha(p), lane, K);
  __syncwarp();
  double* Lc = reinterpret_cast<double*>(work);  // the Gram tile has been read into a[]
  if (!warp_factor<double, KP>(a, rinv, lane, 0.0, d0, Lc, KP + 4)) return false;
  const double x = warp_solve<double, KP>(a, rinv, rac_lm, lane, Lc, KP + 4, z);
  if (lane < K) {
    if (p.out_f64) {
      p.out_f64[(size_t)row * KP + lane] = x;
    } else {
      p.out_f32[(size_t)row * KP + lane] = (float)x;
      store_copy(p, (size_t)row * KP + lane, (float)x);
    }
  }
  return true;
}

template <int KP, typename GT>
__device__ __noinline__ bool warp_finish_f64(const GT* Gs, int ld, const double* Lam_s,
                                             double rac_lm, const SampleParams& p, int row,
                                             uint32_t sweep, unsigned char* work) {
  return warp_finish_f64_body<KP, GT>(Gs, ld, Lam_s, rac_lm, p, row, sweep, work);
}

}  // namespace mg

namespace mg {

// ---- Four rows per warp (K <= 32, FP32), the "quad" layout: quarter q = lane / 8 finishes
// matrix q, and lane i = lane % 8 of the quarter holds rows i, i + 8, i + 16, i + 24 (slot
// k = row / 8), row i + 8k with its columns 0 .. 8k + 7 at a[qoff(k) + c] (its lower triangle and
// the few entries above it, which receive discarded values).  Every lane holds 80 entries.
// Column broadcasts go through 8-wide shuffles, so the four matrices of a warp share every step
// of the dependency chain and no shared memory is needed.  The factor applies the same fma with
// the same operands in the same order as warp_factor / pair_factor, so it produces the same L.

__host__ __device__ constexpr int qoff(int k) { return 4 * k * (k + 1); }  // 0, 8, 24, 48

__device__ __forceinline__ float shfl8(float v, int src) {
  return __shfl_sync(0xffffffffu, v, src, 8);
}

// Factorises the quarter's matrix (d0[k]: the original diagonal entry of row i + 8k); rinv[k]
// receives 1 / L(i + 8k, i + 8k).  Returns the quarter's verdict: every pivot positive and above
// 2^-20 of its original diagonal (warp_factor with rel_floor 2^-20).
__device__ __forceinline__ bool quad_factor(float (&a)[80], float (&rinv)[4], int i,
                                            const float (&d0)[4]) {
  float dg[4];
#pragma unroll
  for (int k = 0; k < 4; k++) dg[k] = d0[k];
  bool bad = false;
#pragma unroll
  for (int j = 0; j < 32; j++) {
    const int jk = j >> 3, ji = j & 7;
    if (i == ji) bad |= !(dg[jk] > 0.f) || !(dg[jk] > 0x1p-20f * d0[jk]);
    const float r = shfl8(rsqrtf(dg[jk]), ji);
    if (i == ji) rinv[jk] = r;
#pragma unroll
    for (int k = 0; k < 4; k++)
      if (8 * k + 7 >= j) {
        const bool own = (i + 8 * k == j);
        a[qoff(k) + j] = (own ? dg[k] : a[qoff(k) + j]) * r;
      }
    if (j + 1 < 32) {
      const float lnext = shfl8(a[qoff((j + 1) >> 3) + j], (j + 1) & 7);  // L(j+1, j)
#pragma unroll
      for (int k = 0; k < 4; k++) {
        if (8 * k + 7 > j && i + 8 * k > j)
          dg[k] = fmaf(-a[qoff(k) + j], a[qoff(k) + j], dg[k]);
        if (8 * k + 7 >= j + 1)
          a[qoff(k) + j + 1] = fmaf(-a[qoff(k) + j], lnext, a[qoff(k) + j + 1]);
      }
    }
    // trailing columns c >= j + 2: L(c, j) from its owner, then a[k][c] -= L(i + 8k, j) L(c, j)
    // two columns (c even, c + 1) per packed FMA where both are due (the same fma per entry
    // as one at a time; half the FMA instructions)
    float lc[32];
#pragma unroll
    for (int c = 2; c < 32; c++)  // constant bounds so that every loop unrolls fully
      if (c >= j + 2) lc[c] = shfl8(a[qoff(c >> 3) + j], c & 7);  // L(c, j)
#pragma unroll
    for (int k = 0; k < 4; k++) {
      const float m = -a[qoff(k) + j];
#pragma unroll
      for (int c = 2; c < 32; c += 2) {
        if (8 * k + 7 < c) continue;  // both c and c + 1 lie in row slot k or neither does
        if (c >= j + 2) {
          const float2 r2 = __ffma2_rn(make_float2(m, m), make_float2(lc[c], lc[c + 1]),
                                       make_float2(a[qoff(k) + c], a[qoff(k) + c + 1]));
          a[qoff(k) + c] = r2.x;
          a[qoff(k) + c + 1] = r2.y;
        } else if (c + 1 >= j + 2) {
          a[qoff(k) + c + 1] = fmaf(m, lc[c + 1], a[qoff(k) + c + 1]);
        }
      }
    }
  }
  const unsigned b = __ballot_sync(0xffffffffu, bad);
  return ((b >> ((threadIdx.x & 31) & 24)) & 0xFFu) == 0u;
}

// y = L^{-1} b (the same operations as warp_solve's forward pass), y += z, then x = L^{-T} y by
// columns from the last: x_j = (y_j - sum_{r > j} L(r, j) x_r) / L(j, j), each sum reduced over
// the quarter's lanes.  b[k] (component i + 8k) holds the right-hand side in and x out.
__device__ __forceinline__ void quad_solve(const float (&a)[80], const float (&rinv)[4],
                                           float (&b)[4], const float (&z)[4], int i) {
#pragma unroll
  for (int j = 0; j < 32; j++) {
    const int jk = j >> 3, ji = j & 7;
    if (i == ji) b[jk] = b[jk] * rinv[jk];
    const float yj = shfl8(b[jk], ji);
#pragma unroll
    for (int k = 0; k < 4; k++)
      if (8 * k + 7 > j && i + 8 * k > j) b[k] = fmaf(-a[qoff(k) + j], yj, b[k]);
  }
#pragma unroll
  for (int k = 0; k < 4; k++) b[k] += z[k];
#pragma unroll
  for (int j = 31; j >= 0; j--) {
    const int jk = j >> 3, ji = j & 7;
    float part = 0.f;
#pragma unroll
    for (int k = 0; k < 4; k++)
      if (8 * k + 7 > j && i + 8 * k > j) part = fmaf(a[qoff(k) + j], b[k], part);
    part += __shfl_xor_sync(0xffffffffu, part, 4, 8);
    part += __shfl_xor_sync(0xffffffffu, part, 2, 8);
    part += __shfl_xor_sync(0xffffffffu, part, 1, 8);
    if (i == ji) b[jk] = (b[jk] - part) * rinv[jk];
  }
}

// The N(0,1) draws of components i + 8k (k = 0..3) of `row`, in FP32 (0 beyond K): injected, or
// keyed like comp_noise and evaluated in FP32 (normal_pair_f32, as the fused kernel's drainers
// do).  Lanes i and i ^ 1 need the two normals of the same four Philox blocks; each computes two
// blocks and they swap halves.
__device__ __forceinline__ void quad_noise(const SampleParams& p, int row, int K, int i,
                                           uint32_t sweep, float (&z)[4]) {
  if (p.znoise) {
#pragma unroll
    for (int k = 0; k < 4; k++) {
      const int c = i + 8 * k;
      z[k] = c < K ? (float)p.znoise[(size_t)row * K + c] : 0.f;
    }
    return;
  }
  const int odd = i & 1;
  float z0[2], z1[2];
#pragma unroll
  for (int t = 0; t < 2; t++)
    normal_pair_f32(p.seed, sweep, stream_id(kRowNoise, (uint32_t)p.mode), (uint32_t)row,
                    (uint32_t)((i >> 1) + 4 * (2 * odd + t)), &z0[t], &z1[t]);
  // even lane: its z0 of blocks k = 0, 1, and sends z1 of them; odd lane: its z1 of k = 2, 3
  const float s0 = __shfl_xor_sync(0xffffffffu, odd ? z0[0] : z1[0], 1);
  const float s1 = __shfl_xor_sync(0xffffffffu, odd ? z0[1] : z1[1], 1);
  float zz[4];
  if (odd) {
    zz[0] = s0;
    zz[1] = s1;
    zz[2] = z1[0];
    zz[3] = z1[1];
  } else {
    zz[0] = z0[0];
    zz[1] = z0[1];
    zz[2] = s0;
    zz[3] = s1;
  }
#pragma unroll
  for (int k = 0; k < 4; k++) z[k] = (i + 8 * k) < K ? zz[k] : 0.f;
}

}  // namespace mg
