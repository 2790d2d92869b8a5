// Per-row latent sampler (sample_latent_blas, latentprior.cpp:361-385, driven by the OpenMP row
// loops of latentprior.cpp:69-77 / 219-227), as one persistent sm_100a launch per mode.
//
// Work decomposition
//   * A "row group" of T = 32*WPR threads samples one row at a time; a CTA holds G groups.
//   * Rows come from a task list sorted by descending length and are taken from a device work
//     queue (atomic head in the control block), so power-law rows balance dynamically.
//   * Rows longer than the split threshold are cut into parts; each part writes its partial
//     Gram + right-hand side into a scratch slot, and the part that arrives last (per-row
//     atomic counter) sums the parts in part order (deterministic) and finishes the row.
//
// Per row: the gathered other-factor rows are staged in shared memory 32 at a time with 16-byte
// vector loads; each thread accumulates a TR x TC tile of the KP x KP Gram in registers and the
// first KP threads accumulate the right-hand side.  Finishing builds MM = Lambda + alpha*G and
// rr = sum v (y - mean) alpha + Lambda mu in shared memory, factorises MM = L L^T, solves
// L y = rr, adds N(0,1) draws and solves L^T x = y.
//
// FP64 path: FP64 everything (parity with the FP64 oracle).  Mixed path: BF16 gathered rows,
// FP32 Gram/factor/solves; a row whose FP32 pivot is not positive or falls below 2^-20 of its
// original diagonal is re-factorised in FP64 in the same launch (counted in ctl->retries).
#include <cuda_bf16.h>

#include "common.cuh"
#include "kernels.h"
#include "rng.cuh"
#include "warp_finish.cuh"

namespace mg {
namespace {

constexpr int kChunk = 32;  // gathered rows staged per step

template <int T>
__device__ __forceinline__ void gsync(int g) {
  if constexpr (T == 32) {
    __syncwarp();
  } else {
    asm volatile("bar.sync %0, %1;" ::"r"(g + 1), "n"(T) : "memory");
  }
}

// Gather element of the mixed path (the Gram precision): BF16 (default), FP16, or FP32 rounded
// to TF32 as it is read (the FP32 master copy, cvt.rna.tf32.f32).
enum GatherElem : int { kGeBf16 = 0, kGeFp16 = 1, kGeTf32 = 2 };

__device__ __forceinline__ float tf32_round(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return __uint_as_float(r);
}

template <int KP, int WPR, bool MIXED, int GE = kGeBf16>
struct Cfg {
  using Acc = typename std::conditional<MIXED, float, double>::type;
  using Elem16 = typename std::conditional<GE == kGeFp16, __half, __nv_bfloat16>::type;
  using ElemM = typename std::conditional<GE == kGeTf32, float, Elem16>::type;
  using Elem = typename std::conditional<MIXED, ElemM, double>::type;
  static constexpr int T = 32 * WPR;
  static constexpr int S = WPR == 1 ? 1 : (WPR == 4 ? 2 : 4);
  static constexpr int GR = 8 * S, GC = 4 * S;
  static constexpr int TR = KP / GR, TC = KP / GC;
  static constexpr int LD = KP + 1;  // leading dimension of MM in shared memory
  static constexpr int EV = 16 / sizeof(Elem);  // elements per 16-byte vector load
  static constexpr int VPR = KP / EV;           // vectors per gathered row
  static constexpr size_t kGath = sizeof(Acc) * kChunk * KP;
  // warp-per-row path: Gram tile (KP x LD, Acc) + L^T (KP x (KP+4)) or an FP64 L^T;
  // multi-warp path: FP64 MM (KP x LD)
  static constexpr size_t kMMw = sizeof(double) * KP * (KP + 4) > sizeof(Acc) * KP * (LD + KP + 4)
                                     ? sizeof(double) * KP * (KP + 4)
                                     : sizeof(Acc) * KP * (LD + KP + 4);
  static constexpr size_t kMM = WPR == 1 ? (kMMw > sizeof(double) * KP * LD ? kMMw
                                                                          : sizeof(double) * KP * LD)
                                         : sizeof(double) * KP * LD;
  static constexpr size_t kWork = (kGath > kMM ? kGath : kMM);
  // work | cidx[kChunk] | cw[kChunk] (double) | rr[KP] (double) | mun[KP] | diag[KP] | bcast[4]
  static constexpr size_t kGroupBytes =
      kWork + sizeof(int) * kChunk + sizeof(double) * (kChunk + 3 * KP) + 16;
  // CTA-wide Lambda + Lambda mu of the warp-per-row path
  static constexpr size_t kCtaBytes = WPR == 1 ? sizeof(double) * (KP * (KP + 1) + KP) : 0;
  static_assert(TR >= 1 && TC >= 1 && GR * TR == KP && GC * TC == KP, "tile");
  static_assert(VPR >= 1, "vector width");
};

// Cholesky + solves + noise for one row, in factor precision F.  MM (lower triangle, K x K),
// rr (right-hand side) and diag (original diagonal) are in shared memory.  Returns false if a
// pivot fails (nothing is written then).  All threads of the group return the same value.
template <typename F, int T, int GR, int GC>
__device__ bool factor_solve(F* M, int ld, F* rr, const double* diag, int K, int t, int g,
                             double rel_floor) {
  const int rt = t / GC, ct = t % GC;
  for (int j = 0; j < K; j++) {
    const F d = M[j * ld + j];
    const bool bad = !(d > (F)0) || !((double)d > rel_floor * diag[j]);
    gsync<T>(g);
    if (bad) return false;
    const F ljj = msqrt(d);
    for (int i = j + t; i < K; i += T) M[i * ld + j] = (i == j) ? ljj : M[i * ld + j] / ljj;
    gsync<T>(g);
    for (int i = j + 1 + rt; i < K; i += GR) {
      const F lij = M[i * ld + j];
      for (int k = j + 1 + ct; k <= i; k += GC) M[i * ld + k] -= lij * M[k * ld + j];
    }
    gsync<T>(g);
  }
  // L y = rr
  for (int j = 0; j < K; j++) {
    if (t == 0) rr[j] = rr[j] / M[j * ld + j];
    gsync<T>(g);
    const F yj = rr[j];
    for (int i = j + 1 + t; i < K; i += T) rr[i] -= M[i * ld + j] * yj;
    gsync<T>(g);
  }
  return true;
}

template <typename F, int T>
__device__ void back_solve(const F* M, int ld, F* rr, int K, int t, int g) {
  for (int j = K - 1; j >= 0; j--) {
    if (t == 0) rr[j] = rr[j] / M[j * ld + j];
    gsync<T>(g);
    const F xj = rr[j];
    for (int i = t; i < j; i += T) rr[i] -= M[j * ld + i] * xj;
    gsync<T>(g);
  }
}

template <typename F, int T>
__device__ void add_noise(const SampleParams& p, F* rr, int row, int K, int t, int g,
                          uint32_t sweep) {
  if (p.znoise) {
    for (int k = t; k < K; k += T) rr[k] += (F)p.znoise[(size_t)row * K + k];
  } else {
    const uint32_t st = stream_id(kRowNoise, (uint32_t)p.mode);
    for (int q = t; q < (K + 1) / 2; q += T) {
      double z0, z1;
      normal_pair(p.seed, sweep, st, (uint32_t)row, (uint32_t)q, &z0, &z1);
      rr[2 * q] += (F)z0;
      if (2 * q + 1 < K) rr[2 * q + 1] += (F)z1;
    }
  }
  gsync<T>(g);
}

// Minimum resident CTAs requested from the register allocator: the resident threads per SM
// (warp-per-row instances: 16 warps for FP32 Grams, 12 for FP64; 8 warps at WPR = 4, 16 at
// WPR = 16) divided by the CTA size, so every CTA shape gets the same register budget.
template <int WPR, int G, bool MIXED>
constexpr int min_ctas() {
  constexpr int thr = WPR == 1 ? (MIXED ? 512 : 384) : (WPR == 4 ? 256 : 512);
  return thr / (32 * WPR * G) > 0 ? thr / (32 * WPR * G) : 1;
}

template <int KP, int WPR, int G, bool MIXED, int GE = kGeBf16>
__global__ void __launch_bounds__(32 * WPR * G, (min_ctas<WPR, G, MIXED>())) k_sample(const SampleParams p) {
  using C = Cfg<KP, WPR, MIXED, GE>;
  using Acc = typename C::Acc;
  using Elem = typename C::Elem;
  constexpr int T = C::T, GR = C::GR, GC = C::GC, TR = C::TR, TC = C::TC, LD = C::LD;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int g = threadIdx.x / T, t = threadIdx.x % T;
  unsigned char* base = smem_raw + C::kCtaBytes + (size_t)g * C::kGroupBytes;
  // warp-per-row path: Lambda (row-major, ld KP+1) and, for BPMF, Lambda mu once per CTA
  double* Lam_s = reinterpret_cast<double*>(smem_raw);
  double* lmu_s = Lam_s + KP * (KP + 1);
  if constexpr (WPR == 1) {
    for (int e = threadIdx.x; e < KP * KP; e += blockDim.x) {
      const int i = e / KP, j = e % KP;
      Lam_s[i * (KP + 1) + j] = (i < p.K && j < p.K) ? p.Lambda[i + j * p.K] : 0.0;
    }
    __syncthreads();
    if (threadIdx.x < KP) {
      double sacc = 0.0;
      if ((int)threadIdx.x < p.K)
        for (int j = 0; j < p.K; j++) sacc += Lam_s[threadIdx.x * (KP + 1) + j] * p.mu[j];
      lmu_s[threadIdx.x] = sacc;
    }
    __syncthreads();
  }
  Acc* gath = reinterpret_cast<Acc*>(base);
  int* cidx = reinterpret_cast<int*>(base + C::kWork);
  double* cw = reinterpret_cast<double*>(cidx + kChunk);
  double* rrd = cw + kChunk;
  double* mun = rrd + KP;
  double* diag = mun + KP;
  int* bcast = reinterpret_cast<int*>(diag + KP);
  const int rt = t / GC, ct = t % GC;
  const int K = p.K;
  const uint32_t sweep = p.ctl->sweep;
  const Elem* other = reinterpret_cast<const Elem*>(p.other);

  const int ntasks = p.ntasks;
  const double alpha = noise_alpha(p);
  const double wscale = packed_scale(p);
  for (;;) {
    if (t == 0) bcast[0] = (int)atomicAdd(&p.ctl->queue[p.qslot], 1u);
    gsync<T>(g);
    const int ti = bcast[0];
    if (ti >= ntasks) break;
    const RowTask tk = p.tasks[ti];
    Acc acc[TR][TC];
#pragma unroll
    for (int i = 0; i < TR; i++)
#pragma unroll
      for (int j = 0; j < TC; j++) acc[i][j] = (Acc)0;
    Acc racc = (Acc)0;

    const long long end = tk.begin + tk.len;
    for (long long b = tk.begin; b < end; b += kChunk) {
      const int cnt = (int)min((long long)kChunk, end - b);
      for (int e = t; e < kChunk; e += T) {
        int c = 0;
        double w = 0.0;
        if (e < cnt) {
          if constexpr (MIXED) {
            const uint2 pk = p.packed[b + e];
            c = (int)pk.x;
            w = (double)__uint_as_float(pk.y) * wscale;
          } else {
            c = p.colidx[b + e];
            w = (p.vals[b + e] - p.mean) * alpha;
          }
        }
        cidx[e] = c;
        cw[e] = w;
      }
      gsync<T>(g);
      // gather: 16-byte vectors of the other factor's rows
#pragma unroll 4
      for (int e = t; e < kChunk * C::VPR; e += T) {
        const int r = e / C::VPR, v = e % C::VPR;
        if (r < cnt) {
          const uint4 raw = __ldg(reinterpret_cast<const uint4*>(other + (size_t)cidx[r] * KP) + v);
          Acc* dst = gath + r * KP + v * C::EV;
          if constexpr (MIXED && GE == kGeTf32) {
            const float4 f = *reinterpret_cast<const float4*>(&raw);
            dst[0] = tf32_round(f.x);
            dst[1] = tf32_round(f.y);
            dst[2] = tf32_round(f.z);
            dst[3] = tf32_round(f.w);
          } else if constexpr (MIXED && GE == kGeFp16) {
            const __half2* h = reinterpret_cast<const __half2*>(&raw);
#pragma unroll
            for (int q = 0; q < 4; q++) {
              const float2 f = __half22float2(h[q]);
              dst[2 * q] = f.x;
              dst[2 * q + 1] = f.y;
            }
          } else if constexpr (MIXED) {
            const __nv_bfloat162* h = reinterpret_cast<const __nv_bfloat162*>(&raw);
#pragma unroll
            for (int q = 0; q < 4; q++) {
              const float2 f = __bfloat1622float2(h[q]);
              dst[2 * q] = f.x;
              dst[2 * q + 1] = f.y;
            }
          } else {
            const double2 d = *reinterpret_cast<const double2*>(&raw);
            dst[0] = d.x;
            dst[1] = d.y;
          }
        }
      }
      gsync<T>(g);
      if (t < KP) {
        for (int r = 0; r < cnt; r++) racc += gath[r * KP + t] * (Acc)cw[r];
      }
      for (int r = 0; r < cnt; r++) {
        Acc a[TR], bb[TC];
#pragma unroll
        for (int i = 0; i < TR; i++) a[i] = gath[r * KP + rt * TR + i];
#pragma unroll
        for (int j = 0; j < TC; j++) bb[j] = gath[r * KP + ct * TC + j];
#pragma unroll
        for (int i = 0; i < TR; i++)
#pragma unroll
          for (int j = 0; j < TC; j++) acc[i][j] = mfma(a[i], bb[j], acc[i][j]);
      }
      gsync<T>(g);
    }

    if (tk.nparts > 1) {
      double* sp = p.scratch + (size_t)(tk.slot + tk.part) * (KP * KP + KP);
#pragma unroll
      for (int i = 0; i < TR; i++)
#pragma unroll
        for (int j = 0; j < TC; j++) sp[(rt * TR + i) * KP + ct * TC + j] = (double)acc[i][j];
      if (t < KP) sp[KP * KP + t] = (double)racc;
      __threadfence();
      gsync<T>(g);
      if (t == 0)
        bcast[1] = (atomicAdd(&p.split_cnt[tk.split], 1u) == (unsigned)(tk.nparts - 1)) ? 1 : 0;
      gsync<T>(g);
      if (!bcast[1]) continue;
      __threadfence();
      double dacc[TR][TC];
      double dr = 0.0;
#pragma unroll
      for (int i = 0; i < TR; i++)
#pragma unroll
        for (int j = 0; j < TC; j++) dacc[i][j] = 0.0;
      for (int q = 0; q < tk.nparts; q++) {
        const double* s = p.scratch + (size_t)(tk.slot + q) * (KP * KP + KP);
#pragma unroll
        for (int i = 0; i < TR; i++)
#pragma unroll
          for (int j = 0; j < TC; j++) dacc[i][j] += __ldcg(s + (rt * TR + i) * KP + ct * TC + j);
        if (t < KP) dr += __ldcg(s + KP * KP + t);
      }
#pragma unroll
      for (int i = 0; i < TR; i++)
#pragma unroll
        for (int j = 0; j < TC; j++) acc[i][j] = (Acc)dacc[i][j];
      racc = (Acc)dr;
      if (t == 0) p.split_cnt[tk.split] = 0u;
    }

    // ---- finish the row ----
    const int row = tk.row;
    if constexpr (WPR == 1) {
      // Gram tile -> shared memory (row-major, ld LD), then lane i owns row i of MM.
      Acc* Gs = reinterpret_cast<Acc*>(base);
#pragma unroll
      for (int i = 0; i < TR; i++)
#pragma unroll
        for (int j = 0; j < TC; j++) Gs[(rt * TR + i) * LD + ct * TC + j] = acc[i][j];
      __syncwarp();
      const int lane = t;
      const Acc rac = wshfl(racc, lane < KP ? lane : 0);  // rhs accumulator of component lane
      if (p.one) {  // univariate prior: coordinate draws from the Gram (warp_finish.cuh)
        Acc gr[KP];
#pragma unroll
        for (int j = 0; j < KP; j++) gr[j] = lane < K ? Gs[lane * LD + j] : (Acc)0;
        double u0 = 0.0;
        if (lane < K) {
          if constexpr (MIXED) u0 = (double)p.out_f32[(size_t)row * KP + lane];
          else u0 = p.out_f64[(size_t)row * KP + lane];
        }
        const double un = one_gs_warp<KP, Acc>(gr, (double)rac, u0, p, row, sweep, lane);
        if (lane < K) {
          if constexpr (MIXED) {
            p.out_f32[(size_t)row * KP + lane] = (float)un;
            store_copy(p, (size_t)row * KP + lane, (float)un);
          } else {
            p.out_f64[(size_t)row * KP + lane] = un;
          }
        }
        __syncwarp();
        continue;
      }
      double lm;
      if (p.uhat) {  // Macau prior mean mu + Uhat[row]
        const double mun = lane < K ? p.mu[lane] + p.uhat[(size_t)row * KP + lane] : 0.0;
        lm = 0.0;
        for (int j = 0; j < K; j++) {
          const double mj = wshfl(mun, j);
          if (lane < K) lm += Lam_s[lane * (KP + 1) + j] * mj;
        }
      } else {
        lm = lane < KP ? lmu_s[lane] : 0.0;
      }
      bool ok = false;
      if constexpr (MIXED) {
        float a[KP], d0 = 1.f, rinv = 1.f;
        warp_load_mm<float, float, KP>(a, d0, reinterpret_cast<const float*>(Gs), LD, Lam_s,
                                       alpha, lane, K);
        // L^T goes after the Gram tile, which must stay readable for an FP64 retry
        float* Lc = reinterpret_cast<float*>(base) + KP * LD;
        const double z = row_noise(p, row, K, lane, sweep);
        ok = warp_factor<float, KP>(a, rinv, lane, 0x1p-20, d0, Lc, KP + 4);
        if (ok) {
          const float x = warp_solve<float, KP>(a, rinv, (float)((double)rac + lm), lane, Lc,
                                                KP + 4, z);
          if (lane < K) {
            p.out_f32[(size_t)row * KP + lane] = x;
            store_copy(p, (size_t)row * KP + lane, x);
          }
        } else if (lane == 0) {
          atomicAdd(&p.ctl->retries[p.mode], 1u);
        }
      }
      if (!ok) {
        ok = warp_finish_f64<KP, Acc>(Gs, LD, Lam_s, (double)rac + lm, p, row, sweep, base);
        if (!ok && lane == 0) {
          atomicOr(&p.ctl->status, kStatCholFail);
          atomicCAS(&p.ctl->bad_row, -1, row);
        }
      }
      __syncwarp();
      continue;
    }
    if (p.one) {
      // univariate prior, K > 32: the coordinate draws of one_gs_warp by the group; thread d
      // owns coordinate d, G (full, FP64) in shared memory, the deltas broadcast through diag[]
      double* M = reinterpret_cast<double*>(base);
#pragma unroll
      for (int i = 0; i < TR; i++)
#pragma unroll
        for (int j = 0; j < TC; j++) {
          const int gi = rt * TR + i, gj = ct * TC + j;
          if (gi < K && gj < K) M[gi * LD + gj] = (double)acc[i][j];
        }
      double u = 0.0;
      if (t < K) {
        if constexpr (MIXED) u = (double)p.out_f32[(size_t)row * KP + t];
        else u = p.out_f64[(size_t)row * KP + t];
        mun[t] = u;
      }
      gsync<T>(g);
      const double alpha = noise_alpha(p);
      double tt = 0.0, lam = 1.0, m = 0.0, z = 0.0;
      const double c = (double)racc;
      if (t < K) {
        for (int j = 0; j < K; j++) tt = fma(M[t * LD + j], mun[j], tt);
        lam = p.Lambda[t + t * K];
        m = lam * (p.mu[t] + (p.uhat ? p.uhat[(size_t)row * KP + t] : 0.0));
        z = p.znoise ? p.znoise[(size_t)row * K + t]
                     : normal_draw(p.seed, sweep, stream_id(kRowNoise, (uint32_t)p.mode),
                                   (uint32_t)row, (uint32_t)t);
      }
      for (int d = 0; d < K; d++) {
        if (t == d) {
          const double gdd = M[d * LD + d];
          const double L = m + c - alpha * (tt - gdd * u);
          const double var = 1.0 / (lam + alpha * gdd);
          const double un = L * var + sqrt(var) * z;
          diag[d] = un - u;
          u = un;
        }
        gsync<T>(g);
        if (t < K) tt = fma(M[t * LD + d], diag[d], tt);
      }
      if (t < K) {
        if constexpr (MIXED) {
          p.out_f32[(size_t)row * KP + t] = (float)u;
          store_copy(p, (size_t)row * KP + t, (float)u);
        } else {
          p.out_f64[(size_t)row * KP + t] = u;
        }
      }
      gsync<T>(g);
      continue;
    }
    if (t < K) mun[t] = p.mu[t] + (p.uhat ? p.uhat[(size_t)row * KP + t] : 0.0);
    gsync<T>(g);
    double lmu = 0.0;
    if (t < K) {
      for (int j = 0; j < K; j++) lmu += p.Lambda[t + j * K] * mun[j];
    }
    gsync<T>(g);
    bool done = false;
    if constexpr (MIXED) {
      float* M = reinterpret_cast<float*>(base);
      float* rr = reinterpret_cast<float*>(rrd);
      const float af = (float)alpha;
#pragma unroll
      for (int i = 0; i < TR; i++)
#pragma unroll
        for (int j = 0; j < TC; j++) {
          const int gi = rt * TR + i, gj = ct * TC + j;
          if (gi < K && gj <= gi) {
            const float v = (float)p.Lambda[gi + gj * K] + af * acc[i][j];
            M[gi * LD + gj] = v;
            if (gi == gj) diag[gi] = (double)v;
          }
        }
      if (t < K) rr[t] = (float)((double)racc + lmu);
      gsync<T>(g);
      done = factor_solve<float, T, GR, GC>(M, LD, rr, diag, K, t, g, 0x1p-20);
      if (done) {
        add_noise<float, T>(p, rr, row, K, t, g, sweep);
        back_solve<float, T>(M, LD, rr, K, t, g);
        if (t < K) {
          p.out_f32[(size_t)row * KP + t] = rr[t];
          store_copy(p, (size_t)row * KP + t, rr[t]);
        }
      } else if (t == 0) {
        atomicAdd(&p.ctl->retries[p.mode], 1u);
      }
      gsync<T>(g);
    }
    if (!done) {
      double* M = reinterpret_cast<double*>(base);
      double* rr = rrd;
#pragma unroll
      for (int i = 0; i < TR; i++)
#pragma unroll
        for (int j = 0; j < TC; j++) {
          const int gi = rt * TR + i, gj = ct * TC + j;
          if (gi < K && gj <= gi) {
            const double v = p.Lambda[gi + gj * K] + alpha * (double)acc[i][j];
            M[gi * LD + gj] = v;
            if (gi == gj) diag[gi] = v;
          }
        }
      if (t < K) rr[t] = (double)racc + lmu;
      gsync<T>(g);
      const bool ok = factor_solve<double, T, GR, GC>(M, LD, rr, diag, K, t, g, 0.0);
      if (ok) {
        add_noise<double, T>(p, rr, row, K, t, g, sweep);
        back_solve<double, T>(M, LD, rr, K, t, g);
        if (t < K) {
          if constexpr (MIXED) {
            p.out_f32[(size_t)row * KP + t] = (float)rr[t];
            store_copy(p, (size_t)row * KP + t, (float)rr[t]);
          } else {
            p.out_f64[(size_t)row * KP + t] = rr[t];
          }
        }
      } else if (t == 0) {
        atomicOr(&p.ctl->status, kStatCholFail);
        atomicCAS(&p.ctl->bad_row, -1, row);
      }
      gsync<T>(g);
    }
  }
}

template <int KP, int WPR, int G, bool MIXED, int GE = kGeBf16>
void launch_t(const SampleParams& p, cudaStream_t s, int num_sms) {
  using C = Cfg<KP, WPR, MIXED, GE>;
  auto kern = k_sample<KP, WPR, G, MIXED, GE>;
  const size_t smem = C::kCtaBytes + C::kGroupBytes * G;
  static int per_sm_cache[64] = {0};  // per template instance and device
  int dev = 0;
  MG_CUDA(cudaGetDevice(&dev));
  int& per_sm = per_sm_cache[dev & 63];
  if (per_sm == 0) {
    MG_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int n = 0;
    MG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kern, 32 * WPR * G, smem));
    per_sm = n < 1 ? 1 : n;
  }
  const int need = (p.ntasks + G - 1) / G;
  int blocks = num_sms * per_sm;
  if (need < blocks) blocks = need > 0 ? need : 1;
  kern<<<blocks, 32 * WPR * G, smem, s>>>(p);
  MG_CUDA(cudaGetLastError());
}

// Row groups per CTA: the default shape, or the autotuner's alternative (groups = 2 at
// WPR = 1, 1 at WPR = 4) for BF16 gathers and FP64.
template <int GE>
void launch_mixed(const SampleParams& p, int KP, int groups, cudaStream_t s, int num_sms) {
  constexpr bool alt_ok = GE == kGeBf16;
  switch (KP) {
    case 8:
      if constexpr (alt_ok)
        if (groups == 2) return launch_t<8, 1, 2, true, GE>(p, s, num_sms);
      return launch_t<8, 1, 4, true, GE>(p, s, num_sms);
    case 16:
      if constexpr (alt_ok)
        if (groups == 2) return launch_t<16, 1, 2, true, GE>(p, s, num_sms);
      return launch_t<16, 1, 4, true, GE>(p, s, num_sms);
    case 32:
      if constexpr (alt_ok)
        if (groups == 2) return launch_t<32, 1, 2, true, GE>(p, s, num_sms);
      return launch_t<32, 1, 4, true, GE>(p, s, num_sms);
    case 64:
      if constexpr (alt_ok)
        if (groups == 1) return launch_t<64, 4, 1, true, GE>(p, s, num_sms);
      return launch_t<64, 4, 2, true, GE>(p, s, num_sms);
    case 128: return launch_t<128, 16, 1, true, GE>(p, s, num_sms);
  }
  throw MgError(MG_ERR_ARG, "unsupported latent dimension");
}

}  // namespace

int sample_default_groups(int KP) { return KP <= 32 ? 4 : (KP == 64 ? 2 : 1); }

std::vector<int> sample_group_options(int KP, bool mixed, int gram) {
  if (mixed && gram != kGeBf16) return {sample_default_groups(KP)};
  if (KP <= 32) return {4, 2};
  if (KP == 64) return {2, 1};
  return {1};
}

void launch_sample(const SampleParams& p, int KP, bool mixed, int gram, cudaStream_t s,
                   int num_sms, int groups) {
  if (mixed) {
    if (gram == kGeFp16) return launch_mixed<kGeFp16>(p, KP, groups, s, num_sms);
    if (gram == kGeTf32) return launch_mixed<kGeTf32>(p, KP, groups, s, num_sms);
    return launch_mixed<kGeBf16>(p, KP, groups, s, num_sms);
  } else {
    switch (KP) {
      case 8:
        if (groups == 2) return launch_t<8, 1, 2, false>(p, s, num_sms);
        return launch_t<8, 1, 4, false>(p, s, num_sms);
      case 16:
        if (groups == 2) return launch_t<16, 1, 2, false>(p, s, num_sms);
        return launch_t<16, 1, 4, false>(p, s, num_sms);
      case 32:
        if (groups == 2) return launch_t<32, 1, 2, false>(p, s, num_sms);
        return launch_t<32, 1, 4, false>(p, s, num_sms);
      case 64:
        if (groups == 1) return launch_t<64, 4, 1, false>(p, s, num_sms);
        return launch_t<64, 4, 2, false>(p, s, num_sms);
      case 128: return launch_t<128, 16, 1, false>(p, s, num_sms);
    }
  }
  throw MgError(MG_ERR_ARG, "unsupported latent dimension");
}

}  // namespace mg
