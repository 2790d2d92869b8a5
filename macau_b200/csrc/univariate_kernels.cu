// Prior update of the univariate sampler (MacauOnePrior, macauoneprior.cpp:189-290): the link
// matrix, one coefficient at a time, and the per-dimension lambda_beta.  The Normal-Wishart part
// (sample_mu_lambda) and compute_uhat reuse the BPMF statistics kernels and the SpMM.
#include <cuda_runtime.h>

#include <algorithm>

#include "common.cuh"
#include "kernels.h"
#include "rng.cuh"

namespace mg {
namespace {

constexpr int kBetaThreads = 512;
constexpr int kBetaWarps = kBetaThreads / 32;

// One link coefficient per lane d < dc (dimension d0 + d) of feature f, sample_beta's update
// (macauoneprior.cpp:243-252):
//   A = lambda_beta_d + lambda_d colsq_f,   B = lambda_d (zx_d + beta_df colsq_f),
//   beta_df <- B / A + z / sqrt(A),   delta_d = beta_df old - beta_df new.
// zx, lam, lb are this lane's components; the N(0,1) draw of (f, d0 + lane) comes from draws
// (filled by k_beta_draws before the sequential sweep); returns delta (0 for lanes >= dc).
__device__ __forceinline__ double beta_coef(int lane, int dc, int d0, int f, double zx,
                                            double lam, double lb, double cs, double* beta,
                                            int bstride, const double* __restrict__ draws) {
  if (lane >= dc) return 0.0;
  const int dx = d0 + lane;
  double* bp = beta + (size_t)f * bstride + dx;
  const double b = *bp;
  const double A = lb + lam * cs;
  const double B = lam * (zx + b * cs);
  const double Ainv = 1.0 / A;
  const double bn = B * Ainv + sqrt(Ainv) * draws[(size_t)f * bstride + dx];
  *bp = bn;
  return b - bn;
}

// sample_beta (macauoneprior.cpp:216-257) for the dimensions d0 .. d0 + 3 of block blockIdx.x.
// Z = U - mu - Uhat (N x zstride, this block's four columns) is formed first; then the features
// are visited level by level.  lvl_feat lists the features sorted by (level, index), where a
// feature's level is one more than the highest level of an earlier feature sharing a row with
// it, so the features of one level touch disjoint rows of Z and their updates commute: the
// result equals the reference's feature-by-feature order.  A level marked in lvl_warp (many
// features, or none longer than 1024 entries) gives one feature to each warp; the others give
// each feature in turn to the whole block.
template <typename T>
__global__ void __launch_bounds__(kBetaThreads)
    k_beta_one(const long long* __restrict__ tptr, const int* __restrict__ tidx,
               const double* __restrict__ tval, const double* __restrict__ colsq,
               const int* __restrict__ lvl_ptr, const int* __restrict__ lvl_feat,
               const int* __restrict__ lvl_warp, int nlevels, const T* __restrict__ U, int ustride, const double* __restrict__ mu,
               const double* __restrict__ uhat, int hstride, const double* __restrict__ Lambda,
               const double* __restrict__ lambda_beta, int K, long long N,
               double* __restrict__ beta, int bstride, double* __restrict__ Z, int zstride,
               const double* __restrict__ draws) {
  __shared__ double red[kBetaWarps][4];
  __shared__ double dl[4];
  const int d0 = blockIdx.x * 4, dc = min(4, K - d0);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  // this lane's dimension d0 + lane (lanes 0 .. dc - 1 update the coefficients)
  const double lam = lane < dc ? Lambda[(size_t)(d0 + lane) * (K + 1)] : 0.0;
  const double lb = lane < dc ? lambda_beta[d0 + lane] : 1.0;
  for (long long i = threadIdx.x; i < N; i += kBetaThreads)
    for (int d = 0; d < dc; d++)
      Z[i * zstride + d0 + d] =
          (double)U[i * ustride + d0 + d] - mu[d0 + d] - uhat[i * hstride + d0 + d];
  __syncthreads();
  for (int L = 0; L < nlevels; L++) {
    const int f0 = lvl_ptr[L], f1 = lvl_ptr[L + 1];
    if (lvl_warp[L]) {
      for (int q = f0 + warp; q < f1; q += kBetaWarps) {
        const int f = lvl_feat[q];
        double zx[4] = {0.0, 0.0, 0.0, 0.0};
        for (long long e = tptr[f] + lane; e < tptr[f + 1]; e += 32) {
          const double v = tval ? tval[e] : 1.0;
          const double* zr = Z + (size_t)tidx[e] * zstride + d0;
#pragma unroll
          for (int d = 0; d < 4; d++)
            if (d < dc) zx[d] = fma(v, zr[d], zx[d]);
        }
#pragma unroll
        for (int d = 0; d < 4; d++)
#pragma unroll
          for (int o = 16; o > 0; o >>= 1) zx[d] += __shfl_xor_sync(0xffffffffu, zx[d], o);
        double mine = 0.0;
#pragma unroll
        for (int d = 0; d < 4; d++)
          if (lane == d) mine = zx[d];
        const double my =
            beta_coef(lane, dc, d0, f, mine, lam, lb, colsq[f], beta, bstride, draws);
        double delta[4];
#pragma unroll
        for (int d = 0; d < 4; d++) delta[d] = __shfl_sync(0xffffffffu, my, d);
        for (long long e = tptr[f] + lane; e < tptr[f + 1]; e += 32) {
          const double v = tval ? tval[e] : 1.0;
          double* zr = Z + (size_t)tidx[e] * zstride + d0;
#pragma unroll
          for (int d = 0; d < 4; d++)
            if (d < dc) zr[d] = fma(v, delta[d], zr[d]);
        }
      }
    } else {
      for (int q = f0; q < f1; q++) {
        const int f = lvl_feat[q];
        double zx[4] = {0.0, 0.0, 0.0, 0.0};
        for (long long e = tptr[f] + threadIdx.x; e < tptr[f + 1]; e += kBetaThreads) {
          const double v = tval ? tval[e] : 1.0;
          const double* zr = Z + (size_t)tidx[e] * zstride + d0;
#pragma unroll
          for (int d = 0; d < 4; d++)
            if (d < dc) zx[d] = fma(v, zr[d], zx[d]);
        }
#pragma unroll
        for (int d = 0; d < 4; d++) {
#pragma unroll
          for (int o = 16; o > 0; o >>= 1) zx[d] += __shfl_xor_sync(0xffffffffu, zx[d], o);
          if (lane == 0) red[warp][d] = zx[d];
        }
        __syncthreads();
        if (warp == 0) {
          double s = 0.0;
          if (lane < dc)
            for (int w = 0; w < kBetaWarps; w++) s += red[w][lane];
          const double my =
              beta_coef(lane, dc, d0, f, s, lam, lb, colsq[f], beta, bstride, draws);
          if (lane < 4) dl[lane] = my;
        }
        __syncthreads();
        const double delta[4] = {dl[0], dl[1], dl[2], dl[3]};
        for (long long e = tptr[f] + threadIdx.x; e < tptr[f + 1]; e += kBetaThreads) {
          const double v = tval ? tval[e] : 1.0;
          double* zr = Z + (size_t)tidx[e] * zstride + d0;
#pragma unroll
          for (int d = 0; d < 4; d++)
            if (d < dc) zr[d] = fma(v, delta[d], zr[d]);
        }
      }
    }
    __syncthreads();
  }
}

// The same link sampler with one block per dimension d and this dimension's column of Z held in
// shared memory (N doubles, N <= kZsMax), so the feature-by-feature chain reads and writes no
// global memory but beta, with 32 warps per block and each feature's entry range (lvl_range)
// read in one load.  The sums are formed as in k_beta_one (lane-strided then an xor tree in a
// warp; thread-strided, per-warp trees, then the warps in order in a block).
constexpr int kZsMax = 26 * 1024;

// What a warp loads ahead about a feature: id, entry range, squared column norm, coefficient,
// draw, and this lane's first entry (row, value).
struct FeaturePre {
  int f;
  longlong2 rg;
  double cs, b, z;
  int i0;
  double v0;
};

__device__ __forceinline__ FeaturePre fetch_feature(int q, int lane, int d,
                                                   const int* __restrict__ lvl_feat,
                                                   const longlong2* __restrict__ lvl_range,
                                                   const double* __restrict__ colsq,
                                                   const double* beta, int bstride,
                                                   const double* __restrict__ draws,
                                                   const int* __restrict__ tidx,
                                                   const double* __restrict__ tval) {
  FeaturePre r;
  r.f = lvl_feat[q];
  r.rg = lvl_range[q];
  r.cs = colsq[r.f];
  r.b = beta[(size_t)r.f * bstride + d];
  r.z = draws[(size_t)r.f * bstride + d];
  const long long e = r.rg.x + lane;
  r.i0 = e < r.rg.y ? tidx[e] : 0;
  r.v0 = e < r.rg.y ? (tval ? tval[e] : 1.0) : 0.0;
  return r;
}
constexpr int kSmemThreads = 1024;
constexpr int kSmemWarps = kSmemThreads / 32;
template <typename T>
__global__ void __launch_bounds__(kSmemThreads)
    k_beta_one_smem(const int* __restrict__ tidx, const double* __restrict__ tval,
                    const double* __restrict__ colsq, const int* __restrict__ lvl_ptr,
                    const int* __restrict__ lvl_feat, const longlong2* __restrict__ lvl_range,
                    const int* __restrict__ lvl_warp, int nlevels, const T* __restrict__ U,
                    int ustride, const double* __restrict__ mu,
                    const double* __restrict__ uhat, int hstride,
                    const double* __restrict__ Lambda, const double* __restrict__ lambda_beta,
                    int K, int N, double* __restrict__ beta, int bstride,
                    const double* __restrict__ draws) {
  extern __shared__ double Zs[];
  __shared__ double red[kSmemWarps];
  __shared__ double dl;
  const int d = blockIdx.x;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const double lam = Lambda[(size_t)d * (K + 1)], lb = lambda_beta[d];
  for (int i = threadIdx.x; i < N; i += kSmemThreads)
    Zs[i] = (double)U[(size_t)i * ustride + d] - mu[d] - uhat[(size_t)i * hstride + d];
  __syncthreads();
  FeaturePre cur{};
  int cur_q = -1;
  bool have = false;
  for (int L = 0; L < nlevels; L++) {
    const int f0 = lvl_ptr[L], f1 = lvl_ptr[L + 1];
    if (lvl_warp[L]) {
      // one feature per warp; while a feature is processed, the warp loads everything about its
      // next one that no other feature changes (id, entry range, colsq, its coefficient and
      // draw, the first 32 entries), including the first feature it takes in the next level
      int q = f0 + warp;
      if (!(have && cur_q == q) && q < f1) {
        cur = fetch_feature(q, lane, d, lvl_feat, lvl_range, colsq, beta, bstride, draws, tidx,
                            tval);
        cur_q = q;
        have = true;
      }
      for (; q < f1; q += kSmemWarps) {
        int qn = q + kSmemWarps;
        if (qn >= f1) {
          qn = (L + 1 < nlevels && lvl_warp[L + 1] && f1 + warp < lvl_ptr[L + 2]) ? f1 + warp : -1;
        }
        FeaturePre nxt{};
        if (qn >= 0)
          nxt = fetch_feature(qn, lane, d, lvl_feat, lvl_range, colsq, beta, bstride, draws, tidx,
                              tval);
        double zx = 0.0;
        if (cur.rg.x + lane < cur.rg.y) zx = fma(cur.v0, Zs[cur.i0], zx);
#pragma unroll 4
        for (long long e = cur.rg.x + 32 + lane; e < cur.rg.y; e += 32)
          zx = fma(tval ? tval[e] : 1.0, Zs[tidx[e]], zx);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) zx += __shfl_xor_sync(0xffffffffu, zx, o);
        const double A = lb + lam * cur.cs;
        const double B = lam * (zx + cur.b * cur.cs);
        const double Ainv = 1.0 / A;
        const double bn = B * Ainv + sqrt(Ainv) * cur.z;
        const double my = cur.b - bn;
        if (lane == 0) beta[(size_t)cur.f * bstride + d] = bn;
        if (cur.rg.x + lane < cur.rg.y) Zs[cur.i0] = fma(cur.v0, my, Zs[cur.i0]);
#pragma unroll 4
        for (long long e = cur.rg.x + 32 + lane; e < cur.rg.y; e += 32)
          Zs[tidx[e]] = fma(tval ? tval[e] : 1.0, my, Zs[tidx[e]]);
        __syncwarp();
        cur = nxt;
        cur_q = qn;
        have = qn >= 0;
      }
    } else {
      for (int q = f0; q < f1; q++) {
        const int f = lvl_feat[q];
        const longlong2 rg = lvl_range[q];
        double cs = 0.0, bv = 0.0, zz = 0.0;  // thread 0 loads them before the reduction
        if (threadIdx.x == 0) {
          cs = colsq[f];
          bv = beta[(size_t)f * bstride + d];
          zz = draws[(size_t)f * bstride + d];
        }
        double zx = 0.0;
#pragma unroll 4
        for (long long e = rg.x + threadIdx.x; e < rg.y; e += kSmemThreads)
          zx = fma(tval ? tval[e] : 1.0, Zs[tidx[e]], zx);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) zx += __shfl_xor_sync(0xffffffffu, zx, o);
        if (lane == 0) red[warp] = zx;
        __syncthreads();
        if (threadIdx.x == 0) {
          double sum = 0.0;
          for (int w = 0; w < kSmemWarps; w++) sum += red[w];
          const double A = lb + lam * cs;
          const double B = lam * (sum + bv * cs);
          const double Ainv = 1.0 / A;
          const double bn = B * Ainv + sqrt(Ainv) * zz;
          beta[(size_t)f * bstride + d] = bn;
          dl = bv - bn;
        }
        __syncthreads();
        const double delta = dl;
#pragma unroll 4
        for (long long e = rg.x + threadIdx.x; e < rg.y; e += kSmemThreads)
          Zs[tidx[e]] = fma(tval ? tval[e] : 1.0, delta, Zs[tidx[e]]);
      }
    }
    __syncthreads();
  }
}

// The link sampler's N(0,1) draws, keyed (kBetaOne, feature f, dimension d) like
// bmrandn_single per feature (macauoneprior.cpp:241): draws[f * stride + d], one Philox block
// per pair of dimensions.
__global__ void k_beta_draws(long long nfeat, int K, int stride, const Ctl* ctl,
                             unsigned long long seed, int mode, double* __restrict__ draws) {
  const int pairs = (K + 1) / 2;
  const uint32_t st = stream_id(kBetaOne, (uint32_t)mode);
  const uint32_t sweep = ctl->sweep;
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < nfeat * pairs;
       e += (long long)gridDim.x * blockDim.x) {
    const long long f = e / pairs;
    const int q = (int)(e % pairs);
    double z0, z1;
    normal_pair(seed, sweep, st, (uint32_t)f, (uint32_t)q, &z0, &z1);
    draws[f * stride + 2 * q] = z0;
    if (2 * q + 1 < K) draws[f * stride + 2 * q + 1] = z1;
  }
}

// sample_lambda_beta (macauoneprior.cpp:267-290): lambda_beta_d ~ Gamma(a0 + nfeat / 2,
// 1 / (b0 + sum_f beta_df^2 / 2)), one warp per dimension, keyed (kLambdaBeta, d).
__global__ void k_lambda_beta_one(const double* __restrict__ beta, int bstride, long long nfeat,
                                  int K, double a0, double b0, const Ctl* ctl,
                                  unsigned long long seed, int mode,
                                  double* __restrict__ lambda_beta) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const double a = a0 + (double)nfeat / 2.0;
  for (int d = warp; d < K; d += blockDim.x >> 5) {
    double s = 0.0;
    for (long long f = lane; f < nfeat; f += 32) {
      const double b = beta[f * bstride + d];
      s = fma(b, b, s);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0)
      lambda_beta[d] = gamma_draw(seed, ctl->sweep, stream_id(kLambdaBeta, (uint32_t)mode),
                                  (uint32_t)d, a) *
                       (1.0 / (b0 + s / 2.0));
  }
}

}  // namespace

void launch_beta_one(const DevCsr& Ft, const double* colsq, const int* lvl_ptr,
                     const int* lvl_feat, const longlong2* lvl_range, const int* lvl_warp,
                     int nlevels, const void* U, bool f32, int ustride,
                     const double* mu, const double* uhat, int hstride, const double* Lambda,
                     const double* lambda_beta, int K, long long N, double* beta, int bstride,
                     double* Z, int zstride, double* draws, const Ctl* ctl,
                     unsigned long long seed, int mode, cudaStream_t s) {
  const long long work = Ft.nrow * ((K + 1) / 2);
  k_beta_draws<<<(int)std::min<long long>(4736, (work + 255) / 256), 256, 0, s>>>(
      Ft.nrow, K, bstride, ctl, seed, mode, draws);
  MG_CUDA(cudaGetLastError());
  if (N <= kZsMax) {  // one block per dimension, Z's column in shared memory
    const size_t smem = sizeof(double) * (size_t)N;
    static bool configured[64] = {false};
    int dev = 0;
    MG_CUDA(cudaGetDevice(&dev));
    if (!configured[dev & 63]) {
      MG_CUDA(cudaFuncSetAttribute(k_beta_one_smem<float>,
                                   cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)(sizeof(double) * kZsMax)));
      MG_CUDA(cudaFuncSetAttribute(k_beta_one_smem<double>,
                                   cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)(sizeof(double) * kZsMax)));
      configured[dev & 63] = true;
    }
    if (f32)
      k_beta_one_smem<float><<<K, kSmemThreads, smem, s>>>(
          Ft.idx, Ft.val, colsq, lvl_ptr, lvl_feat, lvl_range, lvl_warp, nlevels,
          (const float*)U, ustride, mu, uhat, hstride, Lambda, lambda_beta, K, (int)N, beta,
          bstride, draws);
    else
      k_beta_one_smem<double><<<K, kSmemThreads, smem, s>>>(
          Ft.idx, Ft.val, colsq, lvl_ptr, lvl_feat, lvl_range, lvl_warp, nlevels,
          (const double*)U, ustride, mu, uhat, hstride, Lambda, lambda_beta, K, (int)N, beta,
          bstride, draws);
    MG_CUDA(cudaGetLastError());
    return;
  }
  const int blocks = (K + 3) / 4;
  if (f32)
    k_beta_one<float><<<blocks, kBetaThreads, 0, s>>>(
        Ft.ptr, Ft.idx, Ft.val, colsq, lvl_ptr, lvl_feat, lvl_warp, nlevels, (const float*)U, ustride, mu,
        uhat, hstride, Lambda, lambda_beta, K, N, beta, bstride, Z, zstride, draws);
  else
    k_beta_one<double><<<blocks, kBetaThreads, 0, s>>>(
        Ft.ptr, Ft.idx, Ft.val, colsq, lvl_ptr, lvl_feat, lvl_warp, nlevels, (const double*)U, ustride, mu,
        uhat, hstride, Lambda, lambda_beta, K, N, beta, bstride, Z, zstride, draws);
  MG_CUDA(cudaGetLastError());
}

void launch_lambda_beta_one(const double* beta, int bstride, long long nfeat, int K, double a0,
                            double b0, const Ctl* ctl, unsigned long long seed, int mode,
                            double* lambda_beta, cudaStream_t s) {
  k_lambda_beta_one<<<1, 256, 0, s>>>(beta, bstride, nfeat, K, a0, b0, ctl, seed, mode,
                                      lambda_beta);
  MG_CUDA(cudaGetLastError());
}

}  // namespace mg
