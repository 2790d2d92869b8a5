// Normal-Wishart hyperprior update and test-set evaluation.
//
//   k_stats           per-block partial sums of x and x x^T over the rows of a latent matrix
//                     (optionally x = U - Uhat, the Macau residual of latentprior.cpp:257);
//                     FP64 accumulation from FP64 or FP32 latents.
//   k_stats32         the same for K <= 32 with 4 x 4 register tiles of the outer product (four
//                     row groups per block, summed in group order at the end).
//   k_nw32            k_normal_wishart for K <= 32: shared-memory matrices, warp-register
//                     Cholesky factors (warp_finish.cuh) and a warp-parallel triangular inverse.
//   k_normal_wishart  one CTA: reduces the partials in block order (deterministic), then
//                     CondNormalWishart -> NormalWishart -> Wishart/WishartUnit -> MvNormal_prec
//                     (mvnormal.cpp:169-184, 217-287, 314-336) in FP64 with keyed draws.
//   k_lambda_beta     one CTA: posterior_lambda_beta + rgamma (latentprior.cpp:317-331).
//   k_eval / k_eval_finish  eval_rmse (bpmfutils.h:86-114): online posterior mean / variance of
//                     the test predictions and the two RMSEs.
#include "common.cuh"
#include "kernels.h"
#include "rng.cuh"
#include "warp_finish.cuh"

namespace mg {
namespace {

constexpr int kStatThreads = 256;
constexpr int kStatRows = 32;  // rows staged per step

template <typename T, int PER>
__global__ void __launch_bounds__(kStatThreads)
    k_stats(const T* __restrict__ U, const double* __restrict__ Uhat, long long N, int K,
            int stride, int uhat_stride, long long rows_per_block, double* __restrict__ partials) {
  __shared__ double xs[kStatRows * 128];
  const int KK = K * K;
  const long long r0 = (long long)blockIdx.x * rows_per_block;
  const long long r1 = min(N, r0 + rows_per_block);
  double acc[PER];
  int ii[PER], jj[PER];
#pragma unroll
  for (int q = 0; q < PER; q++) {
    acc[q] = 0.0;
    const int e = threadIdx.x + q * kStatThreads;
    ii[q] = e < KK ? e % K : 0;
    jj[q] = e < KK ? e / K : 0;
  }
  double su = 0.0;
  for (long long b = r0; b < r1; b += kStatRows) {
    const int cnt = (int)min((long long)kStatRows, r1 - b);
    __syncthreads();
    for (int e = threadIdx.x; e < cnt * K; e += kStatThreads) {
      const int r = e / K, k = e % K;
      double x = (double)U[(b + r) * stride + k];
      if (Uhat) x -= Uhat[(b + r) * uhat_stride + k];
      xs[r * K + k] = x;
    }
    __syncthreads();
    if (threadIdx.x < K)
      for (int r = 0; r < cnt; r++) su += xs[r * K + threadIdx.x];
#pragma unroll
    for (int q = 0; q < PER; q++) {
      double s = acc[q];
      for (int r = 0; r < cnt; r++) s += xs[r * K + ii[q]] * xs[r * K + jj[q]];
      acc[q] = s;
    }
  }
  double* out = partials + (size_t)blockIdx.x * (K + KK);
  if (threadIdx.x < K) out[threadIdx.x] = su;
#pragma unroll
  for (int q = 0; q < PER; q++) {
    const int e = threadIdx.x + q * kStatThreads;
    if (e < KK) out[K + e] = acc[q];
  }
}

// In-place left-looking lower Cholesky of the K x K column-major matrix A by one CTA (thread i
// computes L(i, j)); the strict upper triangle is zeroed.  Returns false on a non-positive pivot
// (same value in every thread).
__device__ bool cta_chol(double* A, int K, bool* flag) {
  (void)flag;
  __syncthreads();
  for (int j = 0; j < K; j++) {
    double d = A[j + j * K];
    for (int p = 0; p < j; p++) d -= A[j + p * K] * A[j + p * K];
    if (!(d > 0.0)) {
      __syncthreads();
      return false;
    }
    const double ljj = sqrt(d);
    for (int i = j + 1 + threadIdx.x; i < K; i += blockDim.x) {
      double s = A[i + j * K];
      for (int p = 0; p < j; p++) s -= A[i + p * K] * A[j + p * K];
      A[i + j * K] = s / ljj;
    }
    __syncthreads();
    if (threadIdx.x == 0) A[j + j * K] = ljj;
    __syncthreads();
  }
  for (int q = threadIdx.x; q < K * K; q += blockDim.x) {
    const int i = q % K, k = q / K;
    if (i < k) A[i + k * K] = 0.0;
  }
  __syncthreads();
  return true;
}

// x <- L^{-1} x then L^{-T} x for one column, sequential in the calling thread.
__device__ void col_solve_llt(const double* L, double* x, int K, int xs) {
  for (int i = 0; i < K; i++) {
    double s = x[i * xs];
    for (int p = 0; p < i; p++) s -= L[i + p * K] * x[p * xs];
    x[i * xs] = s / L[i + i * K];
  }
  for (int i = K - 1; i >= 0; i--) {
    double s = x[i * xs];
    for (int p = i + 1; p < K; p++) s -= L[p + i * K] * x[p * xs];
    x[i * xs] = s / L[i + i * K];
  }
}

__global__ void __launch_bounds__(256)
    k_normal_wishart(const double* __restrict__ partials, int nparts, long long N, int K,
                     const double* __restrict__ mu0, double kappa, const double* __restrict__ T0,
                     int nu, const double* __restrict__ bb_partials, int bb_nparts,
                     const double* __restrict__ lambda_beta, NwWork w, Ctl* ctl,
                     unsigned long long seed, int mode, double* __restrict__ mu_out,
                     double* __restrict__ Lambda_out) {
  const int KK = K * K;
  const uint32_t sweep = ctl->sweep;
  double* NU = w.vec;          // K
  double* muc = w.vec + K;     // K
  double* z = w.vec + 2 * K;   // K
  double* X = w.m0;            // K x K
  double* Tc = w.m1;
  double* cB = w.m2;           // Bartlett factor (upper)
  double* W = w.m3;
  // 1. reduce partials in block order
  for (int e = threadIdx.x; e < K + KK; e += blockDim.x) {
    double s = 0.0;
    for (int b = 0; b < nparts; b++) s += partials[(size_t)b * (K + KK) + e];
    if (e < K) NU[e] = s;
    else X[e - K] = s;
  }
  if (bb_partials) {  // T = WI + lambda_beta * beta beta^T  (latentprior.cpp:258-260)
    const double lb = *lambda_beta;
    for (int e = threadIdx.x; e < KK; e += blockDim.x) {
      double s = 0.0;
      for (int b = 0; b < bb_nparts; b++) s += bb_partials[(size_t)b * (K + KK) + K + e];
      W[e] = T0[e] + lb * s;
    }
  } else {
    for (int e = threadIdx.x; e < KK; e += blockDim.x) W[e] = T0[e];
  }
  __syncthreads();
  const double kappa_c = kappa + (double)N;
  const int nu_c = nu + (int)N;
  for (int i = threadIdx.x; i < K; i += blockDim.x) muc[i] = (kappa * mu0[i] + NU[i]) / kappa_c;
  __syncthreads();
  // 2. X = T + NS + kappa mu0 mu0^T - kappa_c mu_c mu_c^T
  for (int e = threadIdx.x; e < KK; e += blockDim.x) {
    const int i = e % K, j = e / K;
    X[e] = W[e] + X[e] + kappa * mu0[i] * mu0[j] - kappa_c * muc[i] * muc[j];
  }
  // 3. T_c = X^{-1} through the Cholesky factor of X
  bool ok = cta_chol(X, K, nullptr);
  if (!ok) {
    if (threadIdx.x == 0) atomicOr(&ctl->status, kStatHyperFail);
    return;
  }
  for (int c = threadIdx.x; c < K; c += blockDim.x) {
    for (int i = 0; i < K; i++) Tc[i + c * K] = (i == c) ? 1.0 : 0.0;
    col_solve_llt(X, Tc + c * K, K, 1);
  }
  // 4. L = chol(T_c)
  ok = cta_chol(Tc, K, nullptr);
  if (!ok) {
    if (threadIdx.x == 0) atomicOr(&ctl->status, kStatHyperFail);
    return;
  }
  // 5. Bartlett factor c: c_ii = sqrt(2 Gamma((nu_c - i)/2)), c_ij ~ N(0,1) for j > i
  for (int e = threadIdx.x; e < KK; e += blockDim.x) {
    const int i = e % K, j = e / K;
    double v = 0.0;
    if (i == j)
      v = sqrt(2.0 * gamma_draw(seed, sweep, stream_id(kWishartDiag, mode), (uint32_t)i,
                                0.5 * (double)(nu_c - i)));
    else if (j > i)
      v = normal_draw(seed, sweep, stream_id(kWishartOff, mode), (uint32_t)i,
                      (uint32_t)(j - i - 1));
    cB[e] = v;
  }
  __syncthreads();
  // 6. W = c^T c ; M = L W (into X) ; Lambda = M L^T
  for (int e = threadIdx.x; e < KK; e += blockDim.x) {
    const int i = e % K, j = e / K;
    double s = 0.0;
    for (int p = 0; p < K; p++) s += cB[p + i * K] * cB[p + j * K];
    W[e] = s;
  }
  __syncthreads();
  for (int e = threadIdx.x; e < KK; e += blockDim.x) {
    const int i = e % K, j = e / K;
    double s = 0.0;
    for (int p = 0; p < K; p++) s += Tc[i + p * K] * W[p + j * K];
    X[e] = s;
  }
  __syncthreads();
  for (int e = threadIdx.x; e < KK; e += blockDim.x) {
    const int i = e % K, j = e / K;
    double s = 0.0;
    for (int p = 0; p < K; p++) s += X[i + p * K] * Tc[j + p * K];
    Lambda_out[e] = s;
    cB[e] = s * kappa_c;
  }
  // 7. mu = mu_c + chol(kappa_c Lambda)^{-T} z
  ok = cta_chol(cB, K, nullptr);
  if (!ok) {
    if (threadIdx.x == 0) atomicOr(&ctl->status, kStatHyperFail);
    return;
  }
  for (int i = threadIdx.x; i < K; i += blockDim.x)
    z[i] = normal_draw(seed, sweep, stream_id(kMuDraw, mode), 0u, (uint32_t)i);
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int i = K - 1; i >= 0; i--) {
      double s = z[i];
      for (int p = i + 1; p < K; p++) s -= cB[p + i * K] * z[p];
      z[i] = s / cB[i + i * K];
    }
  }
  __syncthreads();
  for (int i = threadIdx.x; i < K; i += blockDim.x) mu_out[i] = z[i] + muc[i];
}

// lambda_beta ~ Gamma(nux/2, 2 mux/nux), nux = nu + K nfeat,
// mux = mu nux / (nu + mu tr(B B^T Lambda))   (latentprior.cpp:317-331)
__global__ void k_lambda_beta(const double* __restrict__ bb_partials, int nparts, int K,
                              long long nfeat, const double* __restrict__ Lambda, double nu,
                              double mu, const Ctl* ctl, unsigned long long seed, int mode,
                              double* lambda_beta) {
  __shared__ double red[256];
  const int KK = K * K;
  double tr = 0.0;
  for (int e = threadIdx.x; e < KK; e += blockDim.x) {
    double s = 0.0;
    for (int b = 0; b < nparts; b++) s += bb_partials[(size_t)b * (K + KK) + K + e];
    const int i = e % K, j = e / K;
    tr += s * Lambda[j + i * K];
  }
  red[threadIdx.x] = tr;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int q = 0; q < (int)blockDim.x; q++) t += red[q];
    const double nux = nu + (double)K * (double)nfeat;
    const double mux = mu * nux / (nu + mu * t);
    const double b = nux / 2, c = 2 * mux / nux;
    *lambda_beta = c * gamma_draw(seed, ctl->sweep, stream_id(kLambdaBeta, mode), 0u, b);
  }
}

constexpr int kEvalThreads = 256;

// Groups of eight lanes take eight consecutive test entries at a time: for each entry the
// group reads the two latent rows with vector loads (lane l: elements 4l .. 4l + 3, + 32 j) and
// sums the partial dots with three shuffles; lane j keeps entry j's prediction and then does
// the online mean / variance update of eval_rmse (bpmfutils.h:86-114) for it, so the updates
// and their pred / pvar / value accesses run on all eight lanes.  Per block, the squared errors
// are summed in lane and group order into partials[2 * block .. + 1].
template <typename T>
__device__ __forceinline__ double dot4(const T* u, const T* v) {
  if constexpr (sizeof(T) == 4) {
    const float4 a = *reinterpret_cast<const float4*>(u), b = *reinterpret_cast<const float4*>(v);
    return (double)a.x * (double)b.x + (double)a.y * (double)b.y + (double)a.z * (double)b.z +
           (double)a.w * (double)b.w;
  } else {
    const double2 a0 = *reinterpret_cast<const double2*>(u), a1 = *reinterpret_cast<const double2*>(u + 2);
    const double2 b0 = *reinterpret_cast<const double2*>(v), b1 = *reinterpret_cast<const double2*>(v + 2);
    return a0.x * b0.x + a0.y * b0.y + a1.x * b1.x + a1.y * b1.y;
  }
}

template <typename T>
__global__ void __launch_bounds__(kEvalThreads)
    k_eval(const int* __restrict__ trow, const int* __restrict__ tcol,
           const double* __restrict__ tval, long long ntest, const T* __restrict__ U,
           const T* __restrict__ V, int K, int stride, double mean, int n_fixed, const Ctl* ctl,
           double* __restrict__ pred, double* __restrict__ pvar, double* __restrict__ partials) {
  constexpr int kGroups = kEvalThreads / 8;
  __shared__ double r1[kGroups], r2[kGroups];
  int n = n_fixed;
  if (n < 0) n = ((int)ctl->sweep < ctl->burnin) ? 0 : (int)ctl->sweep - ctl->burnin;
  const int g = threadIdx.x >> 3, l = threadIdx.x & 7;
  const unsigned mask = 0xffu << (8 * ((threadIdx.x & 31) >> 3));
  double se = 0.0, sea = 0.0;
  const long long step = (long long)gridDim.x * kGroups * 8;
  for (long long t0 = ((long long)blockIdx.x * kGroups + g) * 8; t0 < ntest; t0 += step) {
    const long long t = t0 + l;  // this lane's entry
    const bool own = t < ntest;
    const int r = own ? trow[t] : 0, c = own ? tcol[t] : 0;
    double mydot = 0.0;
#pragma unroll 2
    for (int j = 0; j < 8; j++) {
      const int rj = __shfl_sync(mask, r, j, 8), cj = __shfl_sync(mask, c, j, 8);
      const T* u = U + (size_t)rj * stride;
      const T* v = V + (size_t)cj * stride;
      double dot = 0.0;
      for (int k0 = 4 * l; k0 < K; k0 += 32) dot += dot4<T>(u + k0, v + k0);
      dot += __shfl_xor_sync(mask, dot, 4, 8);
      dot += __shfl_xor_sync(mask, dot, 2, 8);
      dot += __shfl_xor_sync(mask, dot, 1, 8);
      if (l == j) mydot = dot;
    }
    if (own) {
      const double p = mydot + mean;
      const double y = tval[t];
      se += (y - p) * (y - p);
      double pavg;
      if (n == 0) {
        pavg = p;
      } else {
        const double delta = p - pred[t];
        pavg = pred[t] + delta / (n + 1);
        pvar[t] += delta * (p - pavg);
      }
      sea += (y - pavg) * (y - pavg);
      pred[t] = pavg;
    }
  }
  // group sums in lane order
#pragma unroll
  for (int q = 1; q < 8; q++) {
    const double a1 = __shfl_sync(mask, se, q, 8), b1 = __shfl_sync(mask, sea, q, 8);
    if (l == 0) {
      se += a1;
      sea += b1;
    }
  }
  if (l == 0) {
    r1[g] = se;
    r2[g] = sea;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double a = 0.0, b = 0.0;
    for (int q = 0; q < kGroups; q++) {
      a += r1[q];
      b += r2[q];
    }
    partials[2 * blockIdx.x] = a;
    partials[2 * blockIdx.x + 1] = b;
  }
}

// One warp: lane q sums partials q, q + 32, ... in order, then a fixed shuffle tree.
__global__ void k_eval_finish(const double* partials, int nparts, long long ntest,
                              double* rmse) {
  const int lane = threadIdx.x & 31;
  double a = 0.0, b = 0.0;
  for (int q = lane; q < nparts; q += 32) {
    a += partials[2 * q];
    b += partials[2 * q + 1];
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    a += __shfl_xor_sync(0xffffffffu, a, o);
    b += __shfl_xor_sync(0xffffffffu, b, o);
  }
  if (lane == 0) {
    rmse[0] = sqrt(b / (double)ntest);  // posterior-mean RMSE (rmse_test)
    rmse[1] = sqrt(a / (double)ntest);  // single-sample RMSE (rmse_test_onesample)
  }
}

// Row of every CSR entry (the inverse of the row pointers): entry e lies in the row r with
// ptr[r] <= e < ptr[r + 1], found by binary search so that heavy rows cost no more than others.
__global__ void k_entry_rows(const long long* __restrict__ ptr, long long nrows, long long nnz,
                             int* __restrict__ erow) {
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < nnz; e += stride) {
    long long lo = 0, hi = nrows;  // invariant: ptr[lo] <= e < ptr[hi]
    while (hi - lo > 1) {
      const long long mid = (lo + hi) >> 1;
      if (ptr[mid] <= e) lo = mid;
      else hi = mid;
    }
    erow[e] = (int)lo;
  }
}

// Squared training residuals of AdaptiveGaussianNoise::update (noisemodels.cpp:55-72):
// (U_i . V_j + mean - y)^2 over the entries (i = erow[e], j = col[e], y = val[e]).  Same
// group layout as k_eval: eight lanes share the dot of one entry through vector loads and three
// shuffles, lane l keeps entry t0 + l; the per-block sum goes to partials[block] in lane and
// group order.
template <typename T>
__global__ void __launch_bounds__(kEvalThreads)
    k_noise_sse(const int* __restrict__ erow, const int* __restrict__ col,
                const double* __restrict__ val, long long nnz, const T* __restrict__ U,
                const T* __restrict__ V, int K, int stride, double mean,
                double* __restrict__ partials) {
  constexpr int kGroups = kEvalThreads / 8;
  __shared__ double r1[kGroups];
  const int g = threadIdx.x >> 3, l = threadIdx.x & 7;
  const unsigned mask = 0xffu << (8 * ((threadIdx.x & 31) >> 3));
  double se = 0.0;
  const long long step = (long long)gridDim.x * kGroups * 8;
  for (long long t0 = ((long long)blockIdx.x * kGroups + g) * 8; t0 < nnz; t0 += step) {
    const long long t = t0 + l;
    const bool own = t < nnz;
    const int r = own ? erow[t] : 0, c = own ? col[t] : 0;
    double mydot = 0.0;
#pragma unroll 2
    for (int j = 0; j < 8; j++) {
      const int rj = __shfl_sync(mask, r, j, 8), cj = __shfl_sync(mask, c, j, 8);
      const T* u = U + (size_t)rj * stride;
      const T* v = V + (size_t)cj * stride;
      double dot = 0.0;
      for (int k0 = 4 * l; k0 < K; k0 += 32) dot += dot4<T>(u + k0, v + k0);
      dot += __shfl_xor_sync(mask, dot, 4, 8);
      dot += __shfl_xor_sync(mask, dot, 2, 8);
      dot += __shfl_xor_sync(mask, dot, 1, 8);
      if (l == j) mydot = dot;
    }
    if (own) {
      const double d = (mydot + mean) - val[t];
      se += d * d;
    }
  }
#pragma unroll
  for (int q = 1; q < 8; q++) {
    const double a1 = __shfl_sync(mask, se, q, 8);
    if (l == 0) se += a1;
  }
  if (l == 0) r1[g] = se;
  __syncthreads();
  if (threadIdx.x == 0) {
    double a = 0.0;
    for (int q = 0; q < kGroups; q++) a += r1[q];
    partials[blockIdx.x] = a;
  }
}

// The precision draw of AdaptiveGaussianNoise::update (noisemodels.cpp:73-81), one warp: the
// partial sums in a fixed order, then aN = a0 + nnz / 2, bN = b0 + sumsq / 2 with
// (a0, b0) = (1/2, var_total / 2), alpha = Gamma(aN, 1) / bN capped at alpha_max, into ctl->alpha.
__global__ void k_noise_draw(const double* __restrict__ partials, int nparts, long long nnz,
                             double var_total, double alpha_max, Ctl* ctl,
                             unsigned long long seed) {
  const int lane = threadIdx.x & 31;
  double a = 0.0;
  for (int q = lane; q < nparts; q += 32) a += partials[q];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
  if (lane == 0) {
    const double aN = 0.5 + (double)nnz / 2.0;
    const double bN = 0.5 * var_total + a / 2.0;
    double alpha = gamma_draw(seed, ctl->sweep, stream_id(kNoiseAlpha, 0u), 0u, aN) * (1.0 / bN);
    if (alpha > alpha_max) alpha = alpha_max;
    ctl->alpha = alpha;
  }
}

__global__ void k_set_sweep(Ctl* ctl, uint32_t sweep, int burnin) {
  ctl->sweep = sweep;
  ctl->burnin = burnin;
}

__global__ void k_advance(Ctl* ctl) { ctl->sweep += 1u; }

// Column sums and outer-product sums of rows r0 .. r1 - 1 of (U - Uhat) for K <= 32: thread t
// owns the 4 x 4 tile (4 (t % 64) / 8 .., 4 (t % 8) ..) for the rows of row group t / 64 (every
// fourth staged row); the four groups are summed in group order at the end.  The next 32 rows
// are loaded into registers while the current ones are multiplied (double-buffered staging).
template <typename T>
__device__ __forceinline__ void stats_load(const T* U, const double* Uhat, long long b0, int cnt,
                                           int K, int stride, int uhat_stride, int t,
                                           double (&nx)[4]) {
#pragma unroll
  for (int q = 0; q < 4; q++) {
    const int e = t + kStatThreads * q, r = e >> 5, k = e & 31;
    double x = 0.0;
    if (r < cnt && k < K) {
      x = (double)U[(b0 + r) * stride + k];
      if (Uhat) x -= Uhat[(b0 + r) * uhat_stride + k];
    }
    nx[q] = x;
  }
}

// One block's statistics over rows r0 .. r1 - 1 into out[0 .. K + K*K) (shared by k_stats32 and
// the batched k_stats32_batch).
template <typename T>
__device__ __forceinline__ void stats32_rows(const T* __restrict__ U,
                                             const double* __restrict__ Uhat, long long r0,
                                             long long r1, int K, int stride, int uhat_stride,
                                             double* __restrict__ out) {
  static_assert(kStatRows * 32 == 4 * kStatThreads, "four staged values per thread");
  __shared__ __align__(16) double xs[2][kStatRows][36];
  __shared__ double red[3][64][17];
  const int KK = K * K;
  const int t = threadIdx.x, tile = t & 63, rg = t >> 6;
  const int ti = tile >> 3, tj = tile & 7;
  double acc[4][4];
#pragma unroll
  for (int a = 0; a < 4; a++)
#pragma unroll
    for (int b = 0; b < 4; b++) acc[a][b] = 0.0;
  double su = 0.0;
  double nx[4];
  stats_load(U, Uhat, r0, (int)max(0LL, min((long long)kStatRows, r1 - r0)), K, stride,
             uhat_stride, t, nx);
  int buf = 0;
  for (long long b0 = r0; b0 < r1; b0 += kStatRows) {
    const int cnt = (int)min((long long)kStatRows, r1 - b0);
#pragma unroll
    for (int q = 0; q < 4; q++) {
      const int e = t + kStatThreads * q;
      xs[buf][e >> 5][e & 31] = nx[q];
    }
    __syncthreads();
    const long long nb0 = b0 + kStatRows;
    if (nb0 < r1)
      stats_load(U, Uhat, nb0, (int)min((long long)kStatRows, r1 - nb0), K, stride, uhat_stride,
                 t, nx);
    if (t < K)
      for (int r = 0; r < cnt; r++) su += xs[buf][r][t];
#pragma unroll 2
    for (int r = rg; r < kStatRows; r += 4) {
      const double2 i01 = *reinterpret_cast<const double2*>(&xs[buf][r][4 * ti]);
      const double2 i23 = *reinterpret_cast<const double2*>(&xs[buf][r][4 * ti + 2]);
      const double2 j01 = *reinterpret_cast<const double2*>(&xs[buf][r][4 * tj]);
      const double2 j23 = *reinterpret_cast<const double2*>(&xs[buf][r][4 * tj + 2]);
      const double xi[4] = {i01.x, i01.y, i23.x, i23.y}, xj[4] = {j01.x, j01.y, j23.x, j23.y};
#pragma unroll
      for (int a = 0; a < 4; a++)
#pragma unroll
        for (int b = 0; b < 4; b++) acc[a][b] = fma(xi[a], xj[b], acc[a][b]);
    }
    buf ^= 1;
  }
  __syncthreads();
  if (rg > 0)
#pragma unroll
    for (int a = 0; a < 4; a++)
#pragma unroll
      for (int b = 0; b < 4; b++) red[rg - 1][tile][a * 4 + b] = acc[a][b];
  __syncthreads();
  if (t < K) out[t] = su;
  if (rg == 0) {
#pragma unroll
    for (int a = 0; a < 4; a++)
#pragma unroll
      for (int b = 0; b < 4; b++) {
        const double v = ((acc[a][b] + red[0][tile][a * 4 + b]) + red[1][tile][a * 4 + b]) +
                         red[2][tile][a * 4 + b];
        const int i = 4 * ti + a, j = 4 * tj + b;
        if (i < K && j < K) out[K + i + j * K] = v;
      }
  }
}

template <typename T>
__global__ void __launch_bounds__(kStatThreads)
    k_stats32(const T* __restrict__ U, const double* __restrict__ Uhat, long long N, int K,
              int stride, int uhat_stride, long long rows_per_block, double* __restrict__ partials) {
  const long long r0 = (long long)blockIdx.x * rows_per_block;
  stats32_rows(U, Uhat, r0, min(N, r0 + rows_per_block), K, stride, uhat_stride,
               partials + (size_t)blockIdx.x * (K + K * K));
}

// Sums `nparts` partial records of `len` doubles in a fixed order: CTA c owns elements
// 32 c .. 32 c + 31; warp w adds partials w, w + 8, ... in order, then the 8 warp sums are added
// in warp order.  out = one record.
__global__ void __launch_bounds__(256)
    k_reduce_parts(const double* __restrict__ parts, int nparts, int len, double* __restrict__ out) {
  __shared__ double ws[8][33];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int e = blockIdx.x * 32 + lane;
  double s = 0.0;
  if (e < len) {
#pragma unroll 8
    for (int b = warp; b < nparts; b += 8) s += parts[(size_t)b * len + e];
  }
  ws[warp][lane] = s;
  __syncthreads();
  if (warp == 0 && e < len) {
    double t = ws[0][lane];
#pragma unroll
    for (int w = 1; w < 8; w++) t += ws[w][lane];
    out[e] = t;
  }
}

// CondNormalWishart -> NormalWishart -> MvNormal_prec (mvnormal.cpp:169-184, 217-287, 314-336)
// for K <= 32 in one CTA of 256 threads, matrices in shared memory (row-major, ld 33), same
// draws as k_normal_wishart.  Two identities replace two of the reference's three Cholesky
// factorisations (results agree to FP64 rounding):
//   * chol(X^{-1}) = J M^{-T} J with M = chol(J X J), J the index reversal: one Cholesky of the
//     reversed X (warp 0's registers, warp_factor) and one triangular inverse Y = M^{-1}
//     (lane c solves M y = e_c), L(i, j) = Y(K-1-j, K-1-i);
//   * Lambda = L c^T c L^T = B B^T with B = L c^T lower triangular with positive diagonal, so
//     chol(kappa_c Lambda) = sqrt(kappa_c) B and mu = mu_c + B^{-T} z / sqrt(kappa_c).
// The Bartlett factor c and z are drawn by warps 1-7 while warp 0 factorises.
constexpr int kNwLd = 33;
constexpr int kNwLc = 36;

// T0 == null stands for the identity.
__device__ __forceinline__ void nw32_run(const double* __restrict__ partials, int nparts,
                                         long long N, int K, const double* __restrict__ mu0,
                                         double kappa, const double* __restrict__ T0, int nu,
                                         const double* __restrict__ bb_partials, int bb_nparts,
                                         const double* __restrict__ lambda_beta, Ctl* ctl,
                                         unsigned long long seed, int mode,
                                         double* __restrict__ mu_out,
                                         double* __restrict__ Lambda_out) {
  __shared__ double A[32 * kNwLd], Bm[32 * kNwLd], C[32 * kNwLd], D[32 * kNwLd];
  __shared__ __align__(16) double Lc[32 * kNwLc];
  __shared__ double NU[32], muc[32], m0[32], rl[32], zs[32];
  __shared__ int flag;
  const int t = threadIdx.x, lane = t & 31;
  const int KK = K * K;
  const uint32_t sweep = ctl->sweep;
  // 1. reduce partials in block order: NU = sum x, A = S = sum x x^T; Bm = T.  Thread t sums
  //    elements t + 256 q (q < 5) together so that its loads of one partial are in flight at once.
  {
    double sv[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
#pragma unroll 4
    for (int b = 0; b < nparts; b++) {
      const double* pb = partials + (size_t)b * (K + KK);
#pragma unroll
      for (int q = 0; q < 5; q++)
        if (t + 256 * q < K + KK) sv[q] += pb[t + 256 * q];
    }
#pragma unroll
    for (int q = 0; q < 5; q++) {
      const int e = t + 256 * q;
      if (e < K) NU[e] = sv[q];
      else if (e < K + KK) A[((e - K) % K) * kNwLd + (e - K) / K] = sv[q];
    }
  }
  if (bb_partials) {  // T = WI + lambda_beta * beta beta^T  (latentprior.cpp:258-260)
    const double lb = *lambda_beta;
    double sv[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll 4
    for (int b = 0; b < bb_nparts; b++) {
      const double* pb = bb_partials + (size_t)b * (K + KK) + K;
#pragma unroll
      for (int q = 0; q < 4; q++)
        if (t + 256 * q < KK) sv[q] += pb[t + 256 * q];
    }
#pragma unroll
    for (int q = 0; q < 4; q++) {
      const int e = t + 256 * q;
      if (e < KK) Bm[(e % K) * kNwLd + e / K] = (T0 ? T0[e] : (e % K == e / K ? 1.0 : 0.0)) + lb * sv[q];
    }
  } else {
    for (int e = t; e < KK; e += blockDim.x)
      Bm[(e % K) * kNwLd + e / K] = T0 ? T0[e] : (e % K == e / K ? 1.0 : 0.0);
  }
  if (t < K) m0[t] = mu0 ? mu0[t] : 0.0;
  __syncthreads();
  const double kappa_c = kappa + (double)N;
  const int nu_c = nu + (int)N;
  if (t < K) muc[t] = (kappa * m0[t] + NU[t]) / kappa_c;
  __syncthreads();
  // 2. X = T + NS + kappa mu0 mu0^T - kappa_c mu_c mu_c^T   (into A)
  for (int e = t; e < KK; e += blockDim.x) {
    const int i = e % K, j = e / K;
    A[i * kNwLd + j] =
        Bm[i * kNwLd + j] + A[i * kNwLd + j] + kappa * m0[i] * m0[j] - kappa_c * muc[i] * muc[j];
  }
  __syncthreads();
  if (t < 32) {
    // 3a. M = chol(J X J), M^T rows into Lc
    double a[32], d0 = 1.0, rinv = 1.0;
#pragma unroll
    for (int j = 0; j < 32; j++) {
      a[j] = (lane < K && j < K) ? A[(K - 1 - lane) * kNwLd + (K - 1 - j)] : (lane == j ? 1.0 : 0.0);
      if (j == lane) d0 = a[j];
    }
    const bool ok = warp_factor<double, 32>(a, rinv, lane, 0.0, d0, Lc, kNwLc);
    if (lane == 0) flag = ok ? 1 : 0;
    // 3b. Y = M^{-1}: lane c solves M y = e_c; Y(i, c) into D
    if (ok) {
      rl[lane] = rinv;
      __syncwarp();
      double y[32];
#pragma unroll
      for (int i = 0; i < 32; i++) {
        double s = (lane == i) ? 1.0 : 0.0;
#pragma unroll
        for (int q = 0; q < i; q++) s = fma(-Lc[q * kNwLc + i], y[q], s);
        y[i] = s * rl[i];
      }
#pragma unroll
      for (int i = 0; i < 32; i++) D[i * kNwLd + lane] = y[i];
    }
  } else {
    // 3c. Bartlett factor c (upper) into C: c_ii = sqrt(2 Gamma((nu_c - i)/2)), c_ij ~ N(0,1);
    //     z for the mean draw
    for (int e = t - 32; e < KK; e += blockDim.x - 32) {
      const int i = e % K, j = e / K;
      double v = 0.0;
      if (i == j)
        v = sqrt(2.0 * gamma_draw(seed, sweep, stream_id(kWishartDiag, mode), (uint32_t)i,
                                  0.5 * (double)(nu_c - i)));
      else if (j > i)
        v = normal_draw(seed, sweep, stream_id(kWishartOff, mode), (uint32_t)i,
                        (uint32_t)(j - i - 1));
      C[i * kNwLd + j] = v;
    }
    if (t - 32 < K) zs[t - 32] = normal_draw(seed, sweep, stream_id(kMuDraw, mode), 0u, (uint32_t)(t - 32));
  }
  __syncthreads();
  if (!flag) {
    if (t == 0) atomicOr(&ctl->status, kStatHyperFail);
    return;
  }
  // 4. L = chol(T_c) = chol(X^{-1}) into A: L(i, j) = Y(K-1-j, K-1-i), j <= i
  for (int e = t; e < KK; e += blockDim.x) {
    const int i = e % K, j = e / K;
    A[i * kNwLd + j] = (j <= i) ? D[(K - 1 - j) * kNwLd + (K - 1 - i)] : 0.0;
  }
  __syncthreads();
  // 5. B = L c^T (lower triangular): B(i, j) = sum_{q=j..i} L(i, q) c(j, q)
  for (int e = t; e < KK; e += blockDim.x) {
    const int i = e % K, j = e / K;
    double s = 0.0;
    for (int q = j; q <= i; q++) s += A[i * kNwLd + q] * C[j * kNwLd + q];
    Bm[i * kNwLd + j] = (j <= i) ? s : 0.0;
  }
  __syncthreads();
  // 6. Lambda = B B^T
  for (int e = t; e < KK; e += blockDim.x) {
    const int i = e % K, j = e / K;
    const int m = min(i, j);
    double s = 0.0;
    for (int q = 0; q <= m; q++) s += Bm[i * kNwLd + q] * Bm[j * kNwLd + q];
    Lambda_out[e] = s;
  }
  // 7. mu = mu_c + B^{-T} z / sqrt(kappa_c)
  if (t < 32) {
    double x = lane < K ? zs[lane] / sqrt(kappa_c) : 0.0;
    for (int j = K - 1; j >= 0; j--) {
      if (lane == j) x = x / Bm[j * kNwLd + j];
      const double xj = __shfl_sync(0xffffffffu, x, j);
      if (lane < j) x = fma(-Bm[j * kNwLd + lane], xj, x);
    }
    if (lane < K) mu_out[lane] = x + muc[lane];
  }
}

__global__ void __launch_bounds__(256)
    k_nw32(const double* __restrict__ partials, int nparts, long long N, int K,
           const double* __restrict__ mu0, double kappa, const double* __restrict__ T0, int nu,
           const double* __restrict__ bb_partials, int bb_nparts,
           const double* __restrict__ lambda_beta, Ctl* ctl, unsigned long long seed, int mode,
           double* __restrict__ mu_out, double* __restrict__ Lambda_out) {
  nw32_run(partials, nparts, N, K, mu0, kappa, T0, nu, bb_partials, bb_nparts, lambda_beta, ctl,
           seed, mode, mu_out, Lambda_out);
}

// ---- both modes' BPMF prior updates in one launch per step (K <= 32): blocks of mode 0, then
// of mode 1, each doing what the single-mode kernel's block does, so the results are the same
// bit for bit; the two modes' steps only overlap ----
template <typename T>
__global__ void __launch_bounds__(kStatThreads)
    k_stats32_pair(PriorPair pp, int K, int stride) {
  const int m = blockIdx.x < pp.nblocks[0] ? 0 : 1;
  const int b = blockIdx.x - (m ? pp.nblocks[0] : 0);
  const long long r0 = (long long)b * pp.rows_per_block[m];
  stats32_rows(static_cast<const T*>(pp.U[m]), nullptr, r0, min(pp.N[m], r0 + pp.rows_per_block[m]),
               K, stride, 0, pp.partials[m] + (size_t)b * (K + K * K));
}

__global__ void __launch_bounds__(256) k_reduce_parts_pair(PriorPair pp, int len) {
  __shared__ double ws[8][33];
  const int nblk = (len + 31) / 32;
  const int m = blockIdx.x < nblk ? 0 : 1;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int e = (blockIdx.x - (m ? nblk : 0)) * 32 + lane;
  const double* parts = pp.partials[m];
  const int nparts = pp.nblocks[m];
  double s = 0.0;
  if (e < len) {
#pragma unroll 8
    for (int b = warp; b < nparts; b += 8) s += parts[(size_t)b * len + e];
  }
  ws[warp][lane] = s;
  __syncthreads();
  if (warp == 0 && e < len) {
    double t = ws[0][lane];
#pragma unroll
    for (int w = 1; w < 8; w++) t += ws[w][lane];
    pp.final_[m][e] = t;
  }
}

__global__ void __launch_bounds__(256) k_nw32_pair(PriorPair pp, int K, Ctl* ctl,
                                                   unsigned long long seed) {
  const int m = blockIdx.x;
  nw32_run(pp.final_[m], 1, pp.N[m], K, pp.mu0[m], pp.kappa[m], pp.T0[m], pp.nu[m], nullptr, 0,
           nullptr, ctl, seed, m, pp.mu[m], pp.Lambda[m]);
}

}  // namespace

void launch_prior_pair(const PriorPair& pp, bool f32, int K, int stride, Ctl* ctl,
                       unsigned long long seed, cudaStream_t s) {
  if (K > 32) throw MgError(MG_ERR_ARG, "the two-mode prior update needs K <= 32");
  const int nb = pp.nblocks[0] + pp.nblocks[1];
  if (f32)
    k_stats32_pair<float><<<nb, kStatThreads, 0, s>>>(pp, K, stride);
  else
    k_stats32_pair<double><<<nb, kStatThreads, 0, s>>>(pp, K, stride);
  MG_CUDA(cudaGetLastError());
  const int len = K + K * K;
  k_reduce_parts_pair<<<2 * ((len + 31) / 32), 256, 0, s>>>(pp, len);
  MG_CUDA(cudaGetLastError());
  k_nw32_pair<<<2, 256, 0, s>>>(pp, K, ctl, seed);
  MG_CUDA(cudaGetLastError());
}

int stats_blocks(long long N) {  // at most two blocks per SM: fewer partials to reduce
  long long b = (N + 127) / 128;
  if (b > 296) b = 296;
  return (int)(b < 1 ? 1 : b);
}

void launch_stats(const void* U, bool f32, const double* Uhat, long long N, int K, int stride,
                  int uhat_stride, double* partials, int nblocks, cudaStream_t s) {
  if (K > 128) throw MgError(MG_ERR_ARG, "K > 128 is not supported");
  const long long rpb = (N + nblocks - 1) / nblocks;
  if (K <= 32) {
    if (f32)
      k_stats32<float><<<nblocks, kStatThreads, 0, s>>>((const float*)U, Uhat, N, K, stride,
                                                        uhat_stride, rpb, partials);
    else
      k_stats32<double><<<nblocks, kStatThreads, 0, s>>>((const double*)U, Uhat, N, K, stride,
                                                         uhat_stride, rpb, partials);
    MG_CUDA(cudaGetLastError());
    return;
  }
  const int per = (K * K + kStatThreads - 1) / kStatThreads;
#define MG_STATS(P)                                                                         \
  if (per <= P) {                                                                           \
    if (f32)                                                                                \
      k_stats<float, P><<<nblocks, kStatThreads, 0, s>>>((const float*)U, Uhat, N, K, stride, \
                                                         uhat_stride, rpb, partials);       \
    else                                                                                    \
      k_stats<double, P><<<nblocks, kStatThreads, 0, s>>>((const double*)U, Uhat, N, K,     \
                                                          stride, uhat_stride, rpb, partials); \
    MG_CUDA(cudaGetLastError());                                                            \
    return;                                                                                 \
  }
  MG_STATS(1)
  MG_STATS(4)
  MG_STATS(16)
  MG_STATS(64)
#undef MG_STATS
}

// ---- batched problems (batch.cu): one statistics block and one Normal-Wishart block per
// problem; problem p owns rows row0[p] .. row0[p + 1] - 1 of U (stride 32), K = Kp[p] ----
__global__ void __launch_bounds__(kStatThreads)
    k_stats_batch(const float* __restrict__ U, const int* __restrict__ row0,
                  const int* __restrict__ Kp, double* __restrict__ partials) {
  const int p = blockIdx.x;
  stats32_rows<float>(U, nullptr, row0[p], row0[p + 1], Kp[p], 32, 0,
                      partials + (size_t)p * (32 + 32 * 32));
}

// BPMFPrior::update_prior per problem with mu0 = 0, b0 = 2, W0 = I, df = K_p
// (latentprior.cpp:79-99), keyed with the problem's seed; then the finish's operands: the FP32
// Lambda (32 x 32, zero beyond K) and Lambda mu (FP64, summed in column order).
__global__ void __launch_bounds__(256)
    k_nw_batch(const double* __restrict__ partials, const int* __restrict__ row0,
               const int* __restrict__ Kp, const unsigned long long* __restrict__ seed, Ctl* ctl,
               int mode, double* __restrict__ mu, double* __restrict__ Lambda,
               float* __restrict__ LamF, double* __restrict__ lmu) {
  const int p = blockIdx.x, K = Kp[p];
  double* L = Lambda + (size_t)p * 1024;
  double* m = mu + (size_t)p * 32;
  nw32_run(partials + (size_t)p * (32 + 32 * 32), 1, row0[p + 1] - row0[p], K, nullptr, 2.0,
           nullptr, K, nullptr, 0, nullptr, ctl, seed[p], mode, m, L);
  __syncthreads();
  for (int e = threadIdx.x; e < 1024; e += blockDim.x) {
    const int i = e >> 5, j = e & 31;
    LamF[(size_t)p * 1024 + e] = (i < K && j < K) ? (float)L[i + j * K] : 0.f;
  }
  if (threadIdx.x < 32) {
    double acc = 0.0;
    if ((int)threadIdx.x < K)
      for (int j = 0; j < K; j++) acc += L[threadIdx.x + j * K] * m[j];
    lmu[(size_t)p * 32 + threadIdx.x] = acc;
  }
}

void launch_prior_batch(const float* U, const int* row0, const int* Kp,
                        const unsigned long long* seed, int P, double* partials, Ctl* ctl, int mode,
                        double* mu, double* Lambda, float* LamF, double* lmu, cudaStream_t s) {
  k_stats_batch<<<P, kStatThreads, 0, s>>>(U, row0, Kp, partials);
  MG_CUDA(cudaGetLastError());
  k_nw_batch<<<P, 256, 0, s>>>(partials, row0, Kp, seed, ctl, mode, mu, Lambda, LamF, lmu);
  MG_CUDA(cudaGetLastError());
}

void launch_reduce_parts(const double* parts, int nparts, int len, double* out, cudaStream_t s) {
  k_reduce_parts<<<(len + 31) / 32, 256, 0, s>>>(parts, nparts, len, out);
  MG_CUDA(cudaGetLastError());
}

void launch_normal_wishart(const double* partials, int nparts, long long N, int K,
                           const double* mu0, double kappa, const double* T0, int nu,
                           const double* bb_partials, int bb_nparts, const double* lambda_beta,
                           const NwWork& w, Ctl* ctl, unsigned long long seed, int mode,
                           double* mu_out, double* Lambda_out, cudaStream_t s) {
  if (K <= 32)
    k_nw32<<<1, 256, 0, s>>>(partials, nparts, N, K, mu0, kappa, T0, nu, bb_partials, bb_nparts,
                             lambda_beta, ctl, seed, mode, mu_out, Lambda_out);
  else
    k_normal_wishart<<<1, 256, 0, s>>>(partials, nparts, N, K, mu0, kappa, T0, nu, bb_partials,
                                       bb_nparts, lambda_beta, w, ctl, seed, mode, mu_out,
                                       Lambda_out);
  MG_CUDA(cudaGetLastError());
}

void launch_lambda_beta(const double* bb_partials, int nparts, int K, long long nfeat,
                        const double* Lambda, double nu, double mu, const Ctl* ctl,
                        unsigned long long seed, int mode, double* lambda_beta, cudaStream_t s) {
  k_lambda_beta<<<1, 256, 0, s>>>(bb_partials, nparts, K, nfeat, Lambda, nu, mu, ctl, seed,
                                  mode, lambda_beta);
  MG_CUDA(cudaGetLastError());
}

int eval_blocks(long long ntest) {
  long long b = (ntest + kEvalThreads - 1) / kEvalThreads;
  if (b > 1184) b = 1184;
  return (int)(b < 1 ? 1 : b);
}

void launch_eval(const int* trow, const int* tcol, const double* tval, long long ntest,
                 const void* U, const void* V, bool f32, int K, int stride, double mean,
                 int n_fixed, const Ctl* ctl, double* pred, double* pvar, double* partials,
                 int nblocks, double* rmse, cudaStream_t s) {
  if (f32)
    k_eval<float><<<nblocks, kEvalThreads, 0, s>>>(trow, tcol, tval, ntest, (const float*)U,
                                                   (const float*)V, K, stride, mean, n_fixed,
                                                   ctl, pred, pvar, partials);
  else
    k_eval<double><<<nblocks, kEvalThreads, 0, s>>>(trow, tcol, tval, ntest, (const double*)U,
                                                    (const double*)V, K, stride, mean, n_fixed,
                                                    ctl, pred, pvar, partials);
  MG_CUDA(cudaGetLastError());
  k_eval_finish<<<1, 32, 0, s>>>(partials, nblocks, ntest, rmse);
  MG_CUDA(cudaGetLastError());
}

void launch_entry_rows(const long long* ptr, long long nrows, long long nnz, int* erow,
                       cudaStream_t s) {
  if (nnz <= 0) return;
  long long b = (nnz + 255) / 256;
  if (b > 4736) b = 4736;
  k_entry_rows<<<(int)b, 256, 0, s>>>(ptr, nrows, nnz, erow);
  MG_CUDA(cudaGetLastError());
}

void launch_noise_update(const int* erow, const int* col, const double* val, long long nnz,
                         const void* U, const void* V, bool f32, int K, int stride, double mean,
                         double var_total, double alpha_max, double* partials, int nblocks,
                         Ctl* ctl, unsigned long long seed, cudaStream_t s) {
  if (f32)
    k_noise_sse<float><<<nblocks, kEvalThreads, 0, s>>>(erow, col, val, nnz, (const float*)U,
                                                        (const float*)V, K, stride, mean,
                                                        partials);
  else
    k_noise_sse<double><<<nblocks, kEvalThreads, 0, s>>>(erow, col, val, nnz, (const double*)U,
                                                         (const double*)V, K, stride, mean,
                                                         partials);
  MG_CUDA(cudaGetLastError());
  k_noise_draw<<<1, 32, 0, s>>>(partials, nblocks, nnz, var_total, alpha_max, ctl, seed);
  MG_CUDA(cudaGetLastError());
}

void launch_set_sweep(Ctl* ctl, uint32_t sweep, int burnin, cudaStream_t s) {
  k_set_sweep<<<1, 1, 0, s>>>(ctl, sweep, burnin);
  MG_CUDA(cudaGetLastError());
}

void launch_advance(Ctl* ctl, cudaStream_t s) {
  k_advance<<<1, 1, 0, s>>>(ctl);
  MG_CUDA(cudaGetLastError());
}

}  // namespace mg
