// Many independent BPMF chains in one set of launches (the batched multi-problem workload): P
// problems, each a MacauX<MatrixData, FixedGaussianNoise> with two BPMF priors (macau.cpp:110-147,
// latentprior.cpp:69-99) and its own size, latent dimension K_p <= 32, data mean and seed, are
// laid out block-diagonally so that each sweep runs
//   * per mode, one persistent tensor-core Gram launch over the rows of every problem
//     (k_gram_tc: a row's Gram only involves its own entries), then k_finish_batch, which
//     finishes each row with its problem's Lambda, mu, K and draws;
//   * per mode, one statistics block and one Normal-Wishart block per problem;
//   * optionally, the test-set evaluation of every problem,
// all captured in one CUDA graph.  A problem's rows keep their local index for the keyed draws,
// so its chain draws exactly what a single-problem context with its seed would draw.
//
// Layout: global row r of mode 0 is local row r - row0[p] of problem p (likewise columns for
// mode 1); latents are N x 32 FP32 (zero beyond K_p) plus the BF16 gather copy with its zero
// row; Lambda_p is K_p x K_p at Lambda + 1024 p, mu_p at mu + 32 p.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <memory>
#include <string>
#include <vector>

#include "common.cuh"
#include "host_util.h"
#include "kernels.h"
#include "rng.cuh"
#include "tune.h"
#include "warp_finish.cuh"

namespace mg {
namespace {

constexpr int kRec = 32 * 32 + 32;  // Gram record of k_gram_tc: 32 x 32 Gram, then the rhs
constexpr int kBLc = 36;            // leading dimension of the finish's L^T
constexpr int kFinBatchWarps = 4;

struct BatchRows {
  int nrows;
  const int* prob;     // problem of each row
  const int* row0;     // first row of each problem (P + 1 entries)
  const int* K;        // latent dimension of each problem
  const unsigned long long* seed;
  const double* Lambda;  // 1024 doubles per problem (K_p x K_p used; the FP64 retry)
  const float* LamF;     // 1024 floats per problem: Lambda in FP32, 32 x 32, zero beyond K_p
  const double* lmu;     // 32 per problem: Lambda mu
  float alpha;
  float* out_f32;
  __nv_bfloat16* out_bf16;
  Ctl* ctl;
  int mode;
};

// out[e] = {idx[e], float bits of (val[e] - mean of the entry's problem) * alpha}
__global__ void k_pack_batch(const int* __restrict__ idx, const double* __restrict__ val,
                             long long n, const int* __restrict__ prob_of_idx,
                             const double* __restrict__ mean, double alpha,
                             uint2* __restrict__ out) {
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < n;
       e += (long long)gridDim.x * blockDim.x) {
    const int c = idx[e];
    out[e] = make_uint2((unsigned)c,
                        __float_as_uint((float)((val[e] - mean[prob_of_idx[c]]) * alpha)));
  }
}

// FP64 redo of a row whose FP32 factorisation failed (the single-problem mixed path's retry).
__device__ __noinline__ bool batch_row_f64(const float* gp, const double* Lam, int K, double alpha,
                                           double rhs, double z, int lane, double* Lc,
                                           double* x_out) {
  double a[32], d0 = 1.0, rinv = 1.0;
#pragma unroll
  for (int j = 0; j < 32; j++) {
    const double v = (lane < K && j < K) ? Lam[lane + j * K] + alpha * (double)gp[lane * 32 + j]
                                         : (lane == j ? 1.0 : 0.0);
    a[j] = v;
    if (j == lane) d0 = v;
  }
  if (!warp_factor<double, 32>(a, rinv, lane, 0.0, d0, Lc, kBLc)) return false;
  *x_out = warp_solve<double, 32>(a, rinv, rhs, lane, Lc, kBLc, z);
  return true;
}

// FP32 finish of one row at width KP >= K (lane i: row i of MM = Lambda_p + alpha G, identity
// beyond K).  Returns false when the FP32 pivot fails.
template <int KP>
__device__ __forceinline__ bool batch_row_f32(const float* __restrict__ lf,
                                              const float* __restrict__ gp, int K, float alpha,
                                              double rhs, double z, int lane, float* Lc,
                                              double* x) {
  float a[KP], d0 = 1.f, rinv = 1.f;
#pragma unroll
  for (int q = 0; q < KP / 4; q++) {
    const float4 m4 = lane < KP ? __ldg(reinterpret_cast<const float4*>(lf) + q)
                                : make_float4(0.f, 0.f, 0.f, 0.f);
    const float4 v4 = lane < KP ? __ldcg(reinterpret_cast<const float4*>(gp) + q)
                                : make_float4(0.f, 0.f, 0.f, 0.f);
    const float mm[4] = {m4.x, m4.y, m4.z, m4.w}, gg[4] = {v4.x, v4.y, v4.z, v4.w};
#pragma unroll
    for (int u = 0; u < 4; u++) {
      const int j = 4 * q + u;
      const float v = (lane < K && j < K) ? mm[u] + alpha * gg[u] : (lane == j ? 1.f : 0.f);
      a[j] = v;
      if (j == lane) d0 = v;
    }
  }
  if (!warp_factor<float, KP>(a, rinv, lane, 0x1p-20, d0, Lc, kBLc)) return false;
  *x = (double)warp_solve<float, KP>(a, rinv, (float)rhs, lane, Lc, kBLc, z);
  return true;
}

// One warp per row: MM = Lambda_p + alpha G in FP32 at the smallest width 8, 16 or 32 that holds
// K_p, rhs = record rhs (alpha baked into the weights) + Lambda_p mu_p, Cholesky and solves
// with the row's keyed draws, FP64 retry on a failed pivot (sample_latent_blas,
// latentprior.cpp:361-385).
__global__ void __launch_bounds__(kFinBatchWarps * 32, 4)
    k_finish_batch(const BatchRows b, const float* __restrict__ gram) {
  __shared__ __align__(16) double Lc_s[kFinBatchWarps][32 * kBLc];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const uint32_t sweep = b.ctl->sweep;
  const int nw = gridDim.x * kFinBatchWarps;
  for (int row = blockIdx.x * kFinBatchWarps + warp; row < b.nrows; row += nw) {
    const int p = b.prob[row], K = b.K[p], lr = row - b.row0[p];
    const float* lf = b.LamF + (size_t)p * 1024 + lane * 32;
    const float* gp = gram + (size_t)row * kRec;
    // the record holds the first 8, 16 or 32 rows and columns (k_gram_tc's row_width)
    const double rhs = lane < K ? (double)__ldcg(gp + 32 * 32 + lane) + b.lmu[(size_t)p * 32 + lane]
                                : 0.0;
    double z0, z1;
    normal_pair(b.seed[p], sweep, stream_id(kRowNoise, (uint32_t)b.mode), (uint32_t)lr,
                (uint32_t)(lane >> 1), &z0, &z1);
    const double z = lane < K ? ((lane & 1) ? z1 : z0) : 0.0;
    float* Lcf = reinterpret_cast<float*>(Lc_s[warp]);
    double x = 0.0;
    bool ok;
    if (K <= 8) ok = batch_row_f32<8>(lf, gp + lane * 32, K, b.alpha, rhs, z, lane, Lcf, &x);
    else if (K <= 16) ok = batch_row_f32<16>(lf, gp + lane * 32, K, b.alpha, rhs, z, lane, Lcf, &x);
    else ok = batch_row_f32<32>(lf, gp + lane * 32, K, b.alpha, rhs, z, lane, Lcf, &x);
    if (!ok) {
      if (lane == 0) atomicAdd(&b.ctl->retries[b.mode], 1u);
      __syncwarp();
      const double* Lam = b.Lambda + (size_t)p * 1024;
      if (!batch_row_f64(gp, Lam, K, (double)b.alpha, rhs, z, lane, Lc_s[warp], &x)) {
        if (lane == 0) {
          atomicOr(&b.ctl->status, kStatCholFail);
          atomicCAS(&b.ctl->bad_row, -1, row);
        }
        __syncwarp();
        continue;
      }
    }
    if (lane < K) {
      b.out_f32[(size_t)row * 32 + lane] = (float)x;
      b.out_bf16[(size_t)row * 32 + lane] = __float2bfloat16_rn((float)x);
    }
    __syncwarp();
  }
}

// Test predictions of every problem (eval_rmse, bpmfutils.h:86-114): the online posterior
// mean and variance per entry, and each entry's squared errors for the per-problem sums.
__global__ void k_eval_batch(const int* __restrict__ trow, const int* __restrict__ tcol,
                             const double* __restrict__ tval, const int* __restrict__ tprob,
                             long long ntest, const float* __restrict__ U,
                             const float* __restrict__ V, const double* __restrict__ mean,
                             const Ctl* ctl, double* __restrict__ pred, double* __restrict__ pvar,
                             double* __restrict__ se1, double* __restrict__ sea) {
  const int n = ((int)ctl->sweep < ctl->burnin) ? 0 : (int)ctl->sweep - ctl->burnin;
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < ntest;
       t += (long long)gridDim.x * blockDim.x) {
    const float4* u = reinterpret_cast<const float4*>(U + (size_t)trow[t] * 32);
    const float4* v = reinterpret_cast<const float4*>(V + (size_t)tcol[t] * 32);
    double dot = 0.0;
#pragma unroll
    for (int q = 0; q < 8; q++) {
      const float4 a = u[q], c = v[q];
      dot += (double)a.x * c.x + (double)a.y * c.y + (double)a.z * c.z + (double)a.w * c.w;
    }
    const double pr = dot + mean[tprob[t]];
    const double y = tval[t];
    double pavg;
    if (n == 0) {
      pavg = pr;
    } else {
      const double delta = pr - pred[t];
      pavg = pred[t] + delta / (n + 1);
      pvar[t] += delta * (pr - pavg);
    }
    pred[t] = pavg;
    se1[t] = (y - pr) * (y - pr);
    sea[t] = (y - pavg) * (y - pavg);
  }
}

// One warp per problem: RMSEs over its test segment (lane-strided sums, fixed xor tree);
// rmse[2 p] = posterior mean, rmse[2 p + 1] = single sample (NaN without test entries).
__global__ void k_rmse_batch(const long long* __restrict__ toff, int P,
                             const double* __restrict__ se1, const double* __restrict__ sea,
                             double* __restrict__ rmse) {
  const int lane = threadIdx.x & 31;
  for (int p = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; p < P;
       p += (gridDim.x * blockDim.x) >> 5) {
    double a = 0.0, b1 = 0.0;
    for (long long t = toff[p] + lane; t < toff[p + 1]; t += 32) {
      a += sea[t];
      b1 += se1[t];
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      a += __shfl_xor_sync(0xffffffffu, a, o);
      b1 += __shfl_xor_sync(0xffffffffu, b1, o);
    }
    if (lane == 0) {
      const double cnt = (double)(toff[p + 1] - toff[p]);
      rmse[2 * p] = cnt > 0 ? sqrt(a / cnt) : NAN;
      rmse[2 * p + 1] = cnt > 0 ? sqrt(b1 / cnt) : NAN;
    }
  }
}

int blocks_for(long long n, int threads) {
  long long b = (n + threads - 1) / threads;
  if (b > 4736) b = 4736;
  return (int)(b < 1 ? 1 : b);
}

}  // namespace

// ------------------------------------------------------------------------------------------
class Batch {
 public:
  Batch(int P, const int32_t* nrows, const int32_t* ncols, const int32_t* K,
        const uint64_t* seeds, double alpha, int device)
      : P_(P), alpha_(alpha), dev_(device) {
    if (P < 1) throw MgError(MG_ERR_ARG, "need at least one problem");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
      throw MgError(MG_ERR_NOGPU, "no CUDA device");
    MG_CUDA(cudaSetDevice(dev_));
    cudaDeviceProp prop;
    MG_CUDA(cudaGetDeviceProperties(&prop, dev_));
    if (prop.major < 10)
      throw MgError(MG_ERR_NOGPU, std::string("sm_100a device required, found ") + prop.name);
    num_sms_ = prop.multiProcessorCount;
    dims_[0].assign(nrows, nrows + P);
    dims_[1].assign(ncols, ncols + P);
    K_.assign(K, K + P);
    seeds_.assign(seeds, seeds + P);
    for (int p = 0; p < P; p++) {
      if (K_[p] < 1 || K_[p] > 32) throw MgError(MG_ERR_ARG, "num_latent must be in [1, 32]");
      if (dims_[0][p] < 1 || dims_[1][p] < 1) throw MgError(MG_ERR_ARG, "empty problem");
    }
    for (int m = 0; m < 2; m++) {
      off_[m].assign(P + 1, 0);
      for (int p = 0; p < P; p++) off_[m][p + 1] = off_[m][p] + dims_[m][p];
      N_[m] = off_[m][P];
    }
    MG_CUDA(cudaStreamCreateWithFlags(&s_, cudaStreamNonBlocking));
    MG_CUDA(cudaEventCreate(&ev0_));
    MG_CUDA(cudaEventCreate(&ev1_));
    ctl_.alloc_zero(1, s_);
    std::vector<unsigned long long> sd(seeds_.begin(), seeds_.end());
    seed_d_.upload(sd.data(), sd.size(), s_);
    K_d_.upload(K_.data(), K_.size(), s_);
    for (int m = 0; m < 2; m++) {
      std::vector<int> o(off_[m].begin(), off_[m].end());
      row0_d_[m].upload(o.data(), o.size(), s_);
      std::vector<int> pr(N_[m]);
      for (int p = 0; p < P; p++)
        for (long long r = off_[m][p]; r < off_[m][p + 1]; r++) pr[r] = p;
      prob_d_[m].upload(pr.data(), pr.size(), s_);
      std::vector<int> wd(N_[m]);  // Gram record width of each row: 8, 16 or 32 >= K_p
      for (long long r = 0; r < N_[m]; r++) {
        const int k = K_[pr[r]];
        wd[r] = k <= 8 ? 8 : (k <= 16 ? 16 : 32);
      }
      width_d_[m].upload(wd.data(), wd.size(), s_);
    }
    MG_CUDA(cudaStreamSynchronize(s_));
  }

  ~Batch() {
    if (graph_) cudaGraphExecDestroy(graph_);
    if (graph_eval_) cudaGraphExecDestroy(graph_eval_);
    if (ev0_) cudaEventDestroy(ev0_);
    if (ev1_) cudaEventDestroy(ev1_);
    if (s_) cudaStreamDestroy(s_);
  }

  // Problem p's train entries are rows / cols / vals[toff[p] .. toff[p+1]) in its own indices;
  // likewise its test entries.  Duplicates are summed.
  void set_data(const int64_t* toff, const int32_t* rows, const int32_t* cols, const double* vals,
                const int64_t* eoff, const int32_t* trows, const int32_t* tcols,
                const double* tvals) {
    const long long nnz = toff[P_];
    if (nnz < 1) throw MgError(MG_ERR_ARG, "training data is empty");
    std::vector<int> gr(nnz), gc(nnz);
    for (int p = 0; p < P_; p++)
      for (long long e = toff[p]; e < toff[p + 1]; e++) {
        if (rows[e] < 0 || rows[e] >= dims_[0][p] || cols[e] < 0 || cols[e] >= dims_[1][p])
          throw MgError(MG_ERR_ARG, "training index out of range");
        gr[e] = rows[e] + (int)off_[0][p];
        gc[e] = cols[e] + (int)off_[1][p];
      }
    DBuf<int> dr, dc;
    DBuf<double> dv;
    dr.upload(gr.data(), nnz, s_);
    dc.upload(gc.data(), nnz, s_);
    dv.upload(vals, nnz, s_);
    for (int m = 0; m < 2; m++) {
      md_[m].ptr.alloc((size_t)N_[m] + 1);
      md_[m].idx.alloc((size_t)nnz);
      md_[m].val.alloc((size_t)nnz);
    }
    const long long nu = build_csr_pair(dr.p, dc.p, dv.p, nnz, N_[0], N_[1], md_[0].ptr.p,
                                        md_[0].idx.p, md_[0].val.p, md_[1].ptr.p, md_[1].idx.p,
                                        md_[1].val.p, s_);
    // each problem's mean over its column-major storage (sparsetensor.cpp:82)
    std::vector<double> cval((size_t)nu);
    std::vector<long long> p0((size_t)N_[0] + 1), p1((size_t)N_[1] + 1);
    MG_CUDA(cudaMemcpyAsync(cval.data(), md_[1].val.p, sizeof(double) * nu,
                            cudaMemcpyDeviceToHost, s_));
    MG_CUDA(cudaMemcpyAsync(p0.data(), md_[0].ptr.p, sizeof(long long) * p0.size(),
                            cudaMemcpyDeviceToHost, s_));
    MG_CUDA(cudaMemcpyAsync(p1.data(), md_[1].ptr.p, sizeof(long long) * p1.size(),
                            cudaMemcpyDeviceToHost, s_));
    MG_CUDA(cudaStreamSynchronize(s_));
    mean_.assign(P_, 0.0);
    for (int p = 0; p < P_; p++) {
      const long long b = p1[off_[1][p]], e = p1[off_[1][p + 1]];
      if (e == b) throw MgError(MG_ERR_ARG, "a problem has no training entries");
      double sum = 0.0;
      for (long long q = b; q < e; q++) sum += cval[q];
      mean_[p] = sum / (double)(e - b);
    }
    mean_d_.upload(mean_.data(), P_, s_);
    build_mode(0, p0, nu);
    build_mode(1, p1, nu);
    // test entries, global indices, in problem order
    const long long nt = eoff[P_];
    std::vector<int> tr(nt), tc(nt), tp(nt);
    for (int p = 0; p < P_; p++)
      for (long long e = eoff[p]; e < eoff[p + 1]; e++) {
        if (trows[e] < 0 || trows[e] >= dims_[0][p] || tcols[e] < 0 || tcols[e] >= dims_[1][p])
          throw MgError(MG_ERR_ARG, "test index out of range");
        tr[e] = trows[e] + (int)off_[0][p];
        tc[e] = tcols[e] + (int)off_[1][p];
        tp[e] = p;
      }
    ntest_ = nt;
    trow_.upload(tr.data(), nt, s_);
    tcol_.upload(tc.data(), nt, s_);
    tprob_.upload(tp.data(), nt, s_);
    tval_.upload(tvals, nt, s_);
    std::vector<long long> eo(eoff, eoff + P_ + 1);
    toff_.upload(eo.data(), eo.size(), s_);
    pred_.alloc_zero(std::max(1LL, nt), s_);
    pvar_.alloc_zero(std::max(1LL, nt), s_);
    se1_.alloc(std::max(1LL, nt));
    sea_.alloc(std::max(1LL, nt));
    rmse_.alloc(2 * (size_t)P_);
    MG_CUDA(cudaStreamSynchronize(s_));
    have_data_ = true;
    initialised_ = false;
  }

  // MacauX::init + BPMFPrior::init per problem: latents zero, mu = 0, Lambda = 10 I.
  void init(int burnin) {
    if (!have_data_) throw MgError(MG_ERR_STATE, "no training data");
    burnin_ = burnin;
    for (int m = 0; m < 2; m++) {
      lat32_[m].alloc_zero((size_t)N_[m] * 32, s_);
      lat16_[m].alloc_zero((size_t)(N_[m] + 1) * 32, s_);
      std::vector<double> mu((size_t)P_ * 32, 0.0), lam((size_t)P_ * 1024, 0.0);
      for (int p = 0; p < P_; p++)
        for (int i = 0; i < K_[p]; i++) lam[(size_t)p * 1024 + i + (size_t)i * K_[p]] = 10.0;
      mu_[m].upload(mu.data(), mu.size(), s_);
      Lambda_[m].upload(lam.data(), lam.size(), s_);
      std::vector<float> lf((size_t)P_ * 1024, 0.f);
      for (int p = 0; p < P_; p++)
        for (int i = 0; i < K_[p]; i++) lf[(size_t)p * 1024 + i * 32 + i] = 10.f;
      LamF_[m].upload(lf.data(), lf.size(), s_);
      lmu_[m].alloc_zero((size_t)P_ * 32, s_);
    }
    partials_.alloc((size_t)P_ * kRec);
    if (ntest_ > 0) {
      MG_CUDA(cudaMemsetAsync(pred_.p, 0, ntest_ * sizeof(double), s_));
      MG_CUDA(cudaMemsetAsync(pvar_.p, 0, ntest_ * sizeof(double), s_));
    }
    Ctl zero{};
    zero.bad_row = -1;
    MG_CUDA(cudaMemcpyAsync(ctl_.p, &zero, sizeof(Ctl), cudaMemcpyHostToDevice, s_));
    MG_CUDA(cudaStreamSynchronize(s_));
    drop_graphs();
    initialised_ = true;
  }

  void sweeps(int first_iter, int count, bool eval, bool sync = true) {
    if (!initialised_) throw MgError(MG_ERR_STATE, "call mg_batch_init first");
    launch_set_sweep(ctl_.p, (uint32_t)first_iter, burnin_, s_);
    cudaGraphExec_t& ge = eval ? graph_eval_ : graph_;
    if (!ge && count > 0) {
      sweep_body(eval);  // eager first sweep: one-time attribute set-up outside the capture
      count--;
      cudaGraph_t g = nullptr;
      MG_CUDA(cudaStreamBeginCapture(s_, cudaStreamCaptureModeThreadLocal));
      try {
        sweep_body(eval);
      } catch (...) {
        cudaStreamEndCapture(s_, &g);
        if (g) cudaGraphDestroy(g);
        throw;
      }
      MG_CUDA(cudaStreamEndCapture(s_, &g));
      MG_CUDA(cudaGraphInstantiate(&ge, g, 0));
      cudaGraphDestroy(g);
    }
    for (int i = 0; i < count; i++) MG_CUDA(cudaGraphLaunch(ge, s_));
    if (sync) check_status();
  }

  double time_sweeps(int first_iter, int count) {
    if (!initialised_) throw MgError(MG_ERR_STATE, "call mg_batch_init first");
    if (count < 1) return 0.0;
    if (!graph_) {
      sweeps(first_iter, 1, false, true);
      first_iter++;
      count--;
    }
    MG_CUDA(cudaStreamSynchronize(s_));
    MG_CUDA(cudaEventRecord(ev0_, s_));
    sweeps(first_iter, count, false, false);
    MG_CUDA(cudaEventRecord(ev1_, s_));
    MG_CUDA(cudaEventSynchronize(ev1_));
    float ms = 0.f;
    MG_CUDA(cudaEventElapsedTime(&ms, ev0_, ev1_));
    check_status();
    return ms * 1e-3;
  }

  void get_latents(int p, int mode, double* out) {
    if (p < 0 || p >= P_ || mode < 0 || mode > 1) throw MgError(MG_ERR_ARG, "bad problem / mode");
    if (!initialised_) throw MgError(MG_ERR_STATE, "call mg_batch_init first");
    const long long n = dims_[mode][p];
    std::vector<float> h((size_t)n * 32);
    MG_CUDA(cudaMemcpyAsync(h.data(), lat32_[mode].p + (size_t)off_[mode][p] * 32,
                            h.size() * 4, cudaMemcpyDeviceToHost, s_));
    MG_CUDA(cudaStreamSynchronize(s_));
    for (long long r = 0; r < n; r++)
      for (int k = 0; k < K_[p]; k++) out[r * K_[p] + k] = h[(size_t)r * 32 + k];
  }

  void get_rmse(double* out) {
    if (ntest_ == 0) {
      for (int q = 0; q < 2 * P_; q++) out[q] = NAN;
      return;
    }
    MG_CUDA(cudaMemcpyAsync(out, rmse_.p, sizeof(double) * 2 * P_, cudaMemcpyDeviceToHost, s_));
    MG_CUDA(cudaStreamSynchronize(s_));
  }

  void check_status() {
    Ctl h;
    MG_CUDA(cudaMemcpyAsync(&h, ctl_.p, sizeof(Ctl), cudaMemcpyDeviceToHost, s_));
    MG_CUDA(cudaStreamSynchronize(s_));
    retries_[0] = h.retries[0];
    retries_[1] = h.retries[1];
    if (h.status & kStatTimeout) throw MgError(MG_ERR_TIMEOUT, "device wait timed out");
    if (h.status & kStatCholFail) throw MgError(MG_ERR_CHOL, "Cholesky Decomposition failed!");
    if (h.status & kStatHyperFail)
      throw MgError(MG_ERR_CHOL, "Cholesky Decomposition failed! (hyperprior)");
  }

  long long retries(int m) const { return retries_[m]; }
  long long nnz() const { return md_[0].nnz; }
  long long rows(int m) const { return N_[m]; }

  std::string err;

 private:
  struct Mode {
    long long nnz = 0;
    DBuf<long long> ptr, pptr;
    DBuf<int> idx;
    DBuf<double> val;
    DBuf<uint2> packed, packed_tc;
    DBuf<RowTask> tasks;
    DBuf<int4> split;
    DBuf<float> gram;
    int ntasks = 0, nsplit = 0, nslots = 0;
    // host copy of the padded row pointers, the split threshold of the task list, the row
    // finish's CTAs per SM, and the autotuner's record
    std::vector<long long> hpptr;
    long long thr = 0;
    int fin_per_sm = 8;
    TuneChoice tune;
    int tune_state = 0;
  };

  // Split threshold nnz / (div * 16 * SMs), clamped to [256, 16384] and rounded up to 16
  // entries; div = 2 is the default, the autotuner tries 1 to 16.
  long long split_divisor_thr(int m, int div) const {
    long long thr = md_[m].nnz / ((long long)div * num_sms_ * 16);
    thr = std::max(256LL, std::min(16384LL, thr));
    return (thr + 15) / 16 * 16;
  }

  // Task list of mode m over the padded rows at split threshold thr (16-entry aligned parts),
  // its split-row table and the split-part scratch.
  void build_tasks(int m, long long thr) {
    Mode& md = md_[m];
    md.thr = thr;
    int ns = 0, nsl = 0;
    std::vector<RowTask> tt = make_tasks(md.hpptr, thr, 16, ns, nsl);
    md.ntasks = (int)tt.size();
    md.nsplit = ns;
    md.nslots = nsl;
    md.tasks.upload(tt.data(), tt.size(), s_);
    std::vector<int4> sr;
    for (const RowTask& t : tt)
      if (t.nparts > 1 && t.part == 0) sr.push_back(make_int4(t.row, t.nparts, t.slot, 0));
    std::sort(sr.begin(), sr.end(), [](const int4& a, const int4& b) { return a.x < b.x; });
    md.split.upload(sr.data(), sr.size(), s_);
    const size_t need = (size_t)std::max(md_[0].nslots, md_[1].nslots) * kRec;
    if (need > scratch_.n) scratch_.alloc(need);
  }

  void build_mode(int m, const std::vector<long long>& hptr, long long nnz) {
    Mode& md = md_[m];
    md.nnz = nnz;
    const long long N = N_[m];
    md.packed.alloc((size_t)std::max(1LL, nnz));
    k_pack_batch<<<blocks_for(nnz, 256), 256, 0, s_>>>(md.idx.p, md.val.p, nnz,
                                                         prob_d_[1 - m].p, mean_d_.p, alpha_,
                                                         md.packed.p);
    MG_CUDA(cudaGetLastError());
    std::vector<long long> pptr(N + 1, 0);
    for (long long r = 0; r < N; r++) pptr[r + 1] = pptr[r] + (hptr[r + 1] - hptr[r] + 15) / 16 * 16;
    md.pptr.upload(pptr.data(), pptr.size(), s_);
    md.packed_tc.alloc((size_t)std::max(1LL, pptr[N]));
    launch_pad(md.ptr.p, md.pptr.p, N, md.packed.p, (unsigned)N_[1 - m], md.packed_tc.p, s_);
    md.hpptr = pptr;
    md.fin_per_sm = 8;
    md.tune_state = 0;
    build_tasks(m, split_divisor_thr(m, 2));
    md.gram.alloc((size_t)std::max(1LL, N) * kRec);
    MG_CUDA(cudaStreamSynchronize(s_));
  }

  void drop_graphs() {
    for (cudaGraphExec_t* g : {&graph_, &graph_eval_})
      if (*g) {
        cudaGraphExecDestroy(*g);
        *g = nullptr;
      }
  }

  void sample(int m) {
    Mode& md = md_[m];
    SampleParams sp{};
    sp.tasks = md.tasks.p;
    sp.ntasks = md.ntasks;
    sp.nrows = (int)N_[m];
    sp.nother = (int)N_[1 - m];
    sp.K = 32;
    sp.packed = md.packed_tc.p;
    sp.alpha = 1.0;
    sp.other = lat16_[1 - m].p;
    sp.out_f32 = lat32_[m].p;
    sp.out_bf16 = lat16_[m].p;
    sp.scratch = scratch_.p;
    sp.ctl = ctl_.p;
    sp.qslot = m;
    sp.mode = m;
    sp.row_width = width_d_[m].p;
    launch_gram_tc(sp, md.gram.p, md.split.p, md.nsplit, 32, s_, num_sms_);
    BatchRows b{(int)N_[m], prob_d_[m].p, row0_d_[m].p, K_d_.p, seed_d_.p, Lambda_[m].p,
                LamF_[m].p, lmu_[m].p, (float)alpha_, lat32_[m].p, lat16_[m].p, ctl_.p, m};
    k_finish_batch<<<num_sms_ * md.fin_per_sm, kFinBatchWarps * 32, 0, s_>>>(b, md.gram.p);
    MG_CUDA(cudaGetLastError());
  }

 public:
  // Autotuner of the batched sampler (tune.h): per mode, the split threshold of the task list
  // (divisors 1, 2, 4, 8, 16) and the row finish's CTAs per SM (8, 4, 16), each timed as one
  // warm-up and three timed Gram + finish launches on the current state; the fastest is kept.
  // Latents and the control block are restored afterwards.
  void autotune(bool use_cache) {
    if (!initialised_) throw MgError(MG_ERR_STATE, "call mg_batch_init before autotuning");
    drop_graphs();
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    try {
      DeviceBackup ctl_backup(s_);
      ctl_backup.save(ctl_.p, sizeof(Ctl));
      MG_CUDA(cudaEventCreate(&e0));
      MG_CUDA(cudaEventCreate(&e1));
      for (int m = 0; m < 2; m++) {
        Mode& md = md_[m];
        const std::string key = tune_key("batch", 32, num_sms_, md.hpptr) + ":k" + ks_digest();
        TuneChoice c;
        if (use_cache && TuneCache::get().find(key, &c)) {
          if (md.thr != c.thr || md.fin_per_sm != c.groups) {
            md.fin_per_sm = c.groups;
            build_tasks(m, c.thr);
          }
          md.tune = c;
          md.tune_state = 2;
          continue;
        }
        DeviceBackup lat_backup(s_);  // put back before the next mode, or when a run throws
        lat_backup.save(lat32_[m].p, lat32_[m].n * sizeof(float));
        lat_backup.save(lat16_[m].p, lat16_[m].n * sizeof(__nv_bfloat16));
        std::vector<long long> thrs;
        for (int div : {2, 1, 4, 8, 16}) {
          const long long t = split_divisor_thr(m, div);
          if (std::find(thrs.begin(), thrs.end(), t) == thrs.end()) thrs.push_back(t);
        }
        TuneChoice best;
        best.ms = 1e30;
        int tried = 0;
        for (int fin : {8, 4, 16})
          for (long long t : thrs) {
            md.fin_per_sm = fin;
            build_tasks(m, t);
            float best_ms = 1e30f;
            for (int rep = 0; rep < 4; rep++) {
              MG_CUDA(cudaMemsetAsync(&ctl_.p->queue[0], 0, 8 * sizeof(uint32_t), s_));
              MG_CUDA(cudaEventRecord(e0, s_));
              sample(m);
              MG_CUDA(cudaEventRecord(e1, s_));
              MG_CUDA(cudaEventSynchronize(e1));
              float ms = 0.f;
              MG_CUDA(cudaEventElapsedTime(&ms, e0, e1));
              if (rep > 0) best_ms = std::min(best_ms, ms);
            }
            check_status();
            tried++;
            if (tried == 1) best.ms_default = best_ms;
            if (best_ms < best.ms) {
              best.ms = best_ms;
              best.thr = t;
              best.groups = fin;
            }
          }
        best.candidates = tried;
        md.fin_per_sm = best.groups;
        build_tasks(m, best.thr);
        md.tune = best;
        md.tune_state = 1;
        TuneCache::get().put(key, best);
      }
    } catch (...) {
      if (e0) cudaEventDestroy(e0);
      if (e1) cudaEventDestroy(e1);
      throw;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    MG_CUDA(cudaStreamSynchronize(s_));
    drop_graphs();
  }

  // Problem count and an FNV-1a digest of the problems' K values (part of the tuning key).
  std::string ks_digest() const {
    unsigned long long h = 1469598103934665603ull;
    for (int k : K_) {
      h ^= (unsigned long long)k;
      h *= 1099511628211ull;
    }
    char buf[48];
    std::snprintf(buf, sizeof(buf), "%d:%016llx", P_, h);
    return buf;
  }

  void get_tuning(int m, mg_tuning* out) const {
    if (m < 0 || m > 1) throw MgError(MG_ERR_ARG, "mode must be 0 or 1");
    const Mode& md = md_[m];
    out->split_threshold = md.thr;
    out->cta_groups = 0;
    out->tensor_core = 1;
    out->state = md.tune_state;
    out->candidates = md.tune_state ? md.tune.candidates : 0;
    out->ms_best = md.tune_state ? md.tune.ms : 0.0;
    out->ms_default = md.tune_state ? md.tune.ms_default : 0.0;
    out->finish_ctas_per_sm = md.fin_per_sm;
  }

 private:

  void update_prior(int m) {  // per problem: statistics, then the Normal-Wishart draw
    launch_prior_batch(lat32_[m].p, row0_d_[m].p, K_d_.p, seed_d_.p, P_, partials_.p, ctl_.p,
                       m, mu_[m].p, Lambda_[m].p, LamF_[m].p, lmu_[m].p, s_);
  }

  void eval() {
    if (ntest_ == 0) return;
    k_eval_batch<<<blocks_for(ntest_, 256), 256, 0, s_>>>(trow_.p, tcol_.p, tval_.p, tprob_.p,
                                                           ntest_, lat32_[0].p, lat32_[1].p,
                                                           mean_d_.p, ctl_.p, pred_.p, pvar_.p,
                                                           se1_.p, sea_.p);
    MG_CUDA(cudaGetLastError());
    k_rmse_batch<<<(P_ + 7) / 8, 256, 0, s_>>>(toff_.p, P_, se1_.p, sea_.p, rmse_.p);
    MG_CUDA(cudaGetLastError());
  }

  // One sweep of every problem: sample mode 0, sample mode 1, both priors, eval, advance
  // (macau.cpp:110-147 per problem).
  void sweep_body(bool do_eval) {
    MG_CUDA(cudaMemsetAsync(&ctl_.p->queue[0], 0, 8 * sizeof(uint32_t), s_));
    sample(0);
    sample(1);
    update_prior(0);
    update_prior(1);
    if (do_eval) eval();
    launch_advance(ctl_.p, s_);
  }

  int P_;
  double alpha_;
  int dev_ = 0, num_sms_ = 148;
  cudaStream_t s_ = nullptr;
  cudaEvent_t ev0_ = nullptr, ev1_ = nullptr;
  std::vector<int> dims_[2], K_;
  std::vector<uint64_t> seeds_;
  std::vector<long long> off_[2];
  long long N_[2] = {0, 0};
  std::vector<double> mean_;
  Mode md_[2];
  DBuf<Ctl> ctl_;
  DBuf<unsigned long long> seed_d_;
  DBuf<int> K_d_, row0_d_[2], prob_d_[2], width_d_[2];
  DBuf<double> mean_d_, mu_[2], Lambda_[2], partials_, scratch_;
  DBuf<float> lat32_[2], LamF_[2];
  DBuf<double> lmu_[2];
  DBuf<__nv_bfloat16> lat16_[2];
  DBuf<int> trow_, tcol_, tprob_;
  DBuf<long long> toff_;
  DBuf<double> tval_, pred_, pvar_, se1_, sea_, rmse_;
  long long ntest_ = 0;
  int burnin_ = 0;
  bool have_data_ = false, initialised_ = false;
  cudaGraphExec_t graph_ = nullptr, graph_eval_ = nullptr;
  long long retries_[2] = {0, 0};
};

}  // namespace mg

// ============================== C ABI ==============================
struct mg_batch {
  std::unique_ptr<mg::Batch> b;
  std::string err;
};

namespace {
thread_local std::string g_batch_create_error;

template <typename F>
int bguarded(mg_batch* h, F&& f) {
  if (!h || !h->b) return MG_ERR_ARG;
  try {
    f(*h->b);
    h->err.clear();
    return MG_OK;
  } catch (const mg::MgError& e) {
    h->err = e.what();
    return e.code;
  } catch (const mg::CudaError& e) {
    h->err = e.what();
    return MG_ERR_CUDA;
  } catch (const std::exception& e) {
    h->err = e.what();
    return MG_ERR_ARG;
  }
}
}  // namespace

extern "C" {

int mg_batch_create(mg_batch** out, int nprob, const int32_t* nrows, const int32_t* ncols,
                    const int32_t* num_latent, const uint64_t* seeds, double precision,
                    int device) {
  if (!out || !nrows || !ncols || !num_latent || !seeds) return MG_ERR_ARG;
  *out = nullptr;
  try {
    auto h = std::make_unique<mg_batch>();
    h->b = std::make_unique<mg::Batch>(nprob, nrows, ncols, num_latent, seeds, precision, device);
    *out = h.release();
    return MG_OK;
  } catch (const mg::MgError& e) {
    g_batch_create_error = e.what();
    return e.code;
  } catch (const std::exception& e) {
    g_batch_create_error = e.what();
    return MG_ERR_CUDA;
  }
}

void mg_batch_destroy(mg_batch* h) { delete h; }

const char* mg_batch_last_error(const mg_batch* h) {
  return h ? h->err.c_str() : g_batch_create_error.c_str();
}

int mg_batch_set_data(mg_batch* h, const int64_t* train_off, const int32_t* rows,
                      const int32_t* cols, const double* vals, const int64_t* test_off,
                      const int32_t* trows, const int32_t* tcols, const double* tvals) {
  if (!train_off || !rows || !cols || !vals || !test_off) return MG_ERR_ARG;
  return bguarded(h, [&](mg::Batch& b) {
    b.set_data(train_off, rows, cols, vals, test_off, trows, tcols, tvals);
  });
}

int mg_batch_init(mg_batch* h, int burnin) {
  return bguarded(h, [&](mg::Batch& b) { b.init(burnin); });
}

int mg_batch_sweeps(mg_batch* h, int first_iter, int count, int eval) {
  if (count < 0) return MG_ERR_ARG;
  return bguarded(h, [&](mg::Batch& b) { b.sweeps(first_iter, count, eval != 0, true); });
}

int mg_batch_time_sweeps(mg_batch* h, int first_iter, int count, double* seconds) {
  if (!seconds || count < 0) return MG_ERR_ARG;
  return bguarded(h, [&](mg::Batch& b) { *seconds = b.time_sweeps(first_iter, count); });
}

int mg_batch_get_latents(mg_batch* h, int prob, int mode, double* out) {
  if (!out) return MG_ERR_ARG;
  return bguarded(h, [&](mg::Batch& b) { b.get_latents(prob, mode, out); });
}

int mg_batch_get_rmse(mg_batch* h, double* out) {
  if (!out) return MG_ERR_ARG;
  return bguarded(h, [&](mg::Batch& b) { b.get_rmse(out); });
}

int mg_batch_autotune(mg_batch* h, int use_cache) {
  return bguarded(h, [&](mg::Batch& b) { b.autotune(use_cache != 0); });
}

int mg_batch_get_tuning(mg_batch* h, int mode, mg_tuning* out) {
  if (!out) return MG_ERR_ARG;
  return bguarded(h, [&](mg::Batch& b) { b.get_tuning(mode, out); });
}

int mg_batch_get_info(mg_batch* h, int64_t* out) {
  if (!out) return MG_ERR_ARG;
  return bguarded(h, [&](mg::Batch& b) {
    out[0] = b.rows(0);
    out[1] = b.rows(1);
    out[2] = b.nnz();
    out[3] = b.retries(0);
    out[4] = b.retries(1);
  });
}

}  // extern "C"
