// Shared definitions of the sm_100a Gibbs-sweep library: status codes, the device control block,
// row-task descriptors and small device helpers.
#pragma once
#include <cuda_runtime.h>
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include <cstdint>
#include <cstdio>
#include <stdexcept>
#include <string>

#include "../../include/macau_b200.h"

namespace mg {

// Device control block: one per context, read by every kernel of a sweep so a captured CUDA
// graph can be replayed with a new sweep index.
struct Ctl {
  uint32_t sweep;         // Gibbs iteration index (RNG counter word 3)
  int32_t burnin;         // eval: n = sweep < burnin ? 0 : sweep - burnin
  int32_t status;         // OR of MG_STATUS_* bits raised by kernels
  int32_t bad_row;        // first row whose factorisation failed (diagnostics)
  uint32_t queue[8];      // work-queue heads of persistent kernels ([mode]: the row sampler of
                          // that mode), reset before each sampling launch
  uint32_t retries[2];    // mixed mode: rows re-factorised in FP64, per mode
  uint32_t cg_iters[2];   // last block-CG iteration count, per mode
  uint32_t cg_done;       // block-CG convergence flag
  uint32_t pad[3];
  double alpha;           // current noise precision (AdaptiveGaussianNoise::alpha); with fixed
                          // noise it holds the fixed precision and the samplers ignore it
};

// Status bits raised on the device (the host maps them to MG_ERR_* codes and messages).
enum : int32_t {
  kStatCholFail = 1,    // a row's Lambda + alpha*V'V was not positive definite in FP64
  kStatHyperFail = 2,   // hyperprior factorisation failed
  kStatCgFail = 4,      // block-CG breakdown / iteration cap
  kStatTimeout = 8,     // a bounded wait gave up
};

// One unit of latent-sampler work: a whole row, or one part of a heavy row whose Gram is split
// over `nparts` tasks and reduced by the last part to finish.
struct RowTask {
  long long begin;  // first CSR entry of this part
  int row;          // row being sampled
  int len;          // entries in this part
  int part;         // part index
  int nparts;       // number of parts of the row (1 = unsplit)
  int slot;         // scratch slot of part 0 (slots slot..slot+nparts-1)
  int split;        // index of the row's arrival counter (split rows only)
};

struct SampleParams {
  const RowTask* tasks;
  int ntasks;
  int nrows;
  int nother;                  // rows of the other factor (the BF16 copy holds one more, zero)
  int K;                       // true latent dimension (<= KP)
  const long long* rowptr;     // CSR of the rows being sampled
  const int* colidx;
  const double* vals;          // raw ratings (FP64 path)
  const uint2* packed;         // (column, centred rating as float bits) pairs (mixed path)
  double mean;
  double alpha;                // fixed noise precision (FixedGaussianNoise::alpha)
  const double* alpha_dev;     // adaptive noise: the precision on the device (&ctl->alpha),
                               // and the packed weights then hold y - mean unscaled; null = fixed
  const void* other;           // other factor: double (FP64) or bf16 (mixed), row stride KP
  const double* Lambda;        // K x K
  const double* mu;            // K
  const double* uhat;          // row stride KP, or null (BPMF)
  double* out_f64;             // FP64 latents (row stride KP)
  float* out_f32;              // mixed: FP32 master latents (row stride KP)
  __nv_bfloat16* out_bf16;     // mixed: BF16 copy used as the next half-sweep's gather source
  double* scratch;             // split-row partial Grams: (KP*KP + KP) doubles per slot
  double* retry_work;          // fused tensor-core sampler: per (CTA, finisher warp) work area
                               // of the FP64 redo of a row (tc_retry_work_doubles)
  unsigned* split_cnt;         // arrival counters of split rows (zero between launches)
  Ctl* ctl;
  int qslot;                   // which ctl->queue head this launch uses
  int mode;                    // 0 = rows of Y, 1 = columns
  unsigned long long seed;
  const double* znoise;        // optional injected N(0,1) draws (nrows x K), tests only
  int one;                     // univariate prior (MacauOnePrior): coordinate-wise draws from
                               // the row's Gram with the precisions on Lambda's diagonal
  int half_copy;               // mixed: the 16-bit gather copy (out_bf16) holds FP16, not BF16
  const int* row_width;        // tensor-core Gram records: per row, the width 8, 16 or 32 of the
                               // Gram block and rhs entries the finish reads (null: 32)
  long long wait_cycles;       // tensor-core sampler: clock budget of each barrier wait before
                               // the kernel gives up with kStatTimeout (0: about 2 s)
  int wait_test;               // tensor-core sampler, tests only: the MMA warp first waits on a
                               // barrier that nothing arrives on, so that wait runs out
};

#ifdef __CUDACC__
// Noise precision of a sampler launch: the device value under adaptive noise, else the fixed one.
__device__ __forceinline__ double noise_alpha(const SampleParams& p) {
  return p.alpha_dev ? *p.alpha_dev : p.alpha;
}
// Store of one value into the 16-bit gather copy of the latents (BF16, or FP16 when the Gram
// precision is FP16), rounded to nearest even.
__device__ __forceinline__ void store_copy(const SampleParams& p, size_t i, float x) {
  if (p.half_copy)
    reinterpret_cast<__half*>(p.out_bf16)[i] = __float2half_rn(x);
  else
    p.out_bf16[i] = __float2bfloat16_rn(x);
}
// Factor applied to a packed weight when it is read: packed weights carry the fixed alpha
// already, and are (y - mean) alone under adaptive noise.
__device__ __forceinline__ double packed_scale(const SampleParams& p) {
  return p.alpha_dev ? *p.alpha_dev : 1.0;
}
#endif

#define MG_CUDA(call)                                                                   \
  do {                                                                                  \
    cudaError_t e_ = (call);                                                            \
    if (e_ != cudaSuccess)                                                              \
      throw mg::CudaError(std::string(#call) + ": " + cudaGetErrorString(e_), e_);      \
  } while (0)

struct CudaError : std::runtime_error {
  cudaError_t code;
  CudaError(const std::string& m, cudaError_t c) : std::runtime_error(m), code(c) {}
};

struct MgError : std::runtime_error {
  int code;
  MgError(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

inline int kpad(int K) {
  if (K <= 8) return 8;
  if (K <= 16) return 16;
  if (K <= 32) return 32;
  if (K <= 64) return 64;
  return 128;
}

}  // namespace mg
