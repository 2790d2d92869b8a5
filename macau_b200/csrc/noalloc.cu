// Hyperprior update that allocates no device memory: mg_normal_wishart_noalloc.
//
// The context API (mg_update_prior) keeps its reduction partials and Normal-Wishart workspace in
// buffers it cudaMalloc's at mg_init.  Some hosts cannot allocate at the point where they want
// to resample the hyperparameters: a serving process whose memory pool already owns all of the
// device memory (a further cudaMalloc would fail, or would have to evict the pool's blocks), or
// a latency-sensitive loop that cannot afford cudaMalloc's implicit device synchronisation.  For
// them this entry point runs the same kernels (k_stats + k_normal_wishart) with all of their
// scratch in one file-scope __device__ array of fixed size, so the only device memory it touches
// besides that array is the caller's inputs and outputs.
//
// Limits and sharing rules:
//   * K <= kNoAllocMaxK (64); the row reduction uses at most kNoAllocMaxParts (64) partial sums.
//     The array is 2.3 MB and every GPU that loads the library keeps it until the process exits.
//   * Every call on a device uses the same array; it holds whatever the last call left in it.
//     The control block (status word, sweep index) is cleared by each call; the partials and
//     workspace are fully overwritten before they are read.  Calls whose kernels overlap on the
//     GPU (different streams, or different host threads without ordering) race on the array.
//   * The call is synchronous: it copies the status word back and waits for `stream`, so it
//     cannot be recorded into a CUDA graph.
//   * The first call in a CUDA context of a device looks up the array's device address
//     (cudaGetSymbolAddress) with that device current and caches it under the context's unique
//     id; a context created later on the same device (after cudaDeviceReset) is looked up anew.
#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdio>
#include <mutex>

#include "common.cuh"
#include "kernels.h"

namespace mg {
namespace {

constexpr int kNoAllocMaxK = 64;
constexpr int kNoAllocMaxParts = 64;
constexpr size_t kPartDoubles = (size_t)kNoAllocMaxParts * (kNoAllocMaxK + kNoAllocMaxK * kNoAllocMaxK);
constexpr size_t kWorkDoubles = 3 * (size_t)kNoAllocMaxK + 4 * (size_t)kNoAllocMaxK * kNoAllocMaxK;
constexpr size_t kCtlDoubles = (sizeof(Ctl) + sizeof(double) - 1) / sizeof(double);
constexpr size_t kScratchDoubles = kPartDoubles + kWorkDoubles + kCtlDoubles;

// The scratch array.  In host code `g_noalloc_scratch` names a host-side stand-in, not device
// memory: only the address returned by cudaGetSymbolAddress may be handed to kernels.
__device__ __align__(256) double g_noalloc_scratch[kScratchDoubles];

std::mutex g_setup_mutex;
void* g_scratch_addr[64] = {nullptr};
unsigned long long g_scratch_ctx[64] = {0};  // unique id of the context the address belongs to

// Copies a message into the caller's buffer (no allocation).
void set_error(char* buf, int len, const char* msg) {
  if (buf && len > 0) snprintf(buf, (size_t)len, "%s", msg);
}

// Unique id of the CUDA context current on this thread, 0 when none is bound yet.  The two
// driver functions are fetched through the runtime (cudaGetDriverEntryPoint), so the library
// needs no link-time dependency on the driver library.
unsigned long long current_context_id() {
  using GetCurrent = CUresult (*)(CUcontext*);
  using GetId = CUresult (*)(CUcontext, unsigned long long*);
  static GetCurrent get_current = nullptr;
  static GetId get_id = nullptr;
  if (!get_current || !get_id) {
    void* f0 = nullptr;
    void* f1 = nullptr;
    cudaDriverEntryPointQueryResult q0 = cudaDriverEntryPointSymbolNotFound, q1 = q0;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f0, cudaEnableDefault, &q0) != cudaSuccess ||
        cudaGetDriverEntryPoint("cuCtxGetId", &f1, cudaEnableDefault, &q1) != cudaSuccess ||
        q0 != cudaDriverEntryPointSuccess || q1 != cudaDriverEntryPointSuccess || !f0 || !f1)
      return 0;
    get_current = reinterpret_cast<GetCurrent>(f0);
    get_id = reinterpret_cast<GetId>(f1);
  }
  CUcontext cu = nullptr;
  unsigned long long id = 0;
  if (get_current(&cu) != CUDA_SUCCESS || cu == nullptr) return 0;
  if (get_id(cu, &id) != CUDA_SUCCESS) return 0;
  return id;
}

// Device address of the scratch array on the current device, looked up once per device and
// CUDA context (the lookup itself binds the device's primary context when none is current).
cudaError_t scratch_address(double** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  unsigned long long ctx_id = current_context_id();
  if (ctx_id == 0 || !g_scratch_addr[dev] || g_scratch_ctx[dev] != ctx_id) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return e;
    if (ctx_id == 0) ctx_id = current_context_id();
    if (ctx_id == 0) return cudaErrorDeviceUninitialized;
    g_scratch_addr[dev] = p;
    g_scratch_ctx[dev] = ctx_id;
  }
  *out = static_cast<double*>(g_scratch_addr[dev]);
  return cudaSuccess;
}

}  // namespace
}  // namespace mg

extern "C" int mg_normal_wishart_noalloc(const double* U, int64_t N, int K, int stride,
                                         const double* mu0, double kappa, const double* T,
                                         int nu, uint64_t seed, uint32_t sweep, int mode,
                                         double* mu_out, double* Lambda_out, void* stream,
                                         char* err, int errlen) {
  using namespace mg;
  if (K < 1 || K > kNoAllocMaxK) {
    set_error(err, errlen,
              "mg_normal_wishart_noalloc: K must be in [1, 64] (the size of its fixed scratch "
              "array)");
    return MG_ERR_ARG;
  }
  if (N < 1 || stride < K || !U || !mu0 || !T || !mu_out || !Lambda_out) {
    set_error(err, errlen, "mg_normal_wishart_noalloc: invalid argument");
    return MG_ERR_ARG;
  }
  // the Bartlett factor draws chi-square variates with nu + N - i degrees of freedom (i < K)
  // and the posterior mean is scaled by 1 / (kappa + N): both need nu >= K and kappa > 0
  if (nu < K || !(kappa > 0.0)) {
    set_error(err, errlen, "mg_normal_wishart_noalloc: needs nu >= K and kappa > 0");
    return MG_ERR_ARG;
  }
  try {
    double* base = nullptr;
    MG_CUDA(scratch_address(&base));
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    double* partials = base;
    double* work = base + kPartDoubles;
    Ctl* ctl = reinterpret_cast<Ctl*>(base + kPartDoubles + kWorkDoubles);
    NwWork w;
    w.vec = work;
    w.m0 = work + 3 * K;
    w.m1 = w.m0 + K * K;
    w.m2 = w.m1 + K * K;
    w.m3 = w.m2 + K * K;
    int nb = stats_blocks(N);
    if (nb > kNoAllocMaxParts) nb = kNoAllocMaxParts;
    // the control block starts every call cleared (status = 0), then gets the sweep index
    MG_CUDA(cudaMemsetAsync(ctl, 0, sizeof(Ctl), s));
    launch_set_sweep(ctl, sweep, 0, s);
    launch_stats(U, false, nullptr, N, K, stride, 0, partials, nb, s);
    launch_normal_wishart(partials, nb, N, K, mu0, kappa, T, nu, nullptr, 0, nullptr, w, ctl,
                          seed, mode, mu_out, Lambda_out, s);
    int32_t status = 0;
    MG_CUDA(cudaMemcpyAsync(&status, &ctl->status, sizeof(status), cudaMemcpyDeviceToHost, s));
    MG_CUDA(cudaStreamSynchronize(s));
    if (status & kStatHyperFail) {
      set_error(err, errlen, "Cholesky Decomposition failed! (hyperprior)");
      return MG_ERR_CHOL;
    }
    set_error(err, errlen, "");
    return MG_OK;
  } catch (const MgError& e) {
    set_error(err, errlen, e.what());
    return e.code;
  } catch (const std::exception& e) {
    set_error(err, errlen, e.what());
    return MG_ERR_CUDA;
  }
}
