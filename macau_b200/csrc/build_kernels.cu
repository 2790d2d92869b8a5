// Device construction of the rating matrix layouts (setup, once per data set):
//   build_csr_pair  COO triplets -> CSR of the rows and CSR of the columns (the CSC of Y), both
//                   with indices ascending and duplicate (i, j) entries summed in their input
//                   order, like Eigen's setFromTriplets (sparseFromIJV, bpmfutils.h:57-82).
//   build_coo_sorted  the same sort and duplicate sums, returned as COO triplets in (major,
//                   minor) order (the test set in column-major order).
// Both check every index against the dimensions on the device.
//   launch_pack     per entry {index, float bits of (y - mean) * alpha} (mixed mode).
//   launch_pad      the 16-entry padded copy of the packed entries (tensor-core sampler).
// The sorts are CUB radix sorts over 64-bit (major << 32 | minor) keys; de-duplication, the row
// pointers and the packing are kernels of this file.
#include <algorithm>

#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include "common.cuh"
#include "kernels.h"

namespace mg {
namespace {

// Keys (major << 32 | minor).  An index outside [0, nmajor) x [0, nminor) sets *bad and gets
// key 0, so that the sort and the de-duplication stay in bounds until the host reads *bad.
__global__ void k_make_keys(const int* __restrict__ major, const int* __restrict__ minor,
                            long long n, long long nmajor, long long nminor,
                            unsigned long long* __restrict__ keys, int* __restrict__ bad) {
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n;
       e += (long long)gridDim.x * blockDim.x) {
    const int a = major[e], b = minor[e];
    const bool ok = a >= 0 && a < nmajor && b >= 0 && b < nminor;
    if (!ok) *bad = 1;
    keys[e] = ok ? ((unsigned long long)(unsigned)a << 32) | (unsigned)b : 0ull;
  }
}

__global__ void k_split_keys(const unsigned long long* __restrict__ keys, long long n,
                             int* __restrict__ major, int* __restrict__ minor) {
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n;
       e += (long long)gridDim.x * blockDim.x) {
    major[e] = (int)(keys[e] >> 32);
    minor[e] = (int)(keys[e] & 0xffffffffull);
  }
}

__global__ void k_heads(const unsigned long long* __restrict__ keys, long long n,
                        int* __restrict__ flags) {
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n;
       e += (long long)gridDim.x * blockDim.x)
    flags[e] = (e == 0 || keys[e] != keys[e - 1]) ? 1 : 0;
}

// Run heads write the run's key and the sum of its values in input order.
__global__ void k_dedupe(const unsigned long long* __restrict__ keys,
                         const double* __restrict__ vals, const int* __restrict__ flags,
                         const int* __restrict__ pos, long long n,
                         unsigned long long* __restrict__ ukeys, double* __restrict__ uvals) {
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n;
       e += (long long)gridDim.x * blockDim.x) {
    if (!flags[e]) continue;
    double s = vals[e];
    for (long long q = e + 1; q < n && !flags[q]; q++) s += vals[q];
    ukeys[pos[e]] = keys[e];
    uvals[pos[e]] = s;
  }
}

// From keys sorted by (major, minor): ptr[r] = first entry with major >= r (r = 0..nmajor),
// idx = minor, and swapped keys (minor << 32 | major) for the transpose sort.
__global__ void k_csr_from_sorted(const unsigned long long* __restrict__ keys, long long n,
                                  long long nmajor, long long* __restrict__ ptr,
                                  int* __restrict__ idx, unsigned long long* __restrict__ swapped) {
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e <= n;
       e += (long long)gridDim.x * blockDim.x) {
    const long long r_e = e < n ? (long long)(keys[e] >> 32) : nmajor;
    const long long r_p = e > 0 ? (long long)(keys[e - 1] >> 32) : -1;
    for (long long r = r_p + 1; r <= r_e; r++) ptr[r] = e;
    if (e < n) {
      const unsigned minor = (unsigned)(keys[e] & 0xffffffffull);
      idx[e] = (int)minor;
      if (swapped) swapped[e] = ((unsigned long long)minor << 32) | (keys[e] >> 32);
    }
  }
}

__global__ void k_pack(const int* __restrict__ idx, const double* __restrict__ val, long long n,
                       double mean, double alpha, uint2* __restrict__ out) {
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n;
       e += (long long)gridDim.x * blockDim.x) {
    const float w = (float)((val[e] - mean) * alpha);
    out[e] = make_uint2((unsigned)idx[e], __float_as_uint(w));
  }
}

// One warp per row: copies the row's packed entries to its padded position and fills the rest
// of its padded length with the sentinel {sentinel, 0}.
__global__ void k_pad(const long long* __restrict__ ptr, const long long* __restrict__ pptr,
                      long long nrows, const uint2* __restrict__ packed, unsigned sentinel,
                      uint2* __restrict__ out) {
  const int lane = threadIdx.x & 31;
  for (long long r = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5; r < nrows;
       r += ((long long)gridDim.x * blockDim.x) >> 5) {
    const long long b = ptr[r], len = ptr[r + 1] - b, pb = pptr[r], plen = pptr[r + 1] - pb;
    for (long long i = lane; i < plen; i += 32)
      out[pb + i] = i < len ? packed[b + i] : make_uint2(sentinel, 0u);
  }
}

int grid_for(long long n, int threads) {
  long long g = (n + threads - 1) / threads;
  if (g > 65535) g = 65535;
  return (int)(g < 1 ? 1 : g);
}

int bits_for(long long n) {
  int b = 1;
  while ((1LL << b) < n) b++;
  return b;
}

// Sorts (keys, vals) pairs by key into (keys_out, vals_out) over the low `end_bit` bits.
void sort_pairs(unsigned long long* keys_in, unsigned long long* keys_out, double* vals_in,
                double* vals_out, long long n, int end_bit, cudaStream_t s) {
  size_t tb = 0;
  MG_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tb, keys_in, keys_out, vals_in, vals_out,
                                          (int)n, 0, end_bit, s));
  void* tmp = nullptr;
  MG_CUDA(cudaMallocAsync(&tmp, tb, s));
  const cudaError_t e = cub::DeviceRadixSort::SortPairs(tmp, tb, keys_in, keys_out, vals_in,
                                                        vals_out, (int)n, 0, end_bit, s);
  MG_CUDA(cudaFreeAsync(tmp, s));
  MG_CUDA(e);
}

// Scratch of one build: two key and two value arrays, run-head flags with one extra int for the
// index check, and their output positions.
struct BuildScratch {
  unsigned long long *k0 = nullptr, *k1 = nullptr;
  double *v0 = nullptr, *v1 = nullptr;
  int *flags = nullptr, *pos = nullptr;
  cudaStream_t s;
  BuildScratch(long long n, cudaStream_t st) : s(st) {
    MG_CUDA(cudaMallocAsync(&k0, sizeof(unsigned long long) * n, s));
    MG_CUDA(cudaMallocAsync(&k1, sizeof(unsigned long long) * n, s));
    MG_CUDA(cudaMallocAsync(&v0, sizeof(double) * n, s));
    MG_CUDA(cudaMallocAsync(&v1, sizeof(double) * n, s));
    MG_CUDA(cudaMallocAsync(&flags, sizeof(int) * (n + 1), s));
    MG_CUDA(cudaMallocAsync(&pos, sizeof(int) * n, s));
  }
  ~BuildScratch() {
    cudaFreeAsync(k0, s);
    cudaFreeAsync(k1, s);
    cudaFreeAsync(v0, s);
    cudaFreeAsync(v1, s);
    cudaFreeAsync(flags, s);
    cudaFreeAsync(pos, s);
  }
};

// COO entries sorted by (major, minor) with their values; the LSD radix sort is stable, so
// duplicates keep their input order, and each run of equal keys is summed in that order into
// (b.k0, uvals).  Returns the number of distinct keys.  Throws MG_ERR_ARG with `what` when an
// index is out of range, before any kernel indexes by the keys.
long long sort_unique(const int* d_major, const int* d_minor, const double* d_v, long long nnz,
                      long long nmajor, long long nminor, const char* what, BuildScratch& b,
                      double* uvals) {
  cudaStream_t s = b.s;
  const int T = 256;
  MG_CUDA(cudaMemsetAsync(b.flags + nnz, 0, sizeof(int), s));
  k_make_keys<<<grid_for(nnz, T), T, 0, s>>>(d_major, d_minor, nnz, nmajor, nminor, b.k0,
                                             b.flags + nnz);
  MG_CUDA(cudaGetLastError());
  MG_CUDA(cudaMemcpyAsync(b.v0, d_v, sizeof(double) * nnz, cudaMemcpyDeviceToDevice, s));
  sort_pairs(b.k0, b.k1, b.v0, b.v1, nnz, 32 + bits_for(nmajor), s);
  // run heads, their output positions, sums in input order
  k_heads<<<grid_for(nnz, T), T, 0, s>>>(b.k1, nnz, b.flags);
  MG_CUDA(cudaGetLastError());
  size_t tb = 0;
  MG_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tb, b.flags, b.pos, (int)nnz, s));
  void* tmp = nullptr;
  MG_CUDA(cudaMallocAsync(&tmp, tb, s));
  const cudaError_t se = cub::DeviceScan::ExclusiveSum(tmp, tb, b.flags, b.pos, (int)nnz, s);
  MG_CUDA(cudaFreeAsync(tmp, s));
  MG_CUDA(se);
  k_dedupe<<<grid_for(nnz, T), T, 0, s>>>(b.k1, b.v1, b.flags, b.pos, nnz, b.k0, uvals);
  MG_CUDA(cudaGetLastError());
  int last[3] = {0, 0, 0};
  MG_CUDA(cudaMemcpyAsync(&last[0], b.pos + nnz - 1, sizeof(int), cudaMemcpyDeviceToHost, s));
  MG_CUDA(cudaMemcpyAsync(&last[1], b.flags + nnz - 1, sizeof(int) * 2, cudaMemcpyDeviceToHost,
                          s));
  MG_CUDA(cudaStreamSynchronize(s));
  if (last[2]) throw MgError(MG_ERR_ARG, what);
  return (long long)last[0] + last[1];
}

}  // namespace

long long build_csr_pair(const int* d_r, const int* d_c, const double* d_v, long long nnz,
                         long long nrow, long long ncol, long long* row_ptr, int* row_idx,
                         double* row_val, long long* col_ptr, int* col_idx, double* col_val,
                         cudaStream_t s) {
  if (nnz > 0x7fffffffLL) throw MgError(MG_ERR_ARG, "more than 2^31 - 1 training entries");
  BuildScratch b(nnz, s);
  const int T = 256;
  // 1. sort by (row, col), duplicates summed in input order
  const long long nu =
      sort_unique(d_r, d_c, d_v, nnz, nrow, ncol, "training index out of range", b, row_val);
  // 2. CSR of the rows; swapped keys (col, row) for the columns
  k_csr_from_sorted<<<grid_for(nu + 1, T), T, 0, s>>>(b.k0, nu, nrow, row_ptr, row_idx, b.k1);
  MG_CUDA(cudaGetLastError());
  // 3. CSR of the columns: sort (col, row) keys with the values
  sort_pairs(b.k1, b.k0, row_val, col_val, nu, 32 + bits_for(ncol), s);
  k_csr_from_sorted<<<grid_for(nu + 1, T), T, 0, s>>>(b.k0, nu, ncol, col_ptr, col_idx, nullptr);
  MG_CUDA(cudaGetLastError());
  MG_CUDA(cudaStreamSynchronize(s));
  return nu;
}

long long build_coo_sorted(const int* d_major, const int* d_minor, const double* d_v,
                           long long nnz, long long nmajor, long long nminor, const char* what,
                           int* out_major, int* out_minor, double* out_val, cudaStream_t s) {
  if (nnz > 0x7fffffffLL) throw MgError(MG_ERR_ARG, "more than 2^31 - 1 entries");
  BuildScratch b(nnz, s);
  const long long nu = sort_unique(d_major, d_minor, d_v, nnz, nmajor, nminor, what, b, out_val);
  k_split_keys<<<grid_for(nu, 256), 256, 0, s>>>(b.k0, nu, out_major, out_minor);
  MG_CUDA(cudaGetLastError());
  MG_CUDA(cudaStreamSynchronize(s));
  return nu;
}

// Sum of (v[i] - center) (sq = false) or of its square (sq = true) over n values: a fixed grid
// of blocks, each adding a grid-strided set in order and reducing in a fixed tree, then one
// warp over the block sums (deterministic for a given n).
__global__ void k_moment(const double* __restrict__ v, long long n, double center, bool sq,
                         double* __restrict__ partials) {
  __shared__ double ws[8];
  double acc = 0.0;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const double x = v[i] - center;
    acc += sq ? x * x : x;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) t += ws[w];
    partials[blockIdx.x] = t;
  }
}

__global__ void k_moment_final(const double* __restrict__ partials, int nb, double* out) {
  const int lane = threadIdx.x & 31;
  double t = 0.0;
  for (int b = lane; b < nb; b += 32) t += partials[b];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
  if (lane == 0) out[0] = t;
}

double value_moment(const double* v, long long n, double center, bool sq, cudaStream_t s) {
  const int nb = (int)std::max(1LL, std::min(1184LL, (n + 255) / 256));
  double* d = nullptr;
  MG_CUDA(cudaMallocAsync(&d, sizeof(double) * (nb + 1), s));
  k_moment<<<nb, 256, 0, s>>>(v, n, center, sq, d + 1);
  k_moment_final<<<1, 32, 0, s>>>(d + 1, nb, d);
  double h = 0.0;
  MG_CUDA(cudaMemcpyAsync(&h, d, sizeof(double), cudaMemcpyDeviceToHost, s));
  MG_CUDA(cudaFreeAsync(d, s));
  MG_CUDA(cudaStreamSynchronize(s));
  return h;
}

__global__ void k_copy16(const float* __restrict__ src, void* __restrict__ dst, long long n,
                         bool half) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    if (half) reinterpret_cast<__half*>(dst)[i] = __float2half_rn(src[i]);
    else reinterpret_cast<__nv_bfloat16*>(dst)[i] = __float2bfloat16_rn(src[i]);
  }
}

void launch_copy16(const float* src, void* dst, long long n, bool half, cudaStream_t s) {
  if (n <= 0) return;
  k_copy16<<<grid_for(n, 256), 256, 0, s>>>(src, dst, n, half);
  MG_CUDA(cudaGetLastError());
}

void launch_pack(const int* idx, const double* val, long long n, double mean, double alpha,
                 uint2* out, cudaStream_t s) {
  if (n <= 0) return;
  k_pack<<<grid_for(n, 256), 256, 0, s>>>(idx, val, n, mean, alpha, out);
  MG_CUDA(cudaGetLastError());
}

void launch_pad(const long long* ptr, const long long* pptr, long long nrows, const uint2* packed,
                unsigned sentinel, uint2* out, cudaStream_t s) {
  if (nrows <= 0) return;
  k_pad<<<grid_for(nrows * 32, 256), 256, 0, s>>>(ptr, pptr, nrows, packed, sentinel, out);
  MG_CUDA(cudaGetLastError());
}

}  // namespace mg
