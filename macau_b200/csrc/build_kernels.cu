// Device construction of the rating matrix layouts (setup, once per data set):
//   build_csr_pair  COO triplets -> CSR of the rows and CSR of the columns (the CSC of Y), both
//                   with indices ascending and duplicate (i, j) entries summed in their input
//                   order, like Eigen's setFromTriplets (sparseFromIJV, bpmfutils.h:57-82).
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

__global__ void k_make_keys(const int* __restrict__ major, const int* __restrict__ minor,
                            long long n, unsigned long long* __restrict__ keys) {
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n;
       e += (long long)gridDim.x * blockDim.x)
    keys[e] = ((unsigned long long)(unsigned)major[e] << 32) | (unsigned)minor[e];
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

}  // namespace

long long build_csr_pair(const int* d_r, const int* d_c, const double* d_v, long long nnz,
                         long long nrow, long long ncol, long long* row_ptr, int* row_idx,
                         double* row_val, long long* col_ptr, int* col_idx, double* col_val,
                         cudaStream_t s) {
  if (nnz > 0x7fffffffLL) throw MgError(MG_ERR_ARG, "more than 2^31 - 1 training entries");
  unsigned long long *k0 = nullptr, *k1 = nullptr;
  double *v0 = nullptr, *v1 = nullptr;
  int *flags = nullptr, *pos = nullptr;
  MG_CUDA(cudaMallocAsync(&k0, sizeof(unsigned long long) * nnz, s));
  MG_CUDA(cudaMallocAsync(&k1, sizeof(unsigned long long) * nnz, s));
  MG_CUDA(cudaMallocAsync(&v0, sizeof(double) * nnz, s));
  MG_CUDA(cudaMallocAsync(&v1, sizeof(double) * nnz, s));
  MG_CUDA(cudaMallocAsync(&flags, sizeof(int) * nnz, s));
  MG_CUDA(cudaMallocAsync(&pos, sizeof(int) * nnz, s));
  long long nu = 0;
  try {
    const int T = 256;
    // 1. sort by (row, col); LSD radix sort is stable, so duplicates keep their input order
    k_make_keys<<<grid_for(nnz, T), T, 0, s>>>(d_r, d_c, nnz, k0);
    MG_CUDA(cudaGetLastError());
    MG_CUDA(cudaMemcpyAsync(v0, d_v, sizeof(double) * nnz, cudaMemcpyDeviceToDevice, s));
    sort_pairs(k0, k1, v0, v1, nnz, 32 + bits_for(nrow), s);
    // 2. de-duplicate: run heads, their output positions, sums in input order
    k_heads<<<grid_for(nnz, T), T, 0, s>>>(k1, nnz, flags);
    MG_CUDA(cudaGetLastError());
    size_t tb = 0;
    MG_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tb, flags, pos, (int)nnz, s));
    void* tmp = nullptr;
    MG_CUDA(cudaMallocAsync(&tmp, tb, s));
    const cudaError_t se = cub::DeviceScan::ExclusiveSum(tmp, tb, flags, pos, (int)nnz, s);
    MG_CUDA(cudaFreeAsync(tmp, s));
    MG_CUDA(se);
    k_dedupe<<<grid_for(nnz, T), T, 0, s>>>(k1, v1, flags, pos, nnz, k0, row_val);
    MG_CUDA(cudaGetLastError());
    int last[2] = {0, 0};
    MG_CUDA(cudaMemcpyAsync(&last[0], pos + nnz - 1, sizeof(int), cudaMemcpyDeviceToHost, s));
    MG_CUDA(cudaMemcpyAsync(&last[1], flags + nnz - 1, sizeof(int), cudaMemcpyDeviceToHost, s));
    MG_CUDA(cudaStreamSynchronize(s));
    nu = (long long)last[0] + last[1];
    // 3. CSR of the rows; swapped keys (col, row) for the columns
    k_csr_from_sorted<<<grid_for(nu + 1, T), T, 0, s>>>(k0, nu, nrow, row_ptr, row_idx, k1);
    MG_CUDA(cudaGetLastError());
    // 4. CSR of the columns: sort (col, row) keys with the values
    sort_pairs(k1, k0, row_val, col_val, nu, 32 + bits_for(ncol), s);
    k_csr_from_sorted<<<grid_for(nu + 1, T), T, 0, s>>>(k0, nu, ncol, col_ptr, col_idx, nullptr);
    MG_CUDA(cudaGetLastError());
    MG_CUDA(cudaStreamSynchronize(s));
  } catch (...) {
    cudaFreeAsync(k0, s);
    cudaFreeAsync(k1, s);
    cudaFreeAsync(v0, s);
    cudaFreeAsync(v1, s);
    cudaFreeAsync(flags, s);
    cudaFreeAsync(pos, s);
    throw;
  }
  MG_CUDA(cudaFreeAsync(k0, s));
  MG_CUDA(cudaFreeAsync(k1, s));
  MG_CUDA(cudaFreeAsync(v0, s));
  MG_CUDA(cudaFreeAsync(v1, s));
  MG_CUDA(cudaFreeAsync(flags, s));
  MG_CUDA(cudaFreeAsync(pos, s));
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
