// Side-information kernels: CSR SpMM (compute_uhat, A_mul_B(tmp, F), A_mul_Bx<N>), the
// right-hand side of MacauPrior::sample_beta and the block-CG solver solve_blockcg
// (linop.h:207-343) for (F^T F + reg I) X = B with up to 64 right-hand sides per block.
//
// Layout: a K x nfeat matrix of the reference is stored feature-major with a padded row of
// NRP (32 or 64) values, so one warp owns one feature / CSR row and lane l owns components
// l and l + 32.  SpMMs are warp-per-row gathers of whole 128/256-byte rows (binary F: adds only).
// The K x K reductions (P KP^T, R R^T) are per-block register-tile partials reduced in block
// order by one CTA (deterministic), which also does the small Cholesky solves.
//
// Precision: FP64, or FP32 vectors (P, R, KP, F P) with FP64 X, FP64 K x K algebra and an FP64
// residual replacement R = B - (F^T F + reg I) X every kReplaceEvery iterations.
#include <cmath>

#include "common.cuh"
#include "kernels.h"
#include "rng.cuh"
#include "warp_finish.cuh"

namespace mg {
namespace {

constexpr int kReplaceEvery = 20;
constexpr int kCgBatch = 8;         // CG iterations queued between host convergence checks
constexpr int kMaxCgIter = 100000;  // default iteration cap, the reference's (linop.h:279)
constexpr int kOuterThreads = 256;
constexpr int kOuterRows = 32;

template <typename V>
__device__ __forceinline__ V ldv(const V* p) { return *p; }

// ---------------- SpMM: out[r] = sum val * src[idx] (+ reg * add[r]) ----------------
template <typename V, int NRP>
__global__ void __launch_bounds__(256)
    k_spmm(const long long* __restrict__ ptr, const int* __restrict__ idx,
           const double* __restrict__ val, const float* __restrict__ valf, long long nrow,
           const V* __restrict__ src, int sstride, V* __restrict__ dst, int dstride, int ncomp,
           const V* __restrict__ add, int astride, double reg, const double* __restrict__ reg_dev,
           const uint32_t* __restrict__ done) {
  if (done && *done) return;
  constexpr int C = NRP / 32;
  const int lane = threadIdx.x & 31;
  const long long nw = (long long)gridDim.x * (blockDim.x >> 5);
  const V r = (V)(reg_dev ? *reg_dev : reg);
  for (long long row = (long long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
       row < nrow; row += nw) {
    V acc[C];
#pragma unroll
    for (int c = 0; c < C; c++) acc[c] = (V)0;
    const long long b = ptr[row], e = ptr[row + 1];
    for (long long q = b; q < e; q++) {
      const V* s = src + (size_t)idx[q] * sstride;
      V w = (V)1;
      if constexpr (sizeof(V) == 8) {
        if (val) w = (V)val[q];
      } else {
        if (valf) w = (V)valf[q];
      }
#pragma unroll
      for (int c = 0; c < C; c++) {
        const int k = lane + 32 * c;
        if (k < ncomp) acc[c] += (val || valf) ? s[k] * w : s[k];
      }
    }
#pragma unroll
    for (int c = 0; c < C; c++) {
      const int k = lane + 32 * c;
      if (k < ncomp) {
        V o = acc[c];
        if (add) o += r * add[(size_t)row * astride + k];
        dst[(size_t)row * dstride + k] = o;
      }
    }
  }
}

// ---------------- SpMM over a work split (DevCsr::tasks) ----------------
// One warp per task (a whole row, or one part of a long row).  Entries are read four at a time
// (independent gathers in flight) and added in CSR order.  A part stores its FP64 partial row in
// A.parts; the last part of a row to finish (arrival counter) adds the parts in part order and
// writes the row.  Whole rows give the same sums as k_spmm.
template <typename V, int NRP>
__global__ void __launch_bounds__(256)
    k_spmm_split(const DevCsr A, const V* __restrict__ src, int sstride, V* __restrict__ dst,
                 int dstride, int ncomp, const V* __restrict__ add, int astride, double reg,
                 const double* __restrict__ reg_dev, const uint32_t* __restrict__ done) {
  if (done && *done) return;
  constexpr int C = NRP / 32;
  const int lane = threadIdx.x & 31;
  const int nw = gridDim.x * (blockDim.x >> 5);
  const bool weighted = sizeof(V) == 8 ? A.val != nullptr : A.valf != nullptr;
  for (int ti = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); ti < A.ntasks; ti += nw) {
    const RowTask tk = A.tasks[ti];
    V acc[C];
#pragma unroll
    for (int c = 0; c < C; c++) acc[c] = (V)0;
    const long long b = tk.begin, e = tk.begin + tk.len;
    long long q = b;
    for (; q + 4 <= e; q += 4) {
      const V* s0 = src + (size_t)A.idx[q] * sstride;
      const V* s1 = src + (size_t)A.idx[q + 1] * sstride;
      const V* s2 = src + (size_t)A.idx[q + 2] * sstride;
      const V* s3 = src + (size_t)A.idx[q + 3] * sstride;
      V w0 = (V)1, w1 = (V)1, w2 = (V)1, w3 = (V)1;
      if (weighted) {
        if constexpr (sizeof(V) == 8) {
          w0 = (V)A.val[q]; w1 = (V)A.val[q + 1]; w2 = (V)A.val[q + 2]; w3 = (V)A.val[q + 3];
        } else {
          w0 = (V)A.valf[q]; w1 = (V)A.valf[q + 1]; w2 = (V)A.valf[q + 2]; w3 = (V)A.valf[q + 3];
        }
      }
#pragma unroll
      for (int c = 0; c < C; c++) {
        const int k = lane + 32 * c;
        if (k < ncomp) {
          const V x0 = s0[k], x1 = s1[k], x2 = s2[k], x3 = s3[k];
          if (weighted) {
            acc[c] += x0 * w0;
            acc[c] += x1 * w1;
            acc[c] += x2 * w2;
            acc[c] += x3 * w3;
          } else {
            acc[c] += x0;
            acc[c] += x1;
            acc[c] += x2;
            acc[c] += x3;
          }
        }
      }
    }
    for (; q < e; q++) {
      const V* s0 = src + (size_t)A.idx[q] * sstride;
      V w0 = (V)1;
      if (weighted) {
        if constexpr (sizeof(V) == 8) w0 = (V)A.val[q];
        else w0 = (V)A.valf[q];
      }
#pragma unroll
      for (int c = 0; c < C; c++) {
        const int k = lane + 32 * c;
        if (k < ncomp) acc[c] += weighted ? s0[k] * w0 : s0[k];
      }
    }
    const V r = (V)(reg_dev ? *reg_dev : reg);
    if (tk.nparts == 1) {
#pragma unroll
      for (int c = 0; c < C; c++) {
        const int k = lane + 32 * c;
        if (k < ncomp) {
          V o = acc[c];
          if (add) o += r * add[(size_t)tk.row * astride + k];
          dst[(size_t)tk.row * dstride + k] = o;
        }
      }
      continue;
    }
    double* pp = A.parts + (size_t)(tk.slot + tk.part) * 64;
#pragma unroll
    for (int c = 0; c < C; c++) {
      const int k = lane + 32 * c;
      if (k < ncomp) pp[k] = (double)acc[c];
    }
    __threadfence();
    __syncwarp();
    unsigned last = 0;
    if (lane == 0) last = atomicAdd(&A.split_cnt[tk.split], 1u) == (unsigned)(tk.nparts - 1);
    last = __shfl_sync(0xffffffffu, last, 0);
    if (!last) continue;
    __threadfence();
    const double* p0 = A.parts + (size_t)tk.slot * 64;
#pragma unroll
    for (int c = 0; c < C; c++) {
      const int k = lane + 32 * c;
      if (k < ncomp) {
        double t = 0.0;
        for (int pt = 0; pt < tk.nparts; pt++) t += __ldcg(p0 + (size_t)pt * 64 + k);
        V o = (V)t;
        if (add) o += r * add[(size_t)tk.row * astride + k];
        dst[(size_t)tk.row * dstride + k] = o;
      }
    }
    if (lane == 0) A.split_cnt[tk.split] = 0u;
  }
}

// Sum of `nparts` records of `len` doubles: eight lanes per entry, lane l adding records
// l, l + 8, ... in order, then a fixed xor tree over the eight lanes (deterministic).
__global__ void __launch_bounds__(256)
    k_sum_records(const double* __restrict__ parts, int nparts, int len, double* __restrict__ out,
                  const uint32_t* __restrict__ done) {
  if (done && *done) return;
  const int g = (blockIdx.x * blockDim.x + threadIdx.x) >> 3, l = threadIdx.x & 7;
  double s = 0.0;
  if (g < len)
#pragma unroll 4
    for (int b = l; b < nparts; b += 8) s += parts[(size_t)b * len + g];
  s += __shfl_xor_sync(0xffffffffu, s, 4, 8);
  s += __shfl_xor_sync(0xffffffffu, s, 2, 8);
  s += __shfl_xor_sync(0xffffffffu, s, 1, 8);
  if (l == 0 && g < len) out[g] = s;
}

// ---------------- per-block partial of sum_f a_f b_f^T (NRP x NRP, full) ----------------
// Rows staged 32 at a time in shared memory (the next 32 prefetched into registers); each thread
// accumulates a 4 x 4 tile (i in 4 ti .., j in 4 tj ..) over the rows of its row group (every
// G-th staged row; G = 4 for NRP = 32, 1 for NRP = 64), and the groups' tiles are added in group
// order at the end.  partials[block][i + j * NRP] = sum over the block's rows of a_i b_j.
template <typename V, int NRP>
__global__ void __launch_bounds__(kOuterThreads, 2)
    k_outer(const V* __restrict__ A, const V* __restrict__ B, int stride, long long nrow,
            long long rows_per_block, double* __restrict__ partials,
            const uint32_t* __restrict__ done) {
  if (done && *done) return;
  constexpr int T4 = NRP / 4, TILES = T4 * T4, G = kOuterThreads / TILES;
  constexpr int LD = NRP + 4, PRE = kOuterRows * NRP / kOuterThreads;  // staged values / thread
  static_assert(G >= 1 && TILES * G == kOuterThreads, "tile layout");
  __shared__ __align__(16) double as[kOuterRows][LD], bs[kOuterRows][LD];
  __shared__ double red[G > 1 ? G - 1 : 1][G > 1 ? TILES : 1][16];
  const int t = threadIdx.x, tile = t % TILES, rg = t / TILES;
  const int ti = tile / T4, tj = tile % T4;
  const long long r0 = (long long)blockIdx.x * rows_per_block;
  const long long r1 = min(nrow, r0 + rows_per_block);
  double acc[4][4];
#pragma unroll
  for (int x = 0; x < 4; x++)
#pragma unroll
    for (int y = 0; y < 4; y++) acc[x][y] = 0.0;
  double na[PRE], nb[PRE];
  auto fetch = [&](long long b0) {
#pragma unroll
    for (int q = 0; q < PRE; q++) {
      const int e = t + kOuterThreads * q, rr = e / NRP, k = e % NRP;
      const bool in = b0 + rr < r1;
      na[q] = in ? (double)A[(b0 + rr) * stride + k] : 0.0;
      nb[q] = in ? (double)B[(b0 + rr) * stride + k] : 0.0;
    }
  };
  fetch(r0);
  for (long long b0 = r0; b0 < r1; b0 += kOuterRows) {
    const int cnt = (int)min((long long)kOuterRows, r1 - b0);
    __syncthreads();
#pragma unroll
    for (int q = 0; q < PRE; q++) {
      const int e = t + kOuterThreads * q;
      as[e / NRP][e % NRP] = na[q];
      bs[e / NRP][e % NRP] = nb[q];
    }
    __syncthreads();
    if (b0 + kOuterRows < r1) fetch(b0 + kOuterRows);
    for (int r = rg; r < cnt; r += G) {
      const double2 i01 = *reinterpret_cast<const double2*>(&as[r][4 * ti]);
      const double2 i23 = *reinterpret_cast<const double2*>(&as[r][4 * ti + 2]);
      const double2 j01 = *reinterpret_cast<const double2*>(&bs[r][4 * tj]);
      const double2 j23 = *reinterpret_cast<const double2*>(&bs[r][4 * tj + 2]);
      const double xi[4] = {i01.x, i01.y, i23.x, i23.y}, xj[4] = {j01.x, j01.y, j23.x, j23.y};
#pragma unroll
      for (int x = 0; x < 4; x++)
#pragma unroll
        for (int y = 0; y < 4; y++) acc[x][y] = fma(xi[x], xj[y], acc[x][y]);
    }
  }
  if constexpr (G > 1) {
    if (rg > 0)
#pragma unroll
      for (int x = 0; x < 4; x++)
#pragma unroll
        for (int y = 0; y < 4; y++) red[rg - 1][tile][x * 4 + y] = acc[x][y];
    __syncthreads();
  }
  if (rg == 0) {
    double* out = partials + (size_t)blockIdx.x * NRP * NRP;
#pragma unroll
    for (int x = 0; x < 4; x++)
#pragma unroll
      for (int y = 0; y < 4; y++) {
        double v = acc[x][y];
        if constexpr (G > 1)
#pragma unroll
          for (int g = 0; g < G - 1; g++) v += red[g][tile][x * 4 + y];
        out[(4 * ti + x) + (4 * tj + y) * NRP] = v;
      }
  }
}

// Sum of the block partials of entry (i, j), i,j < n.
__device__ __forceinline__ double sum_part(const double* partials, int nparts, int NRP, int i,
                                           int j) {
  double s = 0.0;
  for (int b = 0; b < nparts; b++) s += partials[(size_t)b * NRP * NRP + i + j * NRP];
  return s;
}

// Left-looking lower Cholesky of the n x n matrix A (leading dimension ld) by one CTA, column by
// column; thread i computes L(i, j).  On a non-positive pivot it stops and leaves column j and
// the columns after it as they were, like the unchecked Eigen llt() the reference uses
// (linop.h:287, 313): the caller's solves then read that partial factor.  Returns false then.
__device__ bool cta_chol_n(double* A, int n, int ld) {
  __syncthreads();
  for (int j = 0; j < n; j++) {
    double d = A[j + j * ld];
    for (int p = 0; p < j; p++) d -= A[j + p * ld] * A[j + p * ld];
    if (!(d > 0.0)) {
      __syncthreads();
      return false;
    }
    const double ljj = sqrt(d);
    for (int i = j + 1 + threadIdx.x; i < n; i += blockDim.x) {
      double s = A[i + j * ld];
      for (int p = 0; p < j; p++) s -= A[i + p * ld] * A[j + p * ld];
      A[i + j * ld] = s / ljj;
    }
    __syncthreads();
    if (threadIdx.x == 0) A[j + j * ld] = ljj;
    __syncthreads();
  }
  return true;
}

// small layout (doubles): RtR[64*64] | RtR2[64*64] | M[64*64] | A[64*64] | Psi[64*64] | norms[64]
//                         | inorms[64] | flags[4]
constexpr int kSq = 64 * 64;
struct SmallView {
  double *RtR, *RtR2, *M, *A, *Psi, *norms, *inorms, *flags;
  __host__ __device__ explicit SmallView(double* s)
      : RtR(s), RtR2(s + kSq), M(s + 2 * kSq), A(s + 3 * kSq), Psi(s + 4 * kSq),
        norms(s + 5 * kSq), inorms(s + 5 * kSq + 64), flags(s + 5 * kSq + 128) {}
};

// RtR = sum partials (full matrix from the lower triangle, A_mul_At_combo + makeSymmetric)
__global__ void k_cg_rtr(const double* partials, int nparts, int NRP, int n, double* small) {
  SmallView v(small);
  for (int e = threadIdx.x; e < n * n; e += blockDim.x) {
    const int i = e % n, j = e / n;
    const int lo = i > j ? i : j, hi = i > j ? j : i;
    v.RtR[i + j * 64] = sum_part(partials, nparts, NRP, lo, hi);
  }
}

// norms of the RHS rows (B.row(rhs) over all features) from the outer partials of (B, B)
__global__ void k_cg_norms(const double* partials, int nparts, int NRP, int n, double* small) {
  SmallView v(small);
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    const double s = sum_part(partials, nparts, NRP, i, i);
    v.norms[i] = sqrt(s);
    v.inorms[i] = 1.0 / v.norms[i];
  }
}

// R = P = B * inorms (V), X = 0, Bn = B * inorms (FP64, for residual replacement)
template <typename V>
__global__ void k_cg_init(const double* __restrict__ B, int bstride, long long nfeat, int n,
                          int NRP, const double* small, V* R, V* P, double* X, double* Bn,
                          Ctl* ctl) {
  SmallView v(const_cast<double*>(small));
  if (blockIdx.x == 0 && threadIdx.x == 0) ctl->cg_done = 0u;  // the iterations' skip flag
  const long long total = nfeat * NRP;
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    const long long f = e / NRP;
    const int k = (int)(e % NRP);
    double r = 0.0;
    if (k < n) r = B[f * bstride + k] * v.inorms[k];
    R[e] = (V)r;
    P[e] = (V)r;
    X[e] = 0.0;
    if (Bn) Bn[e] = r;
  }
}

// Out(c, i) = (M^{-T} M^{-1} Rhs)(i, c) for the n columns of Rhs, M the lower Cholesky factor
// in v.M (leading dimension 64): thread c solves column c, forward then backward substitution in
// the order of the reference's llt().solve.  The general path (n > 32, or a failed pivot).
__device__ void cta_chol_solve_cols(const double* M, const double* Rhs, int n, double* Out) {
  for (int c = threadIdx.x; c < n; c += blockDim.x) {
    double y[64];
    for (int i = 0; i < n; i++) y[i] = Rhs[i + c * 64];
    for (int i = 0; i < n; i++) {
      double s = y[i];
      for (int p = 0; p < i; p++) s -= M[i + p * 64] * y[p];
      y[i] = s / M[i + i * 64];
    }
    for (int i = n - 1; i >= 0; i--) {
      double s = y[i];
      for (int p = i + 1; p < n; p++) s -= M[p + i * 64] * y[p];
      y[i] = s / M[i + i * 64];
    }
    for (int i = 0; i < n; i++) Out[c + i * 64] = y[i];
  }
}

constexpr int kSolveThreads = 256;
constexpr int kLcLd = 36;

// The same solves for n <= 32 with the factor in registers: warp 0 factorises the SPD matrix Ms
// (lower triangle, padded with the identity beyond n) by warp_factor, publishing L^T in Lc;
// then warp w solves columns w, w + 8, ...: lane i holds L(i, j) for j <= i and L(j, i) for
// j > i and runs each substitution as 32 shuffle steps.  Returns false, with Out untouched, when
// a pivot is not positive (the caller then takes the general path).
__device__ bool warp_chol_solve(const double (*Ms)[33], double* Lc, const double* Rhs, int n,
                                double* Out, int* okf) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (warp == 0) {
    double a[32], rinv = 1.0, d0 = 1.0;
#pragma unroll
    for (int j = 0; j < 32; j++) {
      double x;
      if (lane < n && j < n) x = j <= lane ? Ms[lane][j] : Ms[j][lane];
      else x = lane == j ? 1.0 : 0.0;
      a[j] = x;
      if (j == lane) d0 = x;
    }
    const bool ok = warp_factor<double, 32>(a, rinv, lane, 0.0, d0, Lc, kLcLd);
    if (lane == 0) *okf = ok ? 1 : 0;
  }
  __syncthreads();
  if (!*okf) return false;
  double m[32], dinv = 1.0;
#pragma unroll
  for (int j = 0; j < 32; j++) {
    m[j] = j <= lane ? Lc[j * kLcLd + lane] : Lc[lane * kLcLd + j];
    if (j == lane) dinv = 1.0 / m[j];
  }
  for (int c = warp; c < n; c += kSolveThreads / 32) {
    double y = lane < n ? Rhs[lane + c * 64] : 0.0;
#pragma unroll
    for (int j = 0; j < 32; j++) {
      if (lane == j) y *= dinv;
      const double yj = __shfl_sync(0xffffffffu, y, j);
      if (lane > j) y = fma(-m[j], yj, y);
    }
#pragma unroll
    for (int j = 31; j >= 0; j--) {
      if (lane == j) y *= dinv;
      const double xj = __shfl_sync(0xffffffffu, y, j);
      if (lane < j) y = fma(-m[j], xj, y);
    }
    if (lane < n) Out[c + lane * 64] = y;
  }
  return true;
}

// A = (chol(PtKP) \ RtR)^T  (linop.h:286-289); PtKP from the lower triangle of sum P KP^T.
__global__ void __launch_bounds__(kSolveThreads, 1)
    k_cg_solve_a(const double* partials, int nparts, int NRP, int n, double* small, Ctl* ctl) {
  if (ctl->cg_done) return;
  __shared__ double Ms[32][33];
  __shared__ __align__(16) double Lc[32 * kLcLd];
  __shared__ int okf;
  SmallView v(small);
  if (n <= 32) {
    for (int e = threadIdx.x; e < n * n; e += blockDim.x) {
      const int i = e % n, j = e / n;
      if (i >= j) Ms[i][j] = sum_part(partials, nparts, NRP, i, j);
    }
    __syncthreads();
    if (warp_chol_solve(Ms, Lc, v.RtR, n, v.A, &okf)) return;
  }
  for (int e = threadIdx.x; e < n * n; e += blockDim.x) {
    const int i = e % n, j = e / n;
    if (i >= j) v.M[i + j * 64] = sum_part(partials, nparts, NRP, i, j);  // P(i) . KP(j)
  }
  cta_chol_n(v.M, n, 64);  // a failed pivot is not an error in the reference either
  __syncthreads();
  // columns c of RtR solved: Y = L^{-T} L^{-1} RtR ; A(c, i) = Y(i, c)
  cta_chol_solve_cols(v.M, v.RtR, n, v.A);
}

// RtR2 = sum R R^T; converged = all diag < tol^2; Psi = (chol(RtR) \ RtR2)^T; RtR <- RtR2.
__global__ void __launch_bounds__(kSolveThreads, 1)
    k_cg_solve_psi(const double* partials, int nparts, int NRP, int n, double tolsq,
                   double* small, Ctl* ctl, int* flag_out, int iter) {
  if (ctl->cg_done) return;
  __shared__ double Ms[32][33];
  __shared__ __align__(16) double Lc[32 * kLcLd];
  __shared__ int okf;
  SmallView v(small);
  __shared__ int conv;
  for (int e = threadIdx.x; e < n * n; e += blockDim.x) {
    const int i = e % n, j = e / n;
    const int lo = i > j ? i : j, hi = i > j ? j : i;
    v.RtR2[i + j * 64] = sum_part(partials, nparts, NRP, lo, hi);
  }
  if (threadIdx.x == 0) conv = 1;
  __syncthreads();
  __shared__ int bad;
  if (threadIdx.x == 0) bad = 0;
  __syncthreads();
  if (threadIdx.x < n) {
    const double d = v.RtR2[threadIdx.x + threadIdx.x * 64];
    if (!(d < tolsq)) atomicAnd(&conv, 0);
    if (!isfinite(d)) atomicOr(&bad, 1);
  }
  __syncthreads();
  if (bad) {  // non-finite residual: stop the iteration and report a breakdown
    if (threadIdx.x == 0) {
      conv = 1;
      atomicOr(&ctl->status, kStatCgFail);
    }
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    v.flags[0] = conv;
    ctl->cg_done = (uint32_t)conv;
    if (flag_out && conv) {  // [1]: the iteration that converged, then [0]: done
      flag_out[1] = iter;
      __threadfence_system();
      flag_out[0] = 1;
    }
  }
  if (conv) return;
  bool fast = false;
  if (n <= 32) {
    for (int e = threadIdx.x; e < n * n; e += blockDim.x) {
      const int i = e % n, j = e / n;
      if (i >= j) Ms[i][j] = v.RtR[i + j * 64];
    }
    __syncthreads();
    fast = warp_chol_solve(Ms, Lc, v.RtR2, n, v.Psi, &okf);
  }
  if (!fast) {
    for (int e = threadIdx.x; e < n * n; e += blockDim.x) {
      const int i = e % n, j = e / n;
      v.M[i + j * 64] = v.RtR[i + j * 64];
    }
    cta_chol_n(v.M, n, 64);
    __syncthreads();
    cta_chol_solve_cols(v.M, v.RtR2, n, v.Psi);
  }
  __syncthreads();
  for (int e = threadIdx.x; e < n * n; e += blockDim.x) {
    const int i = e % n, j = e / n;
    v.RtR[i + j * 64] = v.RtR2[i + j * 64];
  }
}

// Row updates of the block-CG as small tiled products with the n x n matrix M (A or Psi, in
// shared memory, M[i + k * 64]):
//   UPDATE (linop.h:292-300):   X[f] += M P[f],  R[f] -= M KP[f]
//   PUPDATE (linop.h:319-326):  P[f] = R[f] + M P[f]
// A block takes 32 feature rows, staged k-major in shared memory; thread (trow, tcol) owns rows
// 2 trow, 2 trow + 1 and components tcol * CI .. + CI - 1, and sums over k in order with fma.
constexpr int kRowTile = 32;
constexpr size_t rows_smem(int NRP, bool update) {
  return sizeof(double) * ((size_t)NRP * NRP + (update ? 2 : 1) * (size_t)NRP * (kRowTile + 2));
}
template <typename V, int NRP, bool UPDATE>
__global__ void __launch_bounds__(256)
    k_cg_rows(long long nfeat, int n, const double* small, const V* __restrict__ P,
              const V* __restrict__ KPm, V* __restrict__ R, double* __restrict__ X,
              V* __restrict__ Pout, const uint32_t* __restrict__ done) {
  if (*done) return;
  constexpr int CI = NRP / 16;  // components per thread: 2 or 4
  extern __shared__ __align__(16) double dsm[];  // Ms | Pt | Qt (rows_smem bytes)
  double(*Ms)[NRP] = reinterpret_cast<double(*)[NRP]>(dsm);  // Ms[k][i] = M(i, k)
  double(*Pt)[kRowTile + 2] = reinterpret_cast<double(*)[kRowTile + 2]>(dsm + NRP * NRP);
  double(*Qt)[kRowTile + 2] = Pt + NRP;
  SmallView v(const_cast<double*>(small));
  const double* M = UPDATE ? v.A : v.Psi;
  for (int e = threadIdx.x; e < NRP * NRP; e += blockDim.x) {
    const int i = e % NRP, k = e / NRP;
    Ms[k][i] = (i < n && k < n) ? M[i + k * 64] : 0.0;
  }
  const long long f0 = (long long)blockIdx.x * kRowTile;
  for (int e = threadIdx.x; e < kRowTile * NRP; e += blockDim.x) {
    const int r = e / NRP, k = e % NRP;
    const bool in = f0 + r < nfeat;
    Pt[k][r] = in ? (double)P[(f0 + r) * NRP + k] : 0.0;
    if constexpr (UPDATE) Qt[k][r] = in ? (double)KPm[(f0 + r) * NRP + k] : 0.0;
  }
  __syncthreads();
  const int tcol = threadIdx.x % 16, trow = threadIdx.x / 16;
  double sp[2][CI], sq[2][CI];
#pragma unroll
  for (int x = 0; x < 2; x++)
#pragma unroll
    for (int y = 0; y < CI; y++) sp[x][y] = sq[x][y] = 0.0;
  for (int k = 0; k < n; k++) {
    const double2 pr = *reinterpret_cast<const double2*>(&Pt[k][2 * trow]);
    double m[CI];
#pragma unroll
    for (int y = 0; y < CI; y += 2) {
      const double2 mm = *reinterpret_cast<const double2*>(&Ms[k][CI * tcol + y]);
      m[y] = mm.x;
      m[y + 1] = mm.y;
    }
#pragma unroll
    for (int y = 0; y < CI; y++) {
      sp[0][y] = fma(m[y], pr.x, sp[0][y]);
      sp[1][y] = fma(m[y], pr.y, sp[1][y]);
    }
    if constexpr (UPDATE) {
      const double2 qr = *reinterpret_cast<const double2*>(&Qt[k][2 * trow]);
#pragma unroll
      for (int y = 0; y < CI; y++) {
        sq[0][y] = fma(m[y], qr.x, sq[0][y]);
        sq[1][y] = fma(m[y], qr.y, sq[1][y]);
      }
    }
  }
#pragma unroll
  for (int x = 0; x < 2; x++) {
    const long long f = f0 + 2 * trow + x;
    if (f >= nfeat) continue;
#pragma unroll
    for (int y = 0; y < CI; y++) {
      const int i = CI * tcol + y;
      if (i >= n) continue;
      if constexpr (UPDATE) {
        X[f * NRP + i] += sp[x][y];
        R[f * NRP + i] = (V)((double)R[f * NRP + i] - sq[x][y]);
      } else {
        Pout[f * NRP + i] = (V)((double)R[f * NRP + i] + sp[x][y]);
      }
    }
  }
}

// R = Bn - KX (FP64 residual replacement, rounded to V)
template <typename V>
__global__ void k_cg_resid(long long total, int NRP, int n, const double* __restrict__ Bn,
                           const double* __restrict__ KX, V* __restrict__ R,
                           const uint32_t* __restrict__ done) {
  if (*done) return;
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    const int k = (int)(e % NRP);
    R[e] = (V)(k < n ? Bn[e] - KX[e] : 0.0);
  }
}

// X_out[f, k] = X[f, k] * norms[k]
__global__ void k_cg_finish(long long nfeat, int NRP, int n, const double* small,
                            const double* __restrict__ X, double* __restrict__ out,
                            int ostride) {
  SmallView v(const_cast<double*>(small));
  const long long total = nfeat * n;
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    const long long f = e / n;
    const int k = (int)(e % n);
    out[f * ostride + k] = X[f * NRP + k] * v.norms[k];
  }
}

// ---------------- sample_beta right-hand side ----------------
// MvNormal_prec_omp(Lambda, n) column c (mvnormal.cpp:186-201): x = L^{-T} z with z keyed
// (purpose, c); one thread per column, back substitution in the reference's order.
__device__ __forceinline__ void mvn_col(const double* Ls, int K, unsigned long long seed,
                                        uint32_t sweep, uint32_t stream, uint32_t col,
                                        double* z) {
  for (int i = 0; i < K; i += 2) {
    double z0, z1;
    normal_pair(seed, sweep, stream, col, (uint32_t)(i >> 1), &z0, &z1);
    z[i] = z0;
    if (i + 1 < K) z[i + 1] = z1;
  }
  for (int i = K - 1; i >= 0; i--) {
    double s = z[i];
    for (int p = i + 1; p < K; p++) s -= Ls[p + i * K] * z[p];
    z[i] = s / Ls[i + i * K];
  }
}

// tmp[n] = (U[n] + MvNormal_prec(Lambda)[n]) - mu   (latentprior.cpp:277)
template <typename T>
__global__ void __launch_bounds__(128)
    k_beta_tmp(const T* __restrict__ U, int ustride, long long N, int K,
               const double* __restrict__ L, const double* __restrict__ mu, const Ctl* ctl,
               unsigned long long seed, int mode, double* __restrict__ tmp, int tstride) {
  __shared__ double Ls[64 * 64];
  for (int e = threadIdx.x; e < K * K; e += blockDim.x) Ls[e] = L[e];
  __syncthreads();
  const uint32_t sweep = ctl->sweep;
  const uint32_t st = stream_id(kMvnN, (uint32_t)mode);
  double z[64];
  for (long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x; n < N;
       n += (long long)gridDim.x * blockDim.x) {
    mvn_col(Ls, K, seed, sweep, st, (uint32_t)n, z);
    for (int k = 0; k < K; k++) tmp[n * tstride + k] = ((double)U[n * ustride + k] + z[k]) - mu[k];
  }
}

// B[f] += sqrt(lambda_beta) * MvNormal_prec(Lambda)[f]   (latentprior.cpp:278)
__global__ void __launch_bounds__(128)
    k_beta_noise(long long nfeat, int K, const double* __restrict__ L,
                 const double* __restrict__ lb, const Ctl* ctl, unsigned long long seed,
                 int mode, double* __restrict__ B, int bstride) {
  __shared__ double Ls[64 * 64];
  for (int e = threadIdx.x; e < K * K; e += blockDim.x) Ls[e] = L[e];
  __syncthreads();
  const uint32_t sweep = ctl->sweep;
  const uint32_t st = stream_id(kMvnF, (uint32_t)mode);
  const double slb = sqrt(*lb);
  double z[64];
  for (long long f = (long long)blockIdx.x * blockDim.x + threadIdx.x; f < nfeat;
       f += (long long)gridDim.x * blockDim.x) {
    mvn_col(Ls, K, seed, sweep, st, (uint32_t)f, z);
    for (int k = 0; k < K; k++) B[f * bstride + k] += slb * z[k];
  }
}

__global__ void k_small_chol(const double* A, int K, double* L, Ctl* ctl) {
  __shared__ double M[64 * 64];
  for (int e = threadIdx.x; e < K * K; e += blockDim.x) M[e] = A[e];
  cta_chol_n(M, K, K);  // LLT of MvNormal_prec_omp (mvnormal.cpp:190) is not checked either
  __syncthreads();
  for (int e = threadIdx.x; e < K * K; e += blockDim.x) {
    const int i = e % K, j = e / K;
    L[e] = (i >= j) ? M[e] : 0.0;
  }
}

int grid_for(long long rows, int rows_per_block) {
  long long b = (rows + rows_per_block - 1) / rows_per_block;
  if (b > 148 * 16) b = 148 * 16;
  return (int)(b < 1 ? 1 : b);
}

int outer_blocks(long long nrow) {  // about two blocks per SM at the benchmark's 32,768 features
  long long b = (nrow + 63) / 64;
  if (b > 296) b = 296;
  return (int)(b < 1 ? 1 : b);
}

// The partials' sum in block order into `out` (the 1-CTA solves then read one record).
void sum_records(const double* parts, int nparts, int len, double* out, cudaStream_t s,
                 const uint32_t* done = nullptr) {
  k_sum_records<<<(len * 8 + 255) / 256, 256, 0, s>>>(parts, nparts, len, out, done);
  MG_CUDA(cudaGetLastError());
}

template <typename V, int NRP>
void outer(const V* A, const V* B, long long nrow, double* partials, int nb, cudaStream_t s,
           const uint32_t* done = nullptr) {
  const long long rpb = (nrow + nb - 1) / nb;
  k_outer<V, NRP><<<nb, kOuterThreads, 0, s>>>(A, B, NRP, nrow, rpb, partials, done);
  MG_CUDA(cudaGetLastError());
}

template <typename V, int NRP>
void spmm_t(const DevCsr& A, const V* src, int sstride, V* dst, int dstride, int ncomp,
            const V* add, int astride, double reg, const double* reg_dev, cudaStream_t s,
            const uint32_t* done = nullptr) {
  if (A.tasks) {
    k_spmm_split<V, NRP><<<grid_for(A.ntasks, 8), 256, 0, s>>>(
        A, src, sstride, dst, dstride, ncomp, add, astride, reg, reg_dev, done);
    MG_CUDA(cudaGetLastError());
    return;
  }
  k_spmm<V, NRP><<<grid_for(A.nrow, 8), 256, 0, s>>>(A.ptr, A.idx, A.val, A.valf, A.nrow, src,
                                                      sstride, dst, dstride, ncomp, add,
                                                      astride, reg, reg_dev, done);
  MG_CUDA(cudaGetLastError());
}

template <typename V, int NRP>
int cg_core(const DevCsr& F, const DevCsr& Ft, double reg, const double* reg_dev,
            const double* B, int bstride, int n, double tol, double* Xout, int xstride,
            Ctl* ctl, cudaStream_t s, V* R, V* P, V* KPm, V* inner, double* Xd, double* Bn,
            double* KX, double* innerd, double* small, double* partials, int* flag_dev,
            volatile int* flag_host, int max_iter, bool& converged) {
  const long long nfeat = Ft.nrow;
  const int nb = outer_blocks(nfeat);
  double* reduced = partials + (size_t)296 * 64 * 64;
  const int eg = grid_for(nfeat * NRP, 256);
  // Bn <- B padded to NRP columns, then the RHS norms from diag(B B^T)
  MG_CUDA(cudaMemcpy2DAsync(Bn, NRP * sizeof(double), B, bstride * sizeof(double),
                            n * sizeof(double), nfeat, cudaMemcpyDeviceToDevice, s));
  if (n < NRP)
    MG_CUDA(cudaMemset2DAsync(Bn + n, NRP * sizeof(double), 0, (NRP - n) * sizeof(double),
                              nfeat, s));
  outer<double, NRP>(Bn, Bn, nfeat, partials, nb, s);
  sum_records(partials, nb, NRP * NRP, reduced, s);
  k_cg_norms<<<1, 64, 0, s>>>(reduced, 1, NRP, n, small);
  MG_CUDA(cudaGetLastError());
  k_cg_init<V><<<eg, 256, 0, s>>>(Bn, NRP, nfeat, n, NRP, small, R, P, Xd,
                                  sizeof(V) == 4 ? Bn : nullptr, ctl);
  MG_CUDA(cudaGetLastError());
  outer<V, NRP>(R, R, nfeat, partials, nb, s);
  sum_records(partials, nb, NRP * NRP, reduced, s);
  k_cg_rtr<<<1, 256, 0, s>>>(reduced, 1, NRP, n, small);
  MG_CUDA(cudaGetLastError());
  const double tolsq = tol * tol;
  const int rg = (int)((nfeat + kRowTile - 1) / kRowTile);
  {
    static bool configured[64] = {false};
    int dev = 0;
    MG_CUDA(cudaGetDevice(&dev));
    if (!configured[dev & 63]) {
      MG_CUDA(cudaFuncSetAttribute(k_cg_rows<V, NRP, true>,
                                   cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)rows_smem(NRP, true)));
      MG_CUDA(cudaFuncSetAttribute(k_cg_rows<V, NRP, false>,
                                   cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)rows_smem(NRP, false)));
      configured[dev & 63] = true;
    }
  }
  // Iterations are queued kCgBatch at a time and the host reads the convergence flag between
  // batches; once k_cg_solve_psi has set ctl->cg_done, every later kernel of the batch returns
  // at once, so the result is that of stopping at the converged iteration.
  const uint32_t* done = &ctl->cg_done;
  int iter = 0;
  converged = false;
  while (iter < max_iter) {
    for (int b = 0; b < kCgBatch && iter < max_iter; b++, iter++) {
      spmm_t<V, NRP>(F, P, NRP, inner, NRP, n, nullptr, 0, 0.0, nullptr, s, done);
      spmm_t<V, NRP>(Ft, inner, NRP, KPm, NRP, n, P, NRP, reg, reg_dev, s, done);
      outer<V, NRP>(P, KPm, nfeat, partials, nb, s, done);
      sum_records(partials, nb, NRP * NRP, reduced, s, done);
      k_cg_solve_a<<<1, kSolveThreads, 0, s>>>(reduced, 1, NRP, n, small, ctl);
      MG_CUDA(cudaGetLastError());
      k_cg_rows<V, NRP, true><<<rg, 256, rows_smem(NRP, true), s>>>(nfeat, n, small, P, KPm, R,
                                                                    Xd, nullptr, done);
      MG_CUDA(cudaGetLastError());
      if (sizeof(V) == 4 && (iter + 1) % kReplaceEvery == 0) {
        spmm_t<double, NRP>(F, Xd, NRP, innerd, NRP, n, nullptr, 0, 0.0, nullptr, s, done);
        spmm_t<double, NRP>(Ft, innerd, NRP, KX, NRP, n, Xd, NRP, reg, reg_dev, s, done);
        k_cg_resid<V><<<eg, 256, 0, s>>>(nfeat * NRP, NRP, n, Bn, KX, R, done);
        MG_CUDA(cudaGetLastError());
      }
      outer<V, NRP>(R, R, nfeat, partials, nb, s, done);
      sum_records(partials, nb, NRP * NRP, reduced, s, done);
      k_cg_solve_psi<<<1, kSolveThreads, 0, s>>>(reduced, 1, NRP, n, tolsq, small, ctl, flag_dev,
                                                 iter);
      MG_CUDA(cudaGetLastError());
      k_cg_rows<V, NRP, false><<<rg, 256, rows_smem(NRP, false), s>>>(nfeat, n, small, P, nullptr,
                                                                       R, nullptr, P, done);
      MG_CUDA(cudaGetLastError());
    }
    MG_CUDA(cudaStreamSynchronize(s));
    if (flag_host[0]) {
      iter = flag_host[1];
      converged = true;
      break;
    }
  }
  k_cg_finish<<<grid_for(nfeat * n, 256), 256, 0, s>>>(nfeat, NRP, n, small, Xd, Xout, xstride);
  MG_CUDA(cudaGetLastError());
  return iter;
}

}  // namespace

void launch_spmm(const DevCsr& A, const void* src, int src_stride, void* dst, int dst_stride,
                 int ncomp, bool f32, cudaStream_t s) {
  if (ncomp > 64) throw MgError(MG_ERR_ARG, "spmm: more than 64 components");
  if (f32) {
    if (ncomp <= 32)
      spmm_t<float, 32>(A, (const float*)src, src_stride, (float*)dst, dst_stride, ncomp,
                        nullptr, 0, 0.0, nullptr, s);
    else
      spmm_t<float, 64>(A, (const float*)src, src_stride, (float*)dst, dst_stride, ncomp,
                        nullptr, 0, 0.0, nullptr, s);
  } else {
    if (ncomp <= 32)
      spmm_t<double, 32>(A, (const double*)src, src_stride, (double*)dst, dst_stride, ncomp,
                         nullptr, 0, 0.0, nullptr, s);
    else
      spmm_t<double, 64>(A, (const double*)src, src_stride, (double*)dst, dst_stride, ncomp,
                         nullptr, 0, 0.0, nullptr, s);
  }
}

void launch_beta_rhs_tmp(const void* U, bool f32, int ustride, long long N, int K,
                         const double* Lchol, const double* mu, const Ctl* ctl,
                         unsigned long long seed, int mode, double* tmp, int tstride,
                         cudaStream_t s) {
  const int g = grid_for(N, 128);
  if (f32)
    k_beta_tmp<float><<<g, 128, 0, s>>>((const float*)U, ustride, N, K, Lchol, mu, ctl, seed,
                                        mode, tmp, tstride);
  else
    k_beta_tmp<double><<<g, 128, 0, s>>>((const double*)U, ustride, N, K, Lchol, mu, ctl, seed,
                                         mode, tmp, tstride);
  MG_CUDA(cudaGetLastError());
}

void launch_beta_rhs_b(const DevCsr& Ft, const double* tmp, int tstride, int K,
                       const double* Lchol, const double* lambda_beta, const Ctl* ctl,
                       unsigned long long seed, int mode, double* B, int bstride,
                       cudaStream_t s) {
  // Ft_y = tmp * F (A_mul_B(tmp, F) -> csr_A_mul_Bn over the rows of F^T) ...
  launch_spmm(Ft, tmp, tstride, B, bstride, K, false, s);
  // ... + sqrt(lambda_beta) * MvNormal_prec_omp(Lambda, nfeat)
  k_beta_noise<<<grid_for(Ft.nrow, 128), 128, 0, s>>>(Ft.nrow, K, Lchol, lambda_beta, ctl, seed,
                                                      mode, B, bstride);
  MG_CUDA(cudaGetLastError());
}

void launch_small_chol(const double* A, int K, double* L, Ctl* ctl, cudaStream_t s) {
  k_small_chol<<<1, 64, 0, s>>>(A, K, L, ctl);
  MG_CUDA(cudaGetLastError());
}

void BlockCg::reserve(long long nrow, long long nfeat, int max_rhs, bool f32) {
  if (nrow <= nrow_ && nfeat <= nfeat_ && max_rhs <= maxr_ && f32 == f32_ && R_) return;
  release();
  nrow_ = nrow;
  nfeat_ = nfeat;
  maxr_ = max_rhs;
  f32_ = f32;
  const size_t es = f32 ? 4 : 8;
  const size_t NRP = 64;
  MG_CUDA(cudaMalloc(&R_, es * nfeat * NRP));
  MG_CUDA(cudaMalloc(&P_, es * nfeat * NRP));
  MG_CUDA(cudaMalloc(&KP_, es * nfeat * NRP));
  MG_CUDA(cudaMalloc(&inner_, es * nrow * NRP));
  MG_CUDA(cudaMalloc(&Xd_, 8 * nfeat * NRP));
  MG_CUDA(cudaMalloc(&Bn_, 8 * nfeat * NRP));
  if (f32) {
    MG_CUDA(cudaMalloc(&KX_, 8 * nfeat * NRP));
    MG_CUDA(cudaMalloc(&innerd_, 8 * nrow * NRP));
  }
  MG_CUDA(cudaMalloc(&small_, sizeof(double) * (5 * kSq + 256)));
  MG_CUDA(cudaMalloc(&partials_, sizeof(double) * 297 * 64 * 64));  // 296 partials + their sum
  MG_CUDA(cudaHostAlloc(&flag_host_, 2 * sizeof(int), cudaHostAllocMapped));  // done, iteration
}

void BlockCg::release() {
  for (void* p : {R_, P_, KP_, inner_, (void*)Xd_, (void*)Bn_, (void*)KX_, (void*)innerd_,
                  (void*)small_, (void*)partials_})
    if (p) cudaFree(p);
  if (flag_host_) cudaFreeHost(flag_host_);
  R_ = P_ = KP_ = inner_ = nullptr;
  Xd_ = Bn_ = KX_ = innerd_ = small_ = partials_ = nullptr;
  flag_host_ = nullptr;
  nrow_ = nfeat_ = 0;
  maxr_ = 0;
}

int BlockCg::core(const DevCsr& F, const DevCsr& Ft, double reg, const double* reg_dev,
                  const double* B, int bstride, int n, double tol, double* X, int xstride,
                  Ctl* ctl, cudaStream_t s, bool f32) {
  int* flag_dev = nullptr;
  MG_CUDA(cudaHostGetDevicePointer((void**)&flag_dev, flag_host_, 0));
  flag_host_[0] = 0;
  flag_host_[1] = 0;
  if (f32) {
    if (n <= 32)
      return cg_core<float, 32>(F, Ft, reg, reg_dev, B, bstride, n, tol, X, xstride, ctl, s,
                                (float*)R_, (float*)P_, (float*)KP_, (float*)inner_, Xd_, Bn_,
                                KX_, innerd_, small_, partials_, flag_dev, flag_host_,
                                max_iter_, last_converged_);
    return cg_core<float, 64>(F, Ft, reg, reg_dev, B, bstride, n, tol, X, xstride, ctl, s,
                              (float*)R_, (float*)P_, (float*)KP_, (float*)inner_, Xd_, Bn_,
                              KX_, innerd_, small_, partials_, flag_dev, flag_host_,
                              max_iter_, last_converged_);
  }
  if (n <= 32)
    return cg_core<double, 32>(F, Ft, reg, reg_dev, B, bstride, n, tol, X, xstride, ctl, s,
                               (double*)R_, (double*)P_, (double*)KP_, (double*)inner_, Xd_,
                               Bn_, KX_, innerd_, small_, partials_, flag_dev, flag_host_,
                               max_iter_, last_converged_);
  return cg_core<double, 64>(F, Ft, reg, reg_dev, B, bstride, n, tol, X, xstride, ctl, s,
                             (double*)R_, (double*)P_, (double*)KP_, (double*)inner_, Xd_, Bn_,
                             KX_, innerd_, small_, partials_, flag_dev, flag_host_,
                             max_iter_, last_converged_);
}

int BlockCg::solve(const DevCsr& F, const DevCsr& Ft, double reg, const double* reg_dev,
                   const double* B, int bstride, int nrhs, double tol, double* X, int xstride,
                   Ctl* ctl, cudaStream_t s, bool f32) {
  // solve_blockcg(X, K, reg, B, tol, 32, 8) (linop.h:207-226), including the reference's
  // overlapping extra block when a remainder block is followed by one more start index.
  const int blocksize = 32, excess = 8;
  reserve(F.nrow, Ft.nrow, 64, f32);
  if (nrhs <= excess + blocksize) {
    const int it = core(F, Ft, reg, reg_dev, B, bstride, nrhs, tol, X, xstride, ctl, s, f32);
    converged_ = last_converged_;
    return it;
  }
  int total = 0;
  converged_ = true;
  for (int i = 0; i < nrhs; i += blocksize) {
    int nr = blocksize;
    if (i + blocksize + excess >= nrhs) nr = nrhs - i;
    total += core(F, Ft, reg, reg_dev, B + i, bstride, nr, tol, X + i, xstride, ctl, s, f32);
    converged_ = converged_ && last_converged_;
  }
  return total;
}

}  // namespace mg
