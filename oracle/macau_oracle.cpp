// TEST INFRASTRUCTURE ONLY.  This is the CPU oracle (checker) for the Macau Gibbs-sweep hot path:
// a plain C++17 + OpenMP FP64 restatement of jaak-s/macau 0.5.3, with every random draw taken
// from the keyed Philox stream in oracle_rng.h so the CUDA library can be compared draw for draw.
// Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline / reference arm load it.
//
// What it restates (reference file:line, paths inside the reference project):
//   sample_latent_blas ............ lib/macau-cpp/latentprior.cpp:361-385
//   BPMF/Macau row loops .......... lib/macau-cpp/latentprior.cpp:69-77, 219-227
//   CondNormalWishart chain ....... lib/macau-cpp/mvnormal.cpp:169-184, 217-287, 314-336
//   MacauPrior::update_prior ...... lib/macau-cpp/latentprior.cpp:255-264
//   MacauPrior::sample_beta ....... lib/macau-cpp/latentprior.cpp:273-293 (block-CG branch)
//   posterior/sample_lambda_beta .. lib/macau-cpp/latentprior.cpp:317-331
//   solve_blockcg (+ blocking) .... lib/macau-cpp/linop.h:207-343
//   A_mul_Bx / AtA_mul_Bx ......... lib/macau-cpp/linop.h:345-403, 469-535
//   compute_uhat / A_mul_B(F) ..... lib/macau-cpp/linop.h:192-198, latentprior.cpp:431-435,
//                                   linop.cpp:37-57 (libfastsparse csr_A_mul_Bn restated as the
//                                   plain CSR row loop)
//   eval_rmse ..................... lib/macau-cpp/bpmfutils.h:86-114
//   AdaptiveGaussianNoise ......... lib/macau-cpp/noisemodels.cpp:14-33 (init), 55-81 (update)
//   MacauOnePrior (univariate) .... lib/macau-cpp/macauoneprior.cpp:16-39 (init), 41-95 (row
//                                   sampler), 189-257 (mu/lambda, beta), 267-290 (lambda_beta);
//                                   linop.cpp:374-401 (col_square_sum), linop.h:121-178
//   MacauX::run sweep body ........ lib/macau-cpp/macau.cpp:110-147
// Eigen 3.3.7 (LLT, triangular solves, inverse) is not in the reference tree; its operations are
// restated as textbook left-looking Cholesky and substitution.  X.inverse() (mvnormal.cpp:326),
// an LU inverse in Eigen, is computed here through the Cholesky factor of the SPD matrix X.
#include <omp.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include "oracle_rng.h"

using namespace oracle;

namespace {

// ---------- dense helpers (column-major, K x K) ----------

// In-place lower Cholesky (left-looking).  Returns false when a pivot is not positive.
bool chol_lower(double* A, int n) {
  for (int j = 0; j < n; j++) {
    double d = A[j + j * n];
    for (int p = 0; p < j; p++) d -= A[j + p * n] * A[j + p * n];
    if (!(d > 0.0)) return false;
    const double ljj = std::sqrt(d);
    A[j + j * n] = ljj;
    for (int i = j + 1; i < n; i++) {
      double s = A[i + j * n];
      for (int p = 0; p < j; p++) s -= A[i + p * n] * A[j + p * n];
      A[i + j * n] = s / ljj;
    }
    for (int i = 0; i < j; i++) A[i + j * n] = 0.0;  // keep only the factor
  }
  return true;
}

// Solve L x = b in place (L lower, column-major).
void solve_lower(const double* L, double* x, int n) {
  for (int i = 0; i < n; i++) {
    double s = x[i];
    for (int p = 0; p < i; p++) s -= L[i + p * n] * x[p];
    x[i] = s / L[i + i * n];
  }
}

// Solve L^T x = b in place.
void solve_upper_t(const double* L, double* x, int n) {
  for (int i = n - 1; i >= 0; i--) {
    double s = x[i];
    for (int p = i + 1; p < n; p++) s -= L[p + i * n] * x[p];
    x[i] = s / L[i + i * n];
  }
}

// ---------- sparse helpers ----------

struct Csr {
  const int64_t* ptr;
  const int32_t* idx;
  const double* val;  // nullptr => binary (all ones)
  int nrow;
  int ncol;
};

// out[:, r] = sum_{i in row r} val_i * B[:, idx_i]      (B: N x ncol, out: N x nrow)
// This is csr_A_mul_Bn(out, csr, B, N) as used by A_mul_Bt (linop.cpp:37-57) and A_mul_Bx<N>
// (linop.h:345-403) -- both compute one N-vector per CSR row.
void csr_mul_bn(const Csr& A, const double* B, int N, double* out) {
#pragma omp parallel for schedule(dynamic, 256)
  for (int r = 0; r < A.nrow; r++) {
    std::vector<double> tmp(N, 0.0);
    for (int64_t i = A.ptr[r]; i < A.ptr[r + 1]; i++) {
      const double* x = B + (int64_t)A.idx[i] * N;
      if (A.val) {
        const double v = A.val[i];
        for (int j = 0; j < N; j++) tmp[j] += x[j] * v;
      } else {
        for (int j = 0; j < N; j++) tmp[j] += x[j];
      }
    }
    for (int j = 0; j < N; j++) out[(int64_t)r * N + j] = tmp[j];
  }
}

// out = (F^T F B^T)^T + reg * B  (linop.h:469-535): inner = F * B^T, then out = Ft * inner + reg B.
void ata_mul_bx(const Csr& F, const Csr& Ft, double reg, const double* B, int N, double* out,
                double* inner) {
  csr_mul_bn(F, B, N, inner);
#pragma omp parallel for schedule(dynamic, 256)
  for (int r = 0; r < Ft.nrow; r++) {
    std::vector<double> tmp(N, 0.0);
    for (int64_t i = Ft.ptr[r]; i < Ft.ptr[r + 1]; i++) {
      const double* x = inner + (int64_t)Ft.idx[i] * N;
      if (Ft.val) {
        const double v = Ft.val[i];
        for (int j = 0; j < N; j++) tmp[j] += x[j] * v;
      } else {
        for (int j = 0; j < N; j++) tmp[j] += x[j];
      }
    }
    for (int j = 0; j < N; j++)
      out[(int64_t)r * N + j] = tmp[j] + reg * B[(int64_t)r * N + j];
  }
}

// Number of partial sums of the K x K reductions.  The reference accumulates one partial per
// OpenMP thread over contiguous column ranges and adds the partials in thread order
// (A_mul_At_omp / A_mul_Bt_omp_sym, linop.cpp:280-317, 332-371), so its summation order depends
// on the thread count; the oracle takes the count as a parameter (1 = one sequential sum).
static int g_reduce_parts = 1;

// Lower triangle of A * B^T for n x k column-major A, B (A_mul_Bt_omp_sym, linop.cpp:320-372;
// A_mul_At_omp, linop.cpp:271-318), then mirrored to the upper triangle when `sym`.  Partial
// sums over g_reduce_parts contiguous chunks of ceil(k / parts) columns, added in chunk order.
void a_mul_bt_lower(const double* A, const double* B, int n, int k, double* out, bool sym) {
  std::vector<double> acc((size_t)n * n, 0.0), part((size_t)n * n);
  const int parts = std::max(1, g_reduce_parts);
  const int64_t chunk = ((int64_t)k + parts - 1) / parts;
  for (int q = 0; q < parts; q++) {
    std::fill(part.begin(), part.end(), 0.0);
    const int64_t c1 = std::min<int64_t>(k, (q + 1) * chunk);
    for (int64_t c = q * chunk; c < c1; c++) {
      const double* a = A + c * n;
      const double* b = B + c * n;
      for (int i = 0; i < n; i++)
        for (int j = i; j < n; j++) part[j + (size_t)i * n] += a[j] * b[i];
    }
    for (size_t t = 0; t < acc.size(); t++) acc[t] += part[t];
  }
  for (int i = 0; i < n; i++)
    for (int j = 0; j < n; j++) {
      if (j >= i) out[j + (size_t)i * n] = acc[j + (size_t)i * n];
      else if (sym) out[j + (size_t)i * n] = acc[i + (size_t)j * n];
    }
}

// X = L^{-T} L^{-1} B  (Eigen LLT::solve), n x n L, B n x m.
void llt_solve(const double* L, const double* B, int n, int m, double* X) {
  std::memcpy(X, B, sizeof(double) * (size_t)n * m);
  for (int c = 0; c < m; c++) {
    solve_lower(L, X + (size_t)c * n, n);
    solve_upper_t(L, X + (size_t)c * n, n);
  }
}

void transpose_sq(double* A, int n) {
  for (int i = 0; i < n; i++)
    for (int j = i + 1; j < n; j++) std::swap(A[i + j * n], A[j + i * n]);
}

}  // namespace

// ======================= exported building blocks =======================
extern "C" {

void orc_philox(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) {
  philox4x32_10(ctr, key, out);
}

double orc_normal(uint64_t seed, uint32_t sweep, uint32_t stream, uint32_t index, uint32_t j) {
  return normal_draw(seed, sweep, stream, index, j);
}

double orc_gamma(uint64_t seed, uint32_t sweep, uint32_t stream, uint32_t index, double shape) {
  return gamma_draw(seed, sweep, stream, index, shape);
}

// Sets the number of partial sums of the K x K reductions (see g_reduce_parts); returns it.
int orc_set_reduce_parts(int parts) {
  if (parts > 0) g_reduce_parts = parts;
  return g_reduce_parts;
}

int orc_set_threads(int n) {
  if (n > 0) omp_set_num_threads(n);
  return omp_get_max_threads();
}

// sample_latent_blas for every row of `R` (latentprior.cpp:361-385 inside the OpenMP row loops
// latentprior.cpp:69-77 / 219-227).  R: CSR of the rows being sampled (column indices into
// `other`), other: K x ncol, mu: K, Lambda: K x K, Uhat: K x nrow or null (Macau prior mean
// mu + Uhat[:, n]).  z: optional K x nrow standard normals; when null the keyed draws
// (purpose kRowNoise, index n) are used.  Returns 0, or -1 when a Cholesky factorisation fails
// ("Cholesky Decomposition failed!", latentprior.cpp:374-376).
// Rows lo .. hi - 1 of the sampler below (the draws keyed by the global row index n).
static int sample_latent_rows(int K, int lo, int hi, const int64_t* ptr, const int32_t* idx,
                              const double* val, double mean_rating, const double* other,
                              double alpha, const double* mu, const double* Lambda,
                              const double* Uhat, uint64_t seed, uint32_t sweep, uint32_t mode,
                              const double* z, double* U_out) {
  int failed = 0;
#pragma omp parallel for schedule(dynamic, 2)
  for (int n = lo; n < hi; n++) {
    std::vector<double> MM(Lambda, Lambda + (size_t)K * K);
    std::vector<double> rr(K, 0.0), mun(K);
    for (int64_t e = ptr[n]; e < ptr[n + 1]; e++) {
      const double* col = other + (int64_t)idx[e] * K;
      for (int j = 0; j < K; j++) {
        for (int i = j; i < K; i++) MM[i + j * K] += (alpha * col[i]) * col[j];
      }
      const double w = (val[e] - mean_rating) * alpha;
      for (int i = 0; i < K; i++) rr[i] += col[i] * w;
    }
    if (!chol_lower(MM.data(), K)) {
#pragma omp atomic write
      failed = 1;
      continue;
    }
    for (int i = 0; i < K; i++) mun[i] = mu[i] + (Uhat ? Uhat[(int64_t)n * K + i] : 0.0);
    for (int i = 0; i < K; i++) {
      double s = 0.0;
      for (int j = 0; j < K; j++) s += Lambda[i + j * K] * mun[j];
      rr[i] += s;
    }
    solve_lower(MM.data(), rr.data(), K);
    for (int i = 0; i < K; i++)
      rr[i] += z ? z[(int64_t)n * K + i]
                 : normal_draw(seed, sweep, stream_id(kRowNoise, mode), (uint32_t)n, (uint32_t)i);
    solve_upper_t(MM.data(), rr.data(), K);
    for (int i = 0; i < K; i++) U_out[(int64_t)n * K + i] = rr[i];
  }
  return failed ? -1 : 0;
}

int orc_sample_latents(int K, int nrow, int ncol, const int64_t* ptr, const int32_t* idx,
                       const double* val, double mean_rating, const double* other, double alpha,
                       const double* mu, const double* Lambda, const double* Uhat,
                       uint64_t seed, uint32_t sweep, uint32_t mode, const double* z,
                       double* U_out) {
  (void)ncol;
  return sample_latent_rows(K, 0, nrow, ptr, idx, val, mean_rating, other, alpha, mu, Lambda,
                            Uhat, seed, sweep, mode, z, U_out);
}

// CondNormalWishart(U, mu, kappa, T, nu) (mvnormal.cpp:314-336) followed by NormalWishart /
// Wishart / WishartUnit / MvNormal_prec (mvnormal.cpp:169-184, 217-287).  Draws: Bartlett
// diagonal Gamma(0.5*(nu_c - i)) at (kWishartDiag, i); off-diagonal c(i, j>i) N(0,1) at
// (kWishartOff, i, j-i-1); mean draw at (kMuDraw, 0, k).  Returns 0 or -1 on a failed
// factorisation.
int orc_cond_normal_wishart(int K, int N, const double* U, const double* mu0, double kappa,
                            const double* T, int nu, uint64_t seed, uint32_t sweep, uint32_t mode,
                            double* mu_out, double* Lambda_out) {
  std::vector<double> NU(K, 0.0), NS((size_t)K * K, 0.0);
  for (int64_t n = 0; n < N; n++) {
    const double* u = U + n * K;
    for (int i = 0; i < K; i++) NU[i] += u[i];
    for (int j = 0; j < K; j++)
      for (int i = 0; i < K; i++) NS[i + j * K] += u[i] * u[j];
  }
  const int nu_c = nu + N;
  const double kappa_c = kappa + N;
  std::vector<double> mu_c(K), X((size_t)K * K);
  for (int i = 0; i < K; i++) mu_c[i] = (kappa * mu0[i] + NU[i]) / (kappa + N);
  for (int j = 0; j < K; j++)
    for (int i = 0; i < K; i++)
      X[i + j * K] = T[i + j * K] + NS[i + j * K] + kappa * mu0[i] * mu0[j] -
                     kappa_c * mu_c[i] * mu_c[j];
  // T_c = X^{-1} through X = L L^T.
  if (!chol_lower(X.data(), K)) return -1;
  std::vector<double> Tc((size_t)K * K, 0.0), e(K);
  for (int c = 0; c < K; c++) {
    std::fill(e.begin(), e.end(), 0.0);
    e[c] = 1.0;
    solve_lower(X.data(), e.data(), K);
    solve_upper_t(X.data(), e.data(), K);
    for (int i = 0; i < K; i++) Tc[i + c * K] = e[i];
  }
  // Wishart(T_c, nu_c): L = chol(T_c), Lambda = L (c^T c) L^T with Bartlett c (upper).
  std::vector<double> L = Tc;
  if (!chol_lower(L.data(), K)) return -1;
  std::vector<double> c((size_t)K * K, 0.0);
  for (int i = 0; i < K; i++) {
    c[i + i * K] = std::sqrt(2.0 * gamma_draw(seed, sweep, stream_id(kWishartDiag, mode),
                                              (uint32_t)i, 0.5 * (double)(nu_c - i)));
    for (int j = i + 1; j < K; j++)
      c[i + j * K] = normal_draw(seed, sweep, stream_id(kWishartOff, mode), (uint32_t)i,
                                 (uint32_t)(j - i - 1));
  }
  // W = c^T c, M = L W, Lambda = M L^T
  std::vector<double> W((size_t)K * K, 0.0), M((size_t)K * K, 0.0);
  for (int j = 0; j < K; j++)
    for (int i = 0; i < K; i++) {
      double s = 0.0;
      for (int p = 0; p < K; p++) s += c[p + i * K] * c[p + j * K];
      W[i + j * K] = s;
    }
  for (int j = 0; j < K; j++)
    for (int i = 0; i < K; i++) {
      double s = 0.0;
      for (int p = 0; p < K; p++) s += L[i + p * K] * W[p + j * K];
      M[i + j * K] = s;
    }
  for (int j = 0; j < K; j++)
    for (int i = 0; i < K; i++) {
      double s = 0.0;
      for (int p = 0; p < K; p++) s += M[i + p * K] * L[j + p * K];
      Lambda_out[i + j * K] = s;
    }
  // mu = mu_c + chol(kappa_c * Lambda).U^{-1} z
  std::vector<double> KL((size_t)K * K);
  for (size_t t = 0; t < KL.size(); t++) KL[t] = Lambda_out[t] * kappa_c;
  if (!chol_lower(KL.data(), K)) return -1;
  std::vector<double> z(K);
  for (int i = 0; i < K; i++)
    z[i] = normal_draw(seed, sweep, stream_id(kMuDraw, mode), 0u, (uint32_t)i);
  solve_upper_t(KL.data(), z.data(), K);
  for (int i = 0; i < K; i++) mu_out[i] = z[i] + mu_c[i];
  return 0;
}

// A_mul_Bx<N>(out, A, B) (linop.h:345-403): out[:, r] = sum val * B[:, col].
void orc_csr_mul_bn(int nrow, int ncol, const int64_t* ptr, const int32_t* idx, const double* val,
                    const double* B, int N, double* out) {
  Csr A{ptr, idx, val, nrow, ncol};
  csr_mul_bn(A, B, N, out);
}

// AtA_mul_Bx<N>(out, F, reg, B, inner) (linop.h:469-535).
void orc_ata_mul_bx(int nrow, int ncol, const int64_t* fptr, const int32_t* fidx,
                    const double* fval, const int64_t* tptr, const int32_t* tidx,
                    const double* tval, double reg, const double* B, int N, double* out) {
  Csr F{fptr, fidx, fval, nrow, ncol}, Ft{tptr, tidx, tval, ncol, nrow};
  std::vector<double> inner((size_t)nrow * N);
  ata_mul_bx(F, Ft, reg, B, N, out, inner.data());
}

// solve_blockcg core (linop.h:229-343) on nrhs right-hand sides.  Returns the iteration count.
int orc_blockcg_core(int nrhs, int nrow, int nfeat, const int64_t* fptr, const int32_t* fidx,
                     const double* fval, const int64_t* tptr, const int32_t* tidx,
                     const double* tval, double reg, const double* B, double tol, double* X) {
  Csr F{fptr, fidx, fval, nrow, nfeat}, Ft{tptr, tidx, tval, nfeat, nrow};
  const double tolsq = tol * tol;
  const size_t sz = (size_t)nrhs * nfeat;
  std::vector<double> norms(nrhs), inorms(nrhs);
  {
    std::vector<double> BBt((size_t)nrhs * nrhs);
    a_mul_bt_lower(B, B, nrhs, nfeat, BBt.data(), false);
    for (int r = 0; r < nrhs; r++) {
      norms[r] = std::sqrt(BBt[r + (size_t)r * nrhs]);
      inorms[r] = 1.0 / norms[r];
    }
  }
  std::vector<double> R(sz), P(sz), KP(sz), inner((size_t)nrow * nrhs);
  std::fill(X, X + sz, 0.0);
  for (int f = 0; f < nfeat; f++)
    for (int r = 0; r < nrhs; r++) {
      R[r + (size_t)f * nrhs] = B[r + (size_t)f * nrhs] * inorms[r];
      P[r + (size_t)f * nrhs] = R[r + (size_t)f * nrhs];
    }
  const int n = nrhs;
  std::vector<double> RtR((size_t)n * n), RtR2((size_t)n * n), PtKP((size_t)n * n),
      A((size_t)n * n), Psi((size_t)n * n), Lc((size_t)n * n), tmp(n);
  a_mul_bt_lower(R.data(), R.data(), n, nfeat, RtR.data(), true);
  int iter = 0;
  for (iter = 0; iter < 100000; iter++) {
    ata_mul_bx(F, Ft, reg, P.data(), n, KP.data(), inner.data());
    a_mul_bt_lower(P.data(), KP.data(), n, nfeat, PtKP.data(), false);
    Lc = PtKP;
    chol_lower(Lc.data(), n);  // Eigen's llt() result is used without an info() check
    llt_solve(Lc.data(), RtR.data(), n, n, A.data());
    transpose_sq(A.data(), n);
#pragma omp parallel for schedule(static) firstprivate(tmp)
    for (int f = 0; f < nfeat; f++) {
      double* x = X + (size_t)f * n;
      double* r = R.data() + (size_t)f * n;
      const double* p = P.data() + (size_t)f * n;
      const double* kp = KP.data() + (size_t)f * n;
      for (int i = 0; i < n; i++) {
        double sx = 0.0, sr = 0.0;
        for (int k = 0; k < n; k++) {
          sx += A[i + (size_t)k * n] * p[k];
          sr += A[i + (size_t)k * n] * kp[k];
        }
        x[i] += sx;
        tmp[i] = sr;
      }
      for (int i = 0; i < n; i++) r[i] -= tmp[i];
    }
    a_mul_bt_lower(R.data(), R.data(), n, nfeat, RtR2.data(), true);
    bool done = true;
    for (int i = 0; i < n; i++) done = done && (RtR2[i + (size_t)i * n] < tolsq);
    if (done) break;
    Lc = RtR;
    chol_lower(Lc.data(), n);
    llt_solve(Lc.data(), RtR2.data(), n, n, Psi.data());
    transpose_sq(Psi.data(), n);
#pragma omp parallel for schedule(static) firstprivate(tmp)
    for (int f = 0; f < nfeat; f++) {
      double* p = P.data() + (size_t)f * n;
      const double* r = R.data() + (size_t)f * n;
      for (int i = 0; i < n; i++) {
        double s = 0.0;
        for (int k = 0; k < n; k++) s += Psi[i + (size_t)k * n] * p[k];
        tmp[i] = r[i] + s;
      }
      for (int i = 0; i < n; i++) p[i] = tmp[i];
    }
    std::swap(RtR, RtR2);
  }
  for (int f = 0; f < nfeat; f++)
    for (int r = 0; r < nrhs; r++) X[r + (size_t)f * nrhs] *= norms[r];
  return iter;
}

// Blocked wrapper solve_blockcg(X, K, reg, B, tol, blocksize, excess) (linop.h:207-226).
// Returns the sum of the iteration counts of the blocks.
int orc_blockcg(int nrhs, int nrow, int nfeat, const int64_t* fptr, const int32_t* fidx,
                const double* fval, const int64_t* tptr, const int32_t* tidx, const double* tval,
                double reg, const double* B, double tol, int blocksize, int excess, double* X) {
  if (nrhs <= excess + blocksize)
    return orc_blockcg_core(nrhs, nrow, nfeat, fptr, fidx, fval, tptr, tidx, tval, reg, B, tol,
                            X);
  int total = 0;
  for (int i = 0; i < nrhs; i += blocksize) {
    int nr = blocksize;
    if (i + blocksize + excess >= nrhs) nr = nrhs - i;
    std::vector<double> Bb((size_t)nr * nfeat), Xb((size_t)nr * nfeat);
    for (int f = 0; f < nfeat; f++)
      for (int r = 0; r < nr; r++) Bb[r + (size_t)f * nr] = B[i + r + (size_t)f * nrhs];
    total += orc_blockcg_core(nr, nrow, nfeat, fptr, fidx, fval, tptr, tidx, tval, reg,
                              Bb.data(), tol, Xb.data());
    for (int f = 0; f < nfeat; f++)
      for (int r = 0; r < nr; r++) X[i + r + (size_t)f * nrhs] = Xb[r + (size_t)f * nr];
    // No early exit: like the reference loop, when excess > 0 a remainder block can be followed
    // by one more (overlapping) block whose rows are solved again.
  }
  return total;
}

// posterior_lambda_beta (latentprior.cpp:317-326).
void orc_posterior_lambda_beta(int K, int nfeat, const double* beta, const double* Lambda,
                               double nu, double mu, double* b_out, double* c_out) {
  std::vector<double> BB((size_t)K * K);
  a_mul_bt_lower(beta, beta, K, nfeat, BB.data(), true);
  double tr = 0.0;
  for (int i = 0; i < K; i++)
    for (int j = 0; j < K; j++) tr += BB[i + (size_t)j * K] * Lambda[j + (size_t)i * K];
  const double nux = nu + (double)K * nfeat;
  const double mux = mu * nux / (nu + mu * tr);
  *b_out = nux / 2;
  *c_out = 2 * mux / nux;
}

// eval_rmse (bpmfutils.h:86-114).  Test entries are given in the order of the CSC storage of
// Ytest (column-major), which is also the order of predictions / predictions_var.
void orc_eval_rmse(int ntest, const int32_t* rows, const int32_t* cols, const double* vals, int n,
                   double* pred, double* pred_var, const double* V, const double* U, int K,
                   double mean_rating, double* rmse_out, double* rmse_avg_out) {
  double se = 0.0, se_avg = 0.0;
#pragma omp parallel for schedule(static) reduction(+ : se, se_avg)
  for (int t = 0; t < ntest; t++) {
    const double* v = V + (int64_t)cols[t] * K;
    const double* u = U + (int64_t)rows[t] * K;
    double dot = 0.0;
    for (int k = 0; k < K; k++) dot += v[k] * u[k];
    const double p = dot + mean_rating;
    se += (vals[t] - p) * (vals[t] - p);
    double pavg;
    if (n == 0) {
      pavg = p;
    } else {
      const double delta = p - pred[t];
      pavg = pred[t] + delta / (n + 1);
      pred_var[t] += delta * (p - pavg);
    }
    se_avg += (vals[t] - pavg) * (vals[t] - pavg);
    pred[t] = pavg;
  }
  *rmse_out = std::sqrt(se / ntest);
  *rmse_avg_out = std::sqrt(se_avg / ntest);
}

}  // extern "C"

// ======================= whole-sweep model =======================
namespace {

struct Prior {
  bool macau = false;
  std::vector<double> mu, Lambda, WI, mu0;
  double b0 = 2.0;
  int df = 0;
  // side information (MacauPrior<SparseDoubleFeat>, latentprior.cpp:179-216)
  Csr F{}, Ft{};
  int nfeat = 0;
  std::vector<double> Uhat, beta;
  double lambda_beta = 5.0, lb_mu0 = 1.0, lb_nu0 = 1e-3, tol = 1e-6;
  int cg_iters = 0;
  // MacauOnePrior (macauoneprior.h:8-51): per-dimension precisions lambda = diag(Lambda) and
  // lambda_beta, the squared column norms of F, and the Gamma hyperprior of lambda_beta
  bool one = false;
  std::vector<double> lb_one, colsq;
  double lb_a0 = 0.1, lb_b0 = 0.1;
};

struct Model {
  int K = 0;
  double alpha = 1.0;
  uint64_t seed = 0;
  int dims[2] = {0, 0};
  Csr Y[2]{};  // Y[0]: CSR of rows of Y (cols idx), Y[1]: CSR of columns of Y (row idx)
  double mean = 0.0;
  std::vector<double> lat[2];
  Prior prior[2];
  int ntest = 0;
  const int32_t *trow = nullptr, *tcol = nullptr;
  const double* tval = nullptr;
  std::vector<double> pred, pred_var;
  double rmse = NAN, rmse1 = NAN;
  // AdaptiveGaussianNoise (noisemodels.h:50-86); alpha above is its current precision
  bool adaptive = false;
  double var_total = 1.0, alpha_max = 0.0;
};

void init_prior(Prior& p, int K) {  // BPMFPrior::init / MacauPrior::init (latentprior.cpp:84-99)
  p.mu.assign(K, 0.0);
  p.Lambda.assign((size_t)K * K, 0.0);
  p.WI.assign((size_t)K * K, 0.0);
  for (int i = 0; i < K; i++) {
    p.Lambda[i + (size_t)i * K] = 10.0;
    p.WI[i + (size_t)i * K] = 1.0;
  }
  p.mu0.assign(K, 0.0);
  p.b0 = 2.0;
  p.df = K;
}

// MacauOnePrior::sample_latents (macauoneprior.cpp:41-95): per row, the coordinates are
// resampled one after another, u_d ~ N(L_d / Q_d, 1 / Q_d) with Q_d = lambda_d + alpha sum v_d^2
// and L_d = lambda_d (mu_d + Uhat_d) + alpha sum (y - (yhat - u_d v_d)) v_d, where yhat keeps the
// row's predictions under the coordinates updated so far.  The normals are the row sampler's
// keyed draws (kRowNoise, row, d).
int sample_mode_one(Model& m, int mode, int iter) {
  Prior& p = m.prior[mode];
  const int other = 1 - mode;
  const Csr& R = m.Y[mode];
  const int K = m.K;
  double* U = m.lat[mode].data();
  const double* V = m.lat[other].data();
  const double alpha = m.alpha;
#pragma omp parallel for schedule(dynamic, 4)
  for (int i = 0; i < R.nrow; i++) {
    const int64_t b = R.ptr[i], n = R.ptr[i + 1] - b;
    std::vector<double> yhat(n), Q(K);
    double* u = U + (size_t)i * K;
    for (int d = 0; d < K; d++) Q[d] = p.Lambda[d + (size_t)d * K];
    for (int64_t e = 0; e < n; e++) {
      const double* v = V + (size_t)R.idx[b + e] * K;
      double dot = 0.0;
      for (int d = 0; d < K; d++) {
        Q[d] += alpha * (v[d] * v[d]);
        dot += u[d] * v[d];
      }
      yhat[e] = m.mean + dot;
    }
    for (int d = 0; d < K; d++) {
      const double z = normal_draw(m.seed, (uint32_t)iter, stream_id(kRowNoise, (uint32_t)mode),
                                   (uint32_t)i, (uint32_t)d);
      const double uid = u[d];
      double L = p.Lambda[d + (size_t)d * K] * (p.mu[d] + p.Uhat[(size_t)i * K + d]);
      for (int64_t e = 0; e < n; e++) {
        const double vjd = V[(size_t)R.idx[b + e] * K + d];
        L += alpha * (R.val[b + e] - (yhat[e] - uid * vjd)) * vjd;
      }
      const double var = 1.0 / Q[d];
      u[d] = L * var + std::sqrt(var) * z;
      const double delta = u[d] - uid;
      for (int64_t e = 0; e < n; e++) yhat[e] += delta * V[(size_t)R.idx[b + e] * K + d];
    }
  }
  return 0;
}

int sample_mode(Model& m, int mode, int iter) {
  Prior& p = m.prior[mode];
  if (p.one) return sample_mode_one(m, mode, iter);
  const int other = 1 - mode;
  const Csr& R = m.Y[mode];
  return orc_sample_latents(m.K, R.nrow, R.ncol, R.ptr, R.idx, R.val, m.mean,
                            m.lat[other].data(), m.alpha, p.mu.data(), p.Lambda.data(),
                            p.macau ? p.Uhat.data() : nullptr, m.seed, (uint32_t)iter,
                            (uint32_t)mode, nullptr, m.lat[mode].data());
}

// MacauPrior::sample_beta (latentprior.cpp:273-293), block-CG branch.
int sample_beta(Model& m, Prior& p, const std::vector<double>& U, int mode, int iter) {
  const int K = m.K, N = p.F.nrow, nF = p.nfeat;
  std::vector<double> Lc = p.Lambda;
  chol_lower(Lc.data(), K);
  std::vector<double> tmp((size_t)K * N), Fty((size_t)K * nF);
#pragma omp parallel for schedule(static)
  for (int n = 0; n < N; n++) {
    double z[256];
    for (int i = 0; i < K; i++)
      z[i] = normal_draw(m.seed, (uint32_t)iter, stream_id(kMvnN, (uint32_t)mode), (uint32_t)n,
                         (uint32_t)i);
    solve_upper_t(Lc.data(), z, K);
    for (int i = 0; i < K; i++)
      tmp[(size_t)n * K + i] = (U[(size_t)n * K + i] + z[i]) - p.mu[i];
  }
  csr_mul_bn(p.Ft, tmp.data(), K, Fty.data());
  const double slb = std::sqrt(p.lambda_beta);
#pragma omp parallel for schedule(static)
  for (int f = 0; f < nF; f++) {
    double z[256];
    for (int i = 0; i < K; i++)
      z[i] = normal_draw(m.seed, (uint32_t)iter, stream_id(kMvnF, (uint32_t)mode), (uint32_t)f,
                         (uint32_t)i);
    solve_upper_t(Lc.data(), z, K);
    for (int i = 0; i < K; i++) Fty[(size_t)f * K + i] += slb * z[i];
  }
  p.cg_iters = orc_blockcg(K, N, nF, p.F.ptr, p.F.idx, p.F.val, p.Ft.ptr, p.Ft.idx, p.Ft.val,
                           p.lambda_beta, Fty.data(), p.tol, 32, 8, p.beta.data());
  return 0;
}

// MacauOnePrior::update_prior (macauoneprior.cpp:189-290): sample_mu_lambda (Normal-Wishart
// of U - Uhat with mu0 = 0, kappa = 2, W = I, nu = K; lambda = diag Lambda), sample_beta (each
// link coefficient in turn, features in order within blocks of four dimensions, with the
// residual Z = U - mu - F beta kept current), compute_uhat, sample_lambda_beta (one Gamma per
// dimension, keyed (kLambdaBeta, d)).
int update_prior_one(Model& m, int mode, int iter) {
  Prior& p = m.prior[mode];
  const int K = m.K;
  const std::vector<double>& U = m.lat[mode];
  const int N = m.dims[mode];
  std::vector<double> Ud((size_t)K * N), WI((size_t)K * K, 0.0), mu0(K, 0.0);
  for (size_t t = 0; t < Ud.size(); t++) Ud[t] = U[t] - p.Uhat[t];
  for (int d = 0; d < K; d++) WI[d + (size_t)d * K] = 1.0;
  int st = orc_cond_normal_wishart(K, N, Ud.data(), mu0.data(), 2.0, WI.data(), K, m.seed,
                                   (uint32_t)iter, (uint32_t)mode, p.mu.data(), p.Lambda.data());
  if (st) return st;
  // sample_beta (macauoneprior.cpp:216-257)
  const int nF = p.nfeat;
  std::vector<double> Z((size_t)N * K);  // Z[i * K + d]
  for (int i = 0; i < N; i++)
    for (int d = 0; d < K; d++)
      Z[(size_t)i * K + d] = U[(size_t)i * K + d] - p.mu[d] - p.Uhat[(size_t)i * K + d];
  const Csr& Ft = p.Ft;  // row f: the entries of column f of F
#pragma omp parallel for schedule(static, 1)
  for (int d0 = 0; d0 < K; d0 += 4) {
    const int dc = std::min(4, K - d0);
    for (int f = 0; f < nF; f++) {
      double zx[4] = {0.0, 0.0, 0.0, 0.0}, delta[4];
      for (int64_t e = Ft.ptr[f]; e < Ft.ptr[f + 1]; e++) {
        const double v = Ft.val ? Ft.val[e] : 1.0;
        for (int d = 0; d < dc; d++) zx[d] += v * Z[(size_t)Ft.idx[e] * K + d0 + d];
      }
      for (int d = 0; d < dc; d++) {
        const int dx = d0 + d;
        const double lam = p.Lambda[dx + (size_t)dx * K];
        const double z = normal_draw(m.seed, (uint32_t)iter, stream_id(kBetaOne, (uint32_t)mode),
                                     (uint32_t)f, (uint32_t)dx);
        double& bf = p.beta[(size_t)f * K + dx];
        const double A = p.lb_one[dx] + lam * p.colsq[f];
        const double B = lam * (zx[d] + bf * p.colsq[f]);
        const double Ainv = 1.0 / A;
        const double bnew = B * Ainv + std::sqrt(Ainv) * z;
        delta[d] = bf - bnew;
        bf = bnew;
      }
      for (int64_t e = Ft.ptr[f]; e < Ft.ptr[f + 1]; e++) {
        const double v = Ft.val ? Ft.val[e] : 1.0;
        for (int d = 0; d < dc; d++) Z[(size_t)Ft.idx[e] * K + d0 + d] += v * delta[d];
      }
    }
  }
  csr_mul_bn(p.F, p.beta.data(), K, p.Uhat.data());  // compute_uhat
  // sample_lambda_beta (macauoneprior.cpp:267-290)
  const double a = p.lb_a0 + nF / 2.0;
  for (int d = 0; d < K; d++) {
    double ss = 0.0;
    for (int f = 0; f < nF; f++) ss += p.beta[(size_t)f * K + d] * p.beta[(size_t)f * K + d];
    const double b = p.lb_b0 + ss / 2.0;
    p.lb_one[d] = gamma_draw(m.seed, (uint32_t)iter, stream_id(kLambdaBeta, (uint32_t)mode),
                             (uint32_t)d, a) * (1.0 / b);
  }
  return 0;
}

int update_prior(Model& m, int mode, int iter) {
  Prior& p = m.prior[mode];
  if (p.one) return update_prior_one(m, mode, iter);
  const int K = m.K;
  const std::vector<double>& U = m.lat[mode];
  const int N = m.dims[mode];
  if (!p.macau) {  // BPMFPrior::update_prior (latentprior.cpp:79-81)
    return orc_cond_normal_wishart(K, N, U.data(), p.mu0.data(), p.b0, p.WI.data(), p.df,
                                   m.seed, (uint32_t)iter, (uint32_t)mode, p.mu.data(),
                                   p.Lambda.data());
  }
  // MacauPrior::update_prior (latentprior.cpp:255-264)
  for (size_t t = 0; t < p.Uhat.size(); t++) p.Uhat[t] = U[t] - p.Uhat[t];
  std::vector<double> BBt((size_t)K * K), T((size_t)K * K);
  a_mul_bt_lower(p.beta.data(), p.beta.data(), K, p.nfeat, BBt.data(), true);
  for (size_t t = 0; t < T.size(); t++) T[t] = p.WI[t] + p.lambda_beta * BBt[t];
  int st = orc_cond_normal_wishart(K, N, p.Uhat.data(), p.mu0.data(), p.b0, T.data(),
                                   p.df + p.nfeat, m.seed, (uint32_t)iter, (uint32_t)mode,
                                   p.mu.data(), p.Lambda.data());
  if (st) return st;
  sample_beta(m, p, U, mode, iter);
  csr_mul_bn(p.F, p.beta.data(), K, p.Uhat.data());  // compute_uhat (linop.h:196-198)
  double b, c;
  orc_posterior_lambda_beta(K, p.nfeat, p.beta.data(), p.Lambda.data(), p.lb_nu0, p.lb_mu0, &b,
                            &c);
  p.lambda_beta = c * gamma_draw(m.seed, (uint32_t)iter, stream_id(kLambdaBeta, (uint32_t)mode),
                                 0u, b);
  return 0;
}

// AdaptiveGaussianNoise::update (noisemodels.cpp:55-81): the squared training residuals summed
// over the columns of Y in storage order, then alpha ~ Gamma(aN, 1 / bN) capped at alpha_max,
// with (a0, b0) = (1/2, var_total / 2), one prior sample of noise at the full variance.
void update_noise(Model& m, int iter) {
  if (!m.adaptive) return;
  const Csr& C = m.Y[1];  // columns of Y: C.idx are row indices
  const int K = m.K;
  const double* U = m.lat[0].data();
  const double* V = m.lat[1].data();
  double sumsq = 0.0;
  for (int j = 0; j < C.nrow; j++)
    for (int64_t e = C.ptr[j]; e < C.ptr[j + 1]; e++) {
      const double* u = U + (size_t)C.idx[e] * K;
      const double* v = V + (size_t)j * K;
      double dot = 0.0;
      for (int k = 0; k < K; k++) dot += v[k] * u[k];
      const double d = (dot + m.mean) - C.val[e];
      sumsq += d * d;
    }
  const double nnz = (double)C.ptr[C.nrow];
  const double aN = 0.5 + nnz / 2.0;
  const double bN = 0.5 * m.var_total + sumsq / 2.0;
  double a = gamma_draw(m.seed, (uint32_t)iter, stream_id(kNoiseAlpha, 0u), 0u, aN) * (1.0 / bN);
  if (a > m.alpha_max) a = m.alpha_max;
  m.alpha = a;
}

void eval_model(Model& m, int n) {
  if (m.ntest == 0) {
    m.rmse = NAN;
    m.rmse1 = NAN;
    return;
  }
  orc_eval_rmse(m.ntest, m.trow, m.tcol, m.tval, n, m.pred.data(), m.pred_var.data(),
                m.lat[1].data(), m.lat[0].data(), m.K, m.mean, &m.rmse1, &m.rmse);
}

}  // namespace

extern "C" {

void* orc_model_create(int K, double alpha, uint64_t seed) {
  Model* m = new Model();
  m->K = K;
  m->alpha = alpha;
  m->seed = seed;
  init_prior(m->prior[0], K);
  init_prior(m->prior[1], K);
  return m;
}

void orc_model_destroy(void* h) { delete static_cast<Model*>(h); }

// The model keeps the caller's arrays (no copy); they must outlive the model.
void orc_model_set_train(void* h, int nrow, int ncol, const int64_t* rptr, const int32_t* ridx,
                         const double* rval, const int64_t* cptr, const int32_t* cidx,
                         const double* cval, double mean) {
  Model& m = *static_cast<Model*>(h);
  m.dims[0] = nrow;
  m.dims[1] = ncol;
  m.Y[0] = Csr{rptr, ridx, rval, nrow, ncol};
  m.Y[1] = Csr{cptr, cidx, cval, ncol, nrow};
  m.mean = mean;
  m.lat[0].assign((size_t)m.K * nrow, 0.0);  // MacauX::init zeros (macau.cpp:78-82)
  m.lat[1].assign((size_t)m.K * ncol, 0.0);
}

void orc_model_set_test(void* h, int ntest, const int32_t* rows, const int32_t* cols,
                        const double* vals) {
  Model& m = *static_cast<Model*>(h);
  m.ntest = ntest;
  m.trow = rows;
  m.tcol = cols;
  m.tval = vals;
  m.pred.assign(ntest, 0.0);
  m.pred_var.assign(ntest, 0.0);
}

void orc_model_set_side(void* h, int mode, int nfeat, const int64_t* fptr, const int32_t* fidx,
                        const double* fval, const int64_t* tptr, const int32_t* tidx,
                        const double* tval, double lambda_beta, double tol) {
  Model& m = *static_cast<Model*>(h);
  Prior& p = m.prior[mode];
  const int N = m.dims[mode];
  p.macau = true;
  p.nfeat = nfeat;
  p.F = Csr{fptr, fidx, fval, N, nfeat};
  p.Ft = Csr{tptr, tidx, tval, nfeat, N};
  p.Uhat.assign((size_t)m.K * N, 0.0);
  p.beta.assign((size_t)m.K * nfeat, 0.0);
  p.lambda_beta = lambda_beta;
  p.tol = tol;
}

// MacauOnePrior<SparseFeat | SparseDoubleFeat>(K, F) + setLambdaBeta (macauoneprior.cpp:16-39,
// macau.pyx:194-214): mu = 0, Lambda = 10 I, beta = Uhat = 0, lambda_beta = lambda_beta for every
// dimension, colsq = squared column norms of F (the column counts when F is binary).
void orc_model_set_side_one(void* h, int mode, int nfeat, const int64_t* fptr,
                            const int32_t* fidx, const double* fval, const int64_t* tptr,
                            const int32_t* tidx, const double* tval, double lambda_beta) {
  Model& m = *static_cast<Model*>(h);
  Prior& p = m.prior[mode];
  const int N = m.dims[mode];
  p.macau = false;
  p.one = true;
  p.nfeat = nfeat;
  p.F = Csr{fptr, fidx, fval, N, nfeat};
  p.Ft = Csr{tptr, tidx, tval, nfeat, N};
  p.Uhat.assign((size_t)m.K * N, 0.0);
  p.beta.assign((size_t)m.K * nfeat, 0.0);
  p.lb_one.assign(m.K, lambda_beta);
  p.colsq.assign(nfeat, 0.0);
  for (int f = 0; f < nfeat; f++)
    for (int64_t e = tptr[f]; e < tptr[f + 1]; e++) p.colsq[f] += tval ? tval[e] * tval[e] : 1.0;
}

// sample_mode restricted to rows lo .. hi - 1 (BPMF and Macau priors): one rank's share of a
// row-sharded half-sweep.
int orc_model_sample_rows(void* h, int mode, int iter, int lo, int hi) {
  Model& m = *static_cast<Model*>(h);
  Prior& p = m.prior[mode];
  const Csr& R = m.Y[mode];
  if (p.one || lo < 0 || hi < lo || hi > R.nrow) return -2;
  return sample_latent_rows(m.K, lo, hi, R.ptr, R.idx, R.val, m.mean, m.lat[1 - mode].data(),
                            m.alpha, p.mu.data(), p.Lambda.data(),
                            p.macau ? p.Uhat.data() : nullptr, m.seed, (uint32_t)iter,
                            (uint32_t)mode, nullptr, m.lat[mode].data());
}

int orc_model_sample_mode(void* h, int mode, int iter) {
  return sample_mode(*static_cast<Model*>(h), mode, iter);
}
int orc_model_update_prior(void* h, int mode, int iter) {
  return update_prior(*static_cast<Model*>(h), mode, iter);
}
void orc_model_eval(void* h, int n) { eval_model(*static_cast<Model*>(h), n); }

// One iteration of MacauX::run (macau.cpp:110-147): both modes' latents, both priors, eval.
int orc_model_sweep(void* h, int iter, int burnin) {
  Model& m = *static_cast<Model*>(h);
  for (int mode = 0; mode < 2; mode++)
    if (sample_mode(m, mode, iter)) return -1;
  for (int mode = 0; mode < 2; mode++)
    if (update_prior(m, mode, iter)) return -1;
  update_noise(m, iter);
  eval_model(m, iter < burnin ? 0 : iter - burnin);
  return 0;
}

// AdaptiveGaussianNoise(sn_init, sn_max) + init (noisemodels.cpp:14-33, macau.cpp:222-228):
// var_total = mean squared deviation of the training values from the mean (in column storage
// order; 1 when not positive or NaN), alpha = (sn_init + 1) / var_total, alpha_max =
// (sn_max + 1) / var_total.  Call after orc_model_set_train.
void orc_model_set_noise_adaptive(void* h, double sn_init, double sn_max) {
  Model& m = *static_cast<Model*>(h);
  const Csr& C = m.Y[1];
  const int64_t nnz = C.ptr[C.nrow];
  double se = 0.0;
  for (int64_t e = 0; e < nnz; e++) se += (C.val[e] - m.mean) * (C.val[e] - m.mean);
  double vt = se / (double)nnz;
  if (vt <= 0.0 || std::isnan(vt)) vt = 1.0;
  m.adaptive = true;
  m.var_total = vt;
  m.alpha = (sn_init + 1.0) / vt;
  m.alpha_max = (sn_max + 1.0) / vt;
}

int orc_model_update_noise(void* h, int iter) {
  update_noise(*static_cast<Model*>(h), iter);
  return 0;
}

// what: 0 latents (K x dim), 1 mu (K), 2 Lambda (K x K), 3 beta (K x nfeat), 4 Uhat (K x dim),
//       5 [lambda_beta, cg_iters], 6 predictions, 7 predictions_var, 8 [rmse_avg, rmse_1samp],
//       9 [alpha, alpha_max, var_total] (noise precision), 10 lambda_beta per dimension (K,
//       univariate prior)
void orc_model_get(void* h, int what, int mode, double* out) {
  Model& m = *static_cast<Model*>(h);
  Prior& p = m.prior[mode];
  switch (what) {
    case 0: std::copy(m.lat[mode].begin(), m.lat[mode].end(), out); break;
    case 1: std::copy(p.mu.begin(), p.mu.end(), out); break;
    case 2: std::copy(p.Lambda.begin(), p.Lambda.end(), out); break;
    case 3: std::copy(p.beta.begin(), p.beta.end(), out); break;
    case 4: std::copy(p.Uhat.begin(), p.Uhat.end(), out); break;
    case 5: out[0] = p.lambda_beta; out[1] = p.cg_iters; break;
    case 6: std::copy(m.pred.begin(), m.pred.end(), out); break;
    case 7: std::copy(m.pred_var.begin(), m.pred_var.end(), out); break;
    case 8: out[0] = m.rmse; out[1] = m.rmse1; break;
    case 9: out[0] = m.alpha; out[1] = m.alpha_max; out[2] = m.var_total; break;
    case 10: std::copy(p.lb_one.begin(), p.lb_one.end(), out); break;
    default: break;
  }
}

// what: 0 latents, 1 mu, 2 Lambda, 3 beta, 4 Uhat, 5 lambda_beta, 9 noise precision alpha
void orc_model_set(void* h, int what, int mode, const double* in) {
  Model& m = *static_cast<Model*>(h);
  Prior& p = m.prior[mode];
  switch (what) {
    case 0: std::copy(in, in + m.lat[mode].size(), m.lat[mode].begin()); break;
    case 1: std::copy(in, in + p.mu.size(), p.mu.begin()); break;
    case 2: std::copy(in, in + p.Lambda.size(), p.Lambda.begin()); break;
    case 3: std::copy(in, in + p.beta.size(), p.beta.begin()); break;
    case 4: std::copy(in, in + p.Uhat.size(), p.Uhat.begin()); break;
    case 5: p.lambda_beta = in[0]; break;
    case 9: m.alpha = in[0]; break;
    case 10: std::copy(in, in + p.lb_one.size(), p.lb_one.begin()); break;
    default: break;
  }
}

}  // extern "C"
