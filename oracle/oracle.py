"""TEST INFRASTRUCTURE ONLY: ctypes bindings to the CPU oracle (oracle/_build/liboracle.so).

The oracle is the FP64 restatement of the reference's Gibbs-sweep hot path (see
macau_oracle.cpp for the file:line of every restated function).  Only tests/, the smoke check in
__graft_entry__ and bench.py's CPU-baseline / reference arm may import this module.
"""
import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

_HERE = Path(__file__).resolve().parent
LIB_PATH = _HERE / "_build" / "liboracle.so"

PURPOSE = dict(row_noise=1, mvn_n=2, mvn_f=3, wishart_off=4, wishart_diag=5, mu_draw=6,
               lambda_beta=7, noise_alpha=8, beta_one=9)

_d = C.c_double
_i = C.c_int
_u32 = C.c_uint32
_u64 = C.c_uint64
_p = C.c_void_p


def build():
    """Compiles the oracle with its Makefile (system g++, OpenMP)."""
    subprocess.run(["make", "-s", "-C", str(_HERE)], check=True)


def _load():
    if not LIB_PATH.exists():
        build()
    lib = C.CDLL(str(LIB_PATH))
    sig = {
        "orc_philox": (None, [_p, _p, _p]),
        "orc_normal": (_d, [_u64, _u32, _u32, _u32, _u32]),
        "orc_gamma": (_d, [_u64, _u32, _u32, _u32, _d]),
        "orc_set_threads": (_i, [_i]),
        "orc_set_reduce_parts": (_i, [_i]),
        "orc_sample_latents": (_i, [_i, _i, _i, _p, _p, _p, _d, _p, _d, _p, _p, _p, _u64, _u32,
                                    _u32, _p, _p]),
        "orc_cond_normal_wishart": (_i, [_i, _i, _p, _p, _d, _p, _i, _u64, _u32, _u32, _p, _p]),
        "orc_csr_mul_bn": (None, [_i, _i, _p, _p, _p, _p, _i, _p]),
        "orc_ata_mul_bx": (None, [_i, _i, _p, _p, _p, _p, _p, _p, _d, _p, _i, _p]),
        "orc_blockcg_core": (_i, [_i, _i, _i, _p, _p, _p, _p, _p, _p, _d, _p, _d, _p]),
        "orc_blockcg": (_i, [_i, _i, _i, _p, _p, _p, _p, _p, _p, _d, _p, _d, _i, _i, _p]),
        "orc_posterior_lambda_beta": (None, [_i, _i, _p, _p, _d, _d, _p, _p]),
        "orc_eval_rmse": (None, [_i, _p, _p, _p, _i, _p, _p, _p, _p, _i, _d, _p, _p]),
        "orc_model_create": (_p, [_i, _d, _u64]),
        "orc_model_destroy": (None, [_p]),
        "orc_model_set_train": (None, [_p, _i, _i, _p, _p, _p, _p, _p, _p, _d]),
        "orc_model_set_test": (None, [_p, _i, _p, _p, _p]),
        "orc_model_set_side": (None, [_p, _i, _i, _p, _p, _p, _p, _p, _p, _d, _d]),
        "orc_model_sample_mode": (_i, [_p, _i, _i]),
        "orc_model_sample_rows": (_i, [_p, _i, _i, _i, _i]),
        "orc_model_update_prior": (_i, [_p, _i, _i]),
        "orc_model_eval": (None, [_p, _i]),
        "orc_model_sweep": (_i, [_p, _i, _i]),
        "orc_model_get": (None, [_p, _i, _i, _p]),
        "orc_model_set_noise_adaptive": (None, [_p, _d, _d]),
        "orc_model_set_side_one": (None, [_p, _i, _i, _p, _p, _p, _p, _p, _p, _d]),
        "orc_model_update_noise": (_i, [_p, _i]),
        "orc_model_set": (None, [_p, _i, _i, _p]),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    return lib


_LIB = None


def lib():
    global _LIB
    if _LIB is None:
        _LIB = _load()
    return _LIB


def _ptr(a):
    return None if a is None else a.ctypes.data


def f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def set_threads(n=0):
    return lib().orc_set_threads(int(n))


def set_reduce_parts(n):
    """Partial-sum count of the oracle's K x K reductions (the reference uses one per OpenMP
    thread; linop.cpp:280-317).  Returns the value in force."""
    return lib().orc_set_reduce_parts(int(n))


def philox(ctr, key):
    c = np.asarray(ctr, dtype=np.uint32)
    k = np.asarray(key, dtype=np.uint32)
    out = np.zeros(4, dtype=np.uint32)
    lib().orc_philox(_ptr(c), _ptr(k), _ptr(out))
    return out


def stream(purpose, mode):
    return (PURPOSE[purpose] << 8) | mode


def normal(seed, sweep, purpose, mode, index, j):
    return lib().orc_normal(seed, sweep, stream(purpose, mode), index, j)


def gamma(seed, sweep, purpose, mode, index, shape):
    return lib().orc_gamma(seed, sweep, stream(purpose, mode), index, shape)


class Csr:
    """CSR arrays in the oracle's layout (int64 row pointers, int32 indices, FP64 values or None
    for a binary matrix)."""

    def __init__(self, ptr, idx, val, nrow, ncol):
        self.ptr = np.ascontiguousarray(ptr, dtype=np.int64)
        self.idx = np.ascontiguousarray(idx, dtype=np.int32)
        self.val = None if val is None else f64(val)
        self.nrow, self.ncol = int(nrow), int(ncol)

    @classmethod
    def from_scipy(cls, m, binary=False):
        m = m.tocsr()
        m.sum_duplicates()
        m.sort_indices()
        return cls(m.indptr, m.indices, None if binary else m.data, m.shape[0], m.shape[1])

    def transpose_of(self, m, binary=False):
        return Csr.from_scipy(m.T, binary)


def sample_latents(K, R, other, mean_rating, alpha, mu, Lambda, Uhat=None, seed=0, sweep=0,
                   mode=0, z=None):
    """sample_latent_blas over every row of CSR R; returns (K x nrow FP64, status)."""
    other = f64(other)
    out = np.zeros((R.nrow, K))
    st = lib().orc_sample_latents(K, R.nrow, R.ncol, _ptr(R.ptr), _ptr(R.idx), _ptr(R.val),
                                  mean_rating, _ptr(other), alpha, _ptr(f64(mu)),
                                  _ptr(f64(Lambda)), _ptr(None if Uhat is None else f64(Uhat)),
                                  seed, sweep, mode, _ptr(None if z is None else f64(z)),
                                  _ptr(out))
    return out, st


def cond_normal_wishart(U, mu0, kappa, T, nu, seed=0, sweep=0, mode=0):
    """U: (N, K) array of latent columns.  Returns (mu, Lambda, status)."""
    U = f64(U)
    N, K = U.shape
    mu = np.zeros(K)
    Lam = np.zeros((K, K))
    st = lib().orc_cond_normal_wishart(K, N, _ptr(U), _ptr(f64(mu0)), kappa, _ptr(f64(T)), nu,
                                       seed, sweep, mode, _ptr(mu), _ptr(Lam))
    return mu, Lam, st


def csr_mul_bn(A, B):
    """out[r] = sum val * B[idx] with B given as (ncol, N); returns (nrow, N)."""
    B = f64(B)
    N = B.shape[1]
    out = np.zeros((A.nrow, N))
    lib().orc_csr_mul_bn(A.nrow, A.ncol, _ptr(A.ptr), _ptr(A.idx), _ptr(A.val), _ptr(B), N,
                         _ptr(out))
    return out


def ata_mul_bx(F, Ft, reg, B):
    B = f64(B)
    N = B.shape[1]
    out = np.zeros((F.ncol, N))
    lib().orc_ata_mul_bx(F.nrow, F.ncol, _ptr(F.ptr), _ptr(F.idx), _ptr(F.val), _ptr(Ft.ptr),
                         _ptr(Ft.idx), _ptr(Ft.val), reg, _ptr(B), N, _ptr(out))
    return out


def blockcg(F, Ft, reg, B, tol, blocksize=None, excess=None):
    """B: (nfeat, nrhs) -- column f holds the nrhs right-hand-side values of feature f (the
    reference's K x nfeat column-major B).  Returns (X (nfeat, nrhs), iterations)."""
    B = f64(B)
    nfeat, nrhs = B.shape
    X = np.zeros_like(B)
    args = (nrhs, F.nrow, nfeat, _ptr(F.ptr), _ptr(F.idx), _ptr(F.val), _ptr(Ft.ptr),
            _ptr(Ft.idx), _ptr(Ft.val), reg, _ptr(B), tol)
    if blocksize is None:
        it = lib().orc_blockcg_core(*args, _ptr(X))
    else:
        it = lib().orc_blockcg(*args, blocksize, excess, _ptr(X))
    return X, it


def posterior_lambda_beta(beta, Lambda, nu, mu):
    """beta: (nfeat, K) columns; returns (shape, scale)."""
    beta = f64(beta)
    nfeat, K = beta.shape
    b = np.zeros(1)
    c = np.zeros(1)
    lib().orc_posterior_lambda_beta(K, nfeat, _ptr(beta), _ptr(f64(Lambda)), nu, mu, _ptr(b),
                                    _ptr(c))
    return b[0], c[0]


def eval_rmse(rows, cols, vals, n, pred, pred_var, V, U, mean_rating):
    rows = np.ascontiguousarray(rows, dtype=np.int32)
    cols = np.ascontiguousarray(cols, dtype=np.int32)
    V = f64(V)
    U = f64(U)
    r = np.zeros(1)
    ra = np.zeros(1)
    lib().orc_eval_rmse(len(rows), _ptr(rows), _ptr(cols), _ptr(f64(vals)), n, _ptr(pred),
                        _ptr(pred_var), _ptr(V), _ptr(U), U.shape[1], mean_rating, _ptr(r),
                        _ptr(ra))
    return r[0], ra[0]


class Model:
    """Whole-sweep FP64 model (MacauX::run body, macau.cpp:110-147).  Arrays handed to it are
    kept alive by this object."""

    def __init__(self, K, alpha, seed):
        self.K = K
        self._keep = []
        self.h = lib().orc_model_create(K, alpha, seed)
        self.dims = (0, 0)
        self.nfeat = [0, 0]
        self.ntest = 0

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_model_destroy(self.h)
            self.h = None

    def set_train(self, Rrows, Rcols, mean):
        self._keep += [Rrows, Rcols]
        lib().orc_model_set_train(self.h, Rrows.nrow, Rcols.nrow, _ptr(Rrows.ptr),
                                  _ptr(Rrows.idx), _ptr(Rrows.val), _ptr(Rcols.ptr),
                                  _ptr(Rcols.idx), _ptr(Rcols.val), mean)
        self.dims = (Rrows.nrow, Rcols.nrow)

    def set_test(self, rows, cols, vals):
        rows = np.ascontiguousarray(rows, dtype=np.int32)
        cols = np.ascontiguousarray(cols, dtype=np.int32)
        vals = f64(vals)
        self._keep += [rows, cols, vals]
        self.ntest = len(rows)
        lib().orc_model_set_test(self.h, len(rows), _ptr(rows), _ptr(cols), _ptr(vals))

    def set_side(self, mode, F, Ft, lambda_beta, tol):
        self._keep += [F, Ft]
        self.nfeat[mode] = F.ncol
        lib().orc_model_set_side(self.h, mode, F.ncol, _ptr(F.ptr), _ptr(F.idx), _ptr(F.val),
                                 _ptr(Ft.ptr), _ptr(Ft.idx), _ptr(Ft.val), lambda_beta, tol)

    def set_side_one(self, mode, F, Ft, lambda_beta):
        """MacauOnePrior (univariate sampler) with side information F for `mode`
        (macauoneprior.cpp:16-39; binary F when built with binary=True)."""
        self._keep += [F, Ft]
        self.nfeat[mode] = F.ncol
        lib().orc_model_set_side_one(self.h, mode, F.ncol, _ptr(F.ptr), _ptr(F.idx), _ptr(F.val),
                                     _ptr(Ft.ptr), _ptr(Ft.idx), _ptr(Ft.val), lambda_beta)

    def lambda_beta_one(self, mode):
        """lambda_beta per dimension of a univariate prior (K,)."""
        return self._get(10, mode, (self.K,))

    def set_noise_adaptive(self, sn_init=1.0, sn_max=10.0):
        """AdaptiveGaussianNoise(sn_init, sn_max) + init (noisemodels.cpp:14-33); after set_train."""
        lib().orc_model_set_noise_adaptive(self.h, sn_init, sn_max)

    def update_noise(self, it):
        """AdaptiveGaussianNoise::update with the draw of sweep `it` (noisemodels.cpp:55-81)."""
        return lib().orc_model_update_noise(self.h, it)

    def noise(self):
        """(alpha, alpha_max, var_total) of the noise model."""
        return tuple(self._get(9, 0, (3,)))

    def sweep(self, it, burnin):
        return lib().orc_model_sweep(self.h, it, burnin)

    def sample_mode(self, mode, it):
        return lib().orc_model_sample_mode(self.h, mode, it)

    def sample_rows(self, mode, it, lo, hi):
        """sample_mode for rows lo .. hi - 1 only (draws keyed by the global row index)."""
        return lib().orc_model_sample_rows(self.h, mode, it, int(lo), int(hi))

    def update_prior(self, mode, it):
        return lib().orc_model_update_prior(self.h, mode, it)

    def eval(self, n):
        lib().orc_model_eval(self.h, n)

    def _get(self, what, mode, shape):
        out = np.zeros(shape)
        lib().orc_model_get(self.h, what, mode, _ptr(out))
        return out

    def latents(self, mode):
        return self._get(0, mode, (self.dims[mode], self.K))

    def mu(self, mode):
        return self._get(1, mode, (self.K,))

    def Lambda(self, mode):
        return self._get(2, mode, (self.K, self.K))

    def beta(self, mode):
        return self._get(3, mode, (self.nfeat[mode], self.K))

    def uhat(self, mode):
        return self._get(4, mode, (self.dims[mode], self.K))

    def lambda_beta(self, mode):
        return self._get(5, mode, (2,))

    def predictions(self):
        return self._get(6, 0, (self.ntest,))

    def predictions_var(self):
        return self._get(7, 0, (self.ntest,))

    def rmse(self):
        return tuple(self._get(8, 0, (2,)))

    def set(self, what, mode, arr):
        arr = f64(arr)
        self._keep.append(arr)
        code = dict(latents=0, mu=1, Lambda=2, beta=3, uhat=4, lambda_beta=5, alpha=9,
                    lambda_beta_one=10)[what]
        lib().orc_model_set(self.h, code, mode, _ptr(arr))
