"""ctypes binding of the C ABI in include/macau_b200.h (the in-tree libmacau_b200.so).

There is no CPU fallback: loading fails loudly when the library has not been built, and every
call that needs a GPU fails with the library's own error when no sm_100 device is present.
"""
import ctypes as C
from pathlib import Path

import numpy as np

LIB_PATH = Path(__file__).resolve().parent / "_lib" / "libmacau_b200.so"

MG_COMPUTE_FP64 = 0
MG_COMPUTE_MIXED = 1

MG_ERR_ARG, MG_ERR_CHOL, MG_ERR_CG, MG_ERR_CUDA = -1, -2, -3, -4
MG_ERR_STATE, MG_ERR_TIMEOUT, MG_ERR_NOGPU = -5, -6, -7

ERRORS = {-1: "invalid argument", -2: "Cholesky Decomposition failed!", -3: "block-CG failure",
          -4: "CUDA error", -5: "call out of order", -6: "device wait timed out",
          -7: "no sm_100 GPU"}


class MacauError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(msg)
        self.code = code


class CholeskyError(MacauError):
    """Raised where the reference throws std::runtime_error("Cholesky Decomposition failed!")
    (latentprior.cpp:374-376)."""


class MgConfig(C.Structure):
    _fields_ = [("num_latent", C.c_int), ("precision", C.c_double), ("seed", C.c_uint64),
                ("compute", C.c_int), ("verbose", C.c_int), ("device", C.c_int)]


class MgStats(C.Structure):
    _fields_ = [("sweeps", C.c_double), ("seconds_sample", C.c_double),
                ("seconds_prior", C.c_double), ("seconds_eval", C.c_double),
                ("retries", C.c_int64 * 2), ("rows_sampled", C.c_int64 * 2),
                ("cg_iters", C.c_int * 2), ("graph_captured", C.c_int),
                ("kernel_launches", C.c_int64), ("h2d_bytes", C.c_int64),
                ("d2h_bytes", C.c_int64), ("ntasks", C.c_int64 * 2), ("nnz", C.c_int64 * 2)]


class MgTuning(C.Structure):
    _fields_ = [("split_threshold", C.c_int64), ("cta_groups", C.c_int), ("tensor_core", C.c_int),
                ("state", C.c_int), ("candidates", C.c_int), ("ms_best", C.c_double),
                ("ms_default", C.c_double), ("finish_ctas_per_sm", C.c_int)]


_p = C.c_void_p
_i = C.c_int
_d = C.c_double
_i64 = C.c_int64

_SIGS = {
    "mg_create": (_i, [C.POINTER(_p), C.POINTER(MgConfig)]),
    "mg_destroy": (None, [_p]),
    "mg_last_error": (C.c_char_p, [_p]),
    "mg_set_relation_data": (_i, [_p, _p, _i, _p, _i64, _p]),
    "mg_set_relation_data_test": (_i, [_p, _p, _i, _p, _i64, _p]),
    "mg_set_relation_data_rc": (_i, [_p, _p, _p, _p, _i64, _i, _i]),
    "mg_set_relation_data_test_rc": (_i, [_p, _p, _p, _p, _i64, _i, _i]),
    "mg_set_side": (_i, [_p, _i, _p, _p, _p, _i64, _i, _i, _d, _d]),
    "mg_set_samples": (_i, [_p, _i, _i]),
    "mg_init": (_i, [_p]),
    "mg_sweep": (_i, [_p, _i, _i]),
    "mg_sweeps": (_i, [_p, _i, _i, _i]),
    "mg_run": (_i, [_p]),
    "mg_time_sweeps": (_i, [_p, _i, _i, _i, _i, _p, _p]),
    "mg_sample_latents": (_i, [_p, _i, _i, _p]),
    "mg_update_prior": (_i, [_p, _i, _i]),
    "mg_eval": (_i, [_p, _i]),
    "mg_set_noise_adaptive": (_i, [_p, _d, _d]),
    "mg_set_side_univariate": (_i, [_p, _i, _p, _p, _p, _i64, _i, _i, _d]),
    "mg_get_lambda_beta_univariate": (_i, [_p, _i, _p]),
    "mg_update_noise": (_i, [_p, _i]),
    "mg_get_noise": (_i, [_p, _p]),
    "mg_get_latents": (_i, [_p, _i, _p]),
    "mg_set_latents": (_i, [_p, _i, _p]),
    "mg_get_hyper": (_i, [_p, _i, _p, _p, _p]),
    "mg_set_hyper": (_i, [_p, _i, _p, _p, _p]),
    "mg_get_beta": (_i, [_p, _i, _p]),
    "mg_get_uhat": (_i, [_p, _i, _p]),
    "mg_get_dims": (_i, [_p, _p, _p, _p, _p, _p]),
    "mg_get_rmse": (_i, [_p, _p]),
    "mg_get_predictions": (_i, [_p, _p]),
    "mg_get_stds": (_i, [_p, _p]),
    "mg_get_test_data": (_i, [_p, _p]),
    "mg_get_stats": (_i, [_p, C.POINTER(MgStats)]),
    "mg_set_option": (_i, [_p, C.c_char_p, _i]),
    "mg_autotune": (_i, [_p, _i]),
    "mg_get_tuning": (_i, [_p, _i, C.POINTER(MgTuning)]),
    "mg_blockcg": (_i, [_p, _p, _p, _i64, _i, _i, _p, _i, _d, _d, _i, _p, C.POINTER(_i),
                        C.POINTER(_d)]),
    "mg_batch_create": (_i, [C.POINTER(_p), _i, _p, _p, _p, _p, _d, _i]),
    "mg_batch_destroy": (None, [_p]),
    "mg_batch_last_error": (C.c_char_p, [_p]),
    "mg_batch_set_data": (_i, [_p, _p, _p, _p, _p, _p, _p, _p, _p]),
    "mg_batch_init": (_i, [_p, _i]),
    "mg_batch_sweeps": (_i, [_p, _i, _i, _i]),
    "mg_batch_time_sweeps": (_i, [_p, _i, _i, C.POINTER(_d)]),
    "mg_batch_get_latents": (_i, [_p, _i, _i, _p]),
    "mg_batch_get_rmse": (_i, [_p, _p]),
    "mg_batch_get_info": (_i, [_p, _p]),
    "mg_batch_autotune": (_i, [_p, _i]),
    "mg_batch_get_tuning": (_i, [_p, _i, C.POINTER(MgTuning)]),
    "mg_set_row_range": (_i, [_p, _i, _i64, _i64]),
    "mg_latents_device": (_i, [_p, _i, C.POINTER(_p), C.POINTER(_i), C.POINTER(_i)]),
    "mg_latents_changed": (_i, [_p, _i]),
    "mg_get_stream": (_i, [_p, C.POINTER(_p)]),
    "mg_normal_wishart_noalloc": (_i, [_p, _i64, _i, _i, _p, _d, _p, _i, C.c_uint64, C.c_uint32,
                                       _i, _p, _p, _p, C.c_char_p, _i]),
}

EXPORTED = tuple(_SIGS)

_LIB = None


def lib():
    """Loads libmacau_b200.so (raises if it has not been built)."""
    global _LIB
    if _LIB is None:
        if not LIB_PATH.exists():
            raise ImportError(f"{LIB_PATH} is missing: build it with `python -m macau_b200.build`")
        L = C.CDLL(str(LIB_PATH))
        for name, (res, args) in _SIGS.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _LIB = L
    return _LIB


def ptr(a):
    return None if a is None else a.ctypes.data


def check(code, ctx=None):
    if code == 0:
        return
    msg = lib().mg_last_error(ctx).decode() if lib().mg_last_error(ctx) else ERRORS.get(code, "")
    cls = CholeskyError if code == -2 else MacauError
    raise cls(code, msg or ERRORS.get(code, f"error {code}"))


class Sampler:
    """Thin object wrapper of one mg_ctx (a MacauX<MatrixData, FixedGaussianNoise> on the GPU)."""

    def __init__(self, num_latent, precision, seed=0, compute=MG_COMPUTE_FP64, verbose=False,
                 device=0):
        self.K = int(num_latent)
        self.compute = compute
        cfg = MgConfig(self.K, float(precision), int(seed) & (2**64 - 1), int(compute),
                       int(bool(verbose)), int(device))
        h = _p()
        code = lib().mg_create(C.byref(h), C.byref(cfg))
        check(code, None)
        self.h = h
        self.dims = (0, 0)
        self.nfeat = [0, 0]
        self.ntest = 0

    def close(self):
        if getattr(self, "h", None):
            lib().mg_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def _chk(self, code):
        check(code, self.h)

    def set_relation_data(self, rows, cols, vals, shape):
        if not len(rows) == len(cols) == len(vals):
            raise ValueError("rows, cols and vals must have the same length")
        rows = np.ascontiguousarray(rows, np.int32)
        cols = np.ascontiguousarray(cols, np.int32)
        vals = np.ascontiguousarray(vals, np.float64)
        self._chk(lib().mg_set_relation_data_rc(self.h, ptr(rows), ptr(cols), ptr(vals),
                                                len(vals), int(shape[0]), int(shape[1])))
        self.dims = (int(shape[0]), int(shape[1]))

    def set_relation_data_test(self, rows, cols, vals, shape):
        if not len(rows) == len(cols) == len(vals):
            raise ValueError("rows, cols and vals must have the same length")
        rows = np.ascontiguousarray(rows, np.int32)
        cols = np.ascontiguousarray(cols, np.int32)
        vals = np.ascontiguousarray(vals, np.float64)
        self._chk(lib().mg_set_relation_data_test_rc(self.h, ptr(rows), ptr(cols), ptr(vals),
                                                     len(vals), int(shape[0]), int(shape[1])))
        n = np.zeros(1, np.int64)
        self._chk(lib().mg_get_dims(self.h, None, None, None, ptr(n), None))
        self.ntest = int(n[0])

    def set_side(self, mode, rows, cols, vals, shape, lambda_beta, tol):
        rows = np.ascontiguousarray(rows, np.int32)
        cols = np.ascontiguousarray(cols, np.int32)
        vals = None if vals is None else np.ascontiguousarray(vals, np.float64)
        self._chk(lib().mg_set_side(self.h, mode, ptr(rows), ptr(cols), ptr(vals), len(rows),
                                    int(shape[0]), int(shape[1]), float(lambda_beta), float(tol)))
        self.nfeat[mode] = int(shape[1])

    def set_side_univariate(self, mode, rows, cols, vals, shape, lambda_beta):
        """MacauOnePrior (univariate sampler) with side information for `mode`."""
        rows = np.ascontiguousarray(rows, np.int32)
        cols = np.ascontiguousarray(cols, np.int32)
        vals = None if vals is None else np.ascontiguousarray(vals, np.float64)
        self._chk(lib().mg_set_side_univariate(self.h, mode, ptr(rows), ptr(cols), ptr(vals),
                                               len(rows), int(shape[0]), int(shape[1]),
                                               float(lambda_beta)))
        self.nfeat[mode] = int(shape[1])

    def lambda_beta_univariate(self, mode):
        out = np.zeros(self.K)
        self._chk(lib().mg_get_lambda_beta_univariate(self.h, mode, ptr(out)))
        return out

    def set_samples(self, burnin, nsamples):
        self._chk(lib().mg_set_samples(self.h, int(burnin), int(nsamples)))

    def set_option(self, name, value):
        self._chk(lib().mg_set_option(self.h, name.encode(), int(value)))

    def init(self):
        self._chk(lib().mg_init(self.h))

    def sweep(self, it, eval=True):
        self._chk(lib().mg_sweep(self.h, int(it), int(bool(eval))))

    def sweeps(self, first, count, eval=True):
        self._chk(lib().mg_sweeps(self.h, int(first), int(count), int(bool(eval))))

    def time_sweeps(self, first, count, eval=False, phase_events=False):
        """Device seconds of `count` sweeps (CUDA events on the library stream); with
        phase_events also the per-phase seconds [sample0, sample1, prior0, prior1, eval,
        gram0, gram1] (gram: the tensor-core Gram kernel alone, 0 when not used)."""
        tot = np.zeros(1)
        ph = np.zeros(7)
        self._chk(lib().mg_time_sweeps(self.h, int(first), int(count), int(bool(eval)),
                                       int(bool(phase_events)), ptr(tot), ptr(ph)))
        return float(tot[0]), ph

    def run(self):
        self._chk(lib().mg_run(self.h))

    def sample_latents(self, mode, it, z=None):
        z = None if z is None else np.ascontiguousarray(z, np.float64)
        self._chk(lib().mg_sample_latents(self.h, mode, int(it), ptr(z)))

    def update_prior(self, mode, it):
        self._chk(lib().mg_update_prior(self.h, mode, int(it)))

    def set_noise_adaptive(self, sn_init=1.0, sn_max=10.0):
        """AdaptiveGaussianNoise(sn_init, sn_max) in place of the fixed precision (before init)."""
        self._chk(lib().mg_set_noise_adaptive(self.h, float(sn_init), float(sn_max)))

    def update_noise(self, it):
        self._chk(lib().mg_update_noise(self.h, int(it)))

    def noise(self):
        """(alpha, alpha_max, var_total) of the noise model."""
        out = np.zeros(3)
        self._chk(lib().mg_get_noise(self.h, out.ctypes.data))
        return tuple(float(x) for x in out)

    def eval(self, n):
        self._chk(lib().mg_eval(self.h, int(n)))

    def latents(self, mode):
        out = np.zeros((self.dims[mode], self.K))
        self._chk(lib().mg_get_latents(self.h, mode, ptr(out)))
        return out

    def set_latents(self, mode, arr):
        arr = np.ascontiguousarray(arr, np.float64)
        assert arr.shape == (self.dims[mode], self.K)
        self._chk(lib().mg_set_latents(self.h, mode, ptr(arr)))

    def hyper(self, mode):
        mu = np.zeros(self.K)
        lam = np.zeros((self.K, self.K))
        lb = np.zeros(1)
        self._chk(lib().mg_get_hyper(self.h, mode, ptr(mu), ptr(lam), ptr(lb)))
        return mu, lam, lb[0]

    def set_hyper(self, mode, mu=None, Lambda=None, lambda_beta=None):
        mu = None if mu is None else np.ascontiguousarray(mu, np.float64)
        lam = None if Lambda is None else np.ascontiguousarray(Lambda, np.float64)
        lb = None if lambda_beta is None else np.array([lambda_beta], np.float64)
        self._chk(lib().mg_set_hyper(self.h, mode, ptr(mu), ptr(lam), ptr(lb)))

    def beta(self, mode):
        out = np.zeros((self.nfeat[mode], self.K))
        self._chk(lib().mg_get_beta(self.h, mode, ptr(out)))
        return out

    def uhat(self, mode):
        out = np.zeros((self.dims[mode], self.K))
        self._chk(lib().mg_get_uhat(self.h, mode, ptr(out)))
        return out

    def rmse(self):
        r = np.zeros(2)
        self._chk(lib().mg_get_rmse(self.h, ptr(r)))
        return float(r[0]), float(r[1])

    def predictions(self):
        out = np.zeros(self.ntest)
        self._chk(lib().mg_get_predictions(self.h, ptr(out)))
        return out

    def stds(self):
        out = np.zeros(self.ntest)
        self._chk(lib().mg_get_stds(self.h, ptr(out)))
        return out

    def test_data(self):
        out = np.zeros((3, self.ntest))  # ntest x 3 column-major
        self._chk(lib().mg_get_test_data(self.h, ptr(out)))
        return out.T.copy()

    def mean_value(self):
        m = np.zeros(1)
        self._chk(lib().mg_get_dims(self.h, None, None, None, None, ptr(m)))
        return float(m[0])

    def stats(self):
        st = MgStats()
        self._chk(lib().mg_get_stats(self.h, C.byref(st)))
        return {"sweeps": st.sweeps, "retries": list(st.retries),
                "rows_sampled": list(st.rows_sampled), "cg_iters": list(st.cg_iters),
                "graph_captured": bool(st.graph_captured),
                "kernel_launches": int(st.kernel_launches), "h2d_bytes": int(st.h2d_bytes),
                "d2h_bytes": int(st.d2h_bytes), "ntasks": list(st.ntasks), "nnz": list(st.nnz)}


    def set_row_range(self, mode, lo, hi):
        """Rows [lo, hi) of `mode` are the ones this context samples (mg_set_row_range)."""
        self._chk(lib().mg_set_row_range(self.h, int(mode), int(lo), int(hi)))

    def latents_device(self, mode):
        """(device pointer, row stride in elements, element bytes) of the mode's latents."""
        ptr, stride, eb = C.c_void_p(), C.c_int(), C.c_int()
        self._chk(lib().mg_latents_device(self.h, int(mode), C.byref(ptr), C.byref(stride),
                                          C.byref(eb)))
        return ptr.value, stride.value, eb.value

    def latents_changed(self, mode):
        self._chk(lib().mg_latents_changed(self.h, int(mode)))

    def stream(self):
        s = C.c_void_p()
        self._chk(lib().mg_get_stream(self.h, C.byref(s)))
        return s.value or 0

    def autotune(self, use_cache=True):
        """Times the row samplers' candidate work splits and CTA shapes and keeps the fastest
        (mg_autotune); returns tuning()."""
        self._chk(lib().mg_autotune(self.h, 1 if use_cache else 0))
        return self.tuning()

    _TUNE_STATES = ("default", "timed", "cached")

    def tuning(self):
        """Per mode: the sampler's split threshold, CTA shape and the autotuner's record."""
        out = []
        for m in (0, 1):
            t = MgTuning()
            self._chk(lib().mg_get_tuning(self.h, m, C.byref(t)))
            out.append({"split_threshold": int(t.split_threshold), "cta_groups": t.cta_groups,
                        "tensor_core": bool(t.tensor_core), "state": self._TUNE_STATES[t.state],
                        "candidates": t.candidates, "ms_best": t.ms_best,
                        "ms_default": t.ms_default})
        return out


class Batch:
    """Many independent BPMF chains sampled together (mg_batch): problem p is the matrix
    problems[p] = dict(rows, cols, vals, trows, tcols, tvals, shape) with latent dimension
    num_latent[p] <= 32 and seed seeds[p]; mixed precision."""

    def __init__(self, problems, num_latent, seeds, precision, device=0):
        P = len(problems)
        self.P = P
        self.K = [int(k) for k in num_latent]
        self.shapes = [tuple(int(x) for x in pr["shape"]) for pr in problems]
        nr = np.array([s[0] for s in self.shapes], np.int32)
        nc = np.array([s[1] for s in self.shapes], np.int32)
        kk = np.array(self.K, np.int32)
        sd = np.array([int(x) & (2**64 - 1) for x in seeds], np.uint64)
        h = _p()
        code = lib().mg_batch_create(C.byref(h), P, ptr(nr), ptr(nc), ptr(kk), ptr(sd),
                                     float(precision), int(device))
        if code != 0:
            raise MacauError(code, lib().mg_batch_last_error(None).decode())
        self.h = h

        def cat(key, dtype):
            return np.ascontiguousarray(np.concatenate([np.asarray(pr[key], dtype) for pr in problems]))

        def offs(key):
            return np.concatenate([[0], np.cumsum([len(pr[key]) for pr in problems])]).astype(np.int64)

        a = [cat("rows", np.int32), cat("cols", np.int32), cat("vals", np.float64),
             cat("trows", np.int32), cat("tcols", np.int32), cat("tvals", np.float64)]
        to, eo = offs("vals"), offs("tvals")
        self._chk(lib().mg_batch_set_data(self.h, ptr(to), ptr(a[0]), ptr(a[1]), ptr(a[2]),
                                          ptr(eo), ptr(a[3]), ptr(a[4]), ptr(a[5])))

    def _chk(self, code):
        if code != 0:
            cls = CholeskyError if code == -2 else MacauError
            raise cls(code, lib().mg_batch_last_error(self.h).decode())

    def init(self, burnin=0):
        self._chk(lib().mg_batch_init(self.h, int(burnin)))

    def sweeps(self, first, count, eval=True):
        self._chk(lib().mg_batch_sweeps(self.h, int(first), int(count), int(bool(eval))))

    def time_sweeps(self, first, count):
        sec = C.c_double(0.0)
        self._chk(lib().mg_batch_time_sweeps(self.h, int(first), int(count), C.byref(sec)))
        return sec.value

    def latents(self, p, mode):
        out = np.zeros((self.shapes[p][mode], self.K[p]))
        self._chk(lib().mg_batch_get_latents(self.h, int(p), int(mode), ptr(out)))
        return out

    def rmse(self):
        out = np.zeros(2 * self.P)
        self._chk(lib().mg_batch_get_rmse(self.h, ptr(out)))
        return out.reshape(self.P, 2)

    def autotune(self, use_cache=True):
        """Times the batched sampler's candidate work splits and finish grids and keeps the
        fastest (mg_batch_autotune); returns tuning()."""
        self._chk(lib().mg_batch_autotune(self.h, 1 if use_cache else 0))
        return self.tuning()

    def tuning(self):
        out = []
        for m in (0, 1):
            t = MgTuning()
            self._chk(lib().mg_batch_get_tuning(self.h, m, C.byref(t)))
            out.append({"split_threshold": int(t.split_threshold),
                        "finish_ctas_per_sm": t.finish_ctas_per_sm,
                        "state": Sampler._TUNE_STATES[t.state], "candidates": t.candidates,
                        "ms_best": t.ms_best, "ms_default": t.ms_default})
        return out

    def info(self):
        out = np.zeros(5, np.int64)
        self._chk(lib().mg_batch_get_info(self.h, ptr(out)))
        return dict(rows=int(out[0]), cols=int(out[1]), nnz=int(out[2]),
                    retries=[int(out[3]), int(out[4])])

    def close(self):
        if getattr(self, "h", None):
            lib().mg_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()


def blockcg_raw(rows, cols, vals, shape, B, reg, tol, compute=MG_COMPUTE_FP64):
    """Runs mg_blockcg: B is (nrhs, nfeat); returns (X (nrhs, nfeat), niter, seconds)."""
    rows = np.ascontiguousarray(rows, np.int32)
    cols = np.ascontiguousarray(cols, np.int32)
    vals = None if vals is None else np.ascontiguousarray(vals, np.float64)
    B = np.asfortranarray(B, np.float64)
    nrhs, nfeat = B.shape
    X = np.zeros((nrhs, nfeat), order="F")
    it = C.c_int(0)
    sec = C.c_double(0)
    code = lib().mg_blockcg(ptr(rows), ptr(cols), ptr(vals), len(rows), int(shape[0]),
                            int(shape[1]), B.ctypes.data, nrhs, float(reg), float(tol),
                            int(compute), X.ctypes.data, C.byref(it), C.byref(sec))
    check(code, None)
    return X, it.value, sec.value
