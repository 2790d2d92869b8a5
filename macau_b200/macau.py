"""Python entry points mirroring the reference's Cython module (python/macau/macau.pyx).

``macau()``, ``bpmf()``, ``blockcg()``, ``make_train_test()``, ``make_train_test_df()`` and
``MacauResult`` keep the reference's names, argument meaning, validation and error types
(macau.pyx:67-152, 221-451).  The Gibbs sweeps run on the GPU through the C ABI of
include/macau_b200.h; there is no CPU fallback.

Supported by the GPU sampler (the hot path): a 2-mode sparse matrix or 2-index-column
DataFrame, fixed Gaussian noise (numeric ``precision``) or adaptive Gaussian noise
(``precision="adaptive"``), BPMF priors and Macau priors with sparse or dense side information
(block-CG; the reference switches to a direct FtF Cholesky solve when a side matrix has at most
10000 columns, macau.pyx:160, which solves the same system), and with ``univariate=True`` the
univariate MacauOnePrior for sparse side information (macau.pyx:194-214).  Tensors and
``precision="probit"`` raise ValueError.

Two keyword arguments are added: ``seed`` (key of all random draws; the reference is
unseeded) and ``compute`` ("fp64" or "mixed"; default from the MACAU_GPU_PRECISION environment
variable, else "fp64").
"""
import numbers
import os
import signal
import sys
import threading

import numpy as np
import pandas as pd
import scipy.sparse

from . import _lib

_MATRIX_TYPES = (scipy.sparse.coo_matrix, scipy.sparse.csr_matrix, scipy.sparse.csc_matrix)


class MacauResult(object):
    """Result of macau(): rmse_test, auc_test, Yshape, ntrain, ntest, prediction (macau.pyx:12-22)."""

    def __init__(self):
        pass

    def __repr__(self):
        s = ("Matrix factorization results\n" +
             "Test RMSE:        %.4f\n" % self.rmse_test +
             "Matrix size:      [%s]\n" % " x ".join([str(x) for x in self.Yshape]) +
             "Number of train:  %d\n" % self.ntrain +
             "Number of test:   %d\n" % self.ntest +
             "To see predictions on test set see '.prediction' field.")
        return s


def _is_matrix(Y):
    return isinstance(Y, _MATRIX_TYPES) or (hasattr(scipy.sparse, "sparray") and
                                           isinstance(Y, scipy.sparse.sparray) and
                                           Y.format in ("coo", "csr", "csc"))


def _holdout_split(n, ntest, seed):
    """Random train / test positions among n items: ntest < 1 is a fraction of n, otherwise a
    count (rounded).  Returns (train positions, test positions)."""
    if not isinstance(ntest, numbers.Real) or ntest < 0:
        raise TypeError("ntest has to be a non-negative number (number or ratio of test samples).")
    count = int(round(n * ntest if ntest < 1 else ntest))
    order = (np.random if seed is None else np.random.default_rng(seed)).permutation(n)
    return order[count:], order[:count]


def make_train_test(Y, ntest, seed=None):
    """Random holdout of the observed cells of a sparse matrix.

    Y: a scipy sparse matrix (COO, CSR or CSC).  ntest: a fraction in [0, 1) of the cells, or a
    number of cells, that go to the test matrix.  seed: None uses numpy's global generator.
    Returns the train and test matrices as COO matrices of Y's shape.  Same arguments and
    errors as the reference's make_train_test (macau.pyx:109-130)."""
    if not _is_matrix(Y):
        raise TypeError("Unsupported Y type: %s" % type(Y))
    C = Y.tocoo(copy=False)
    tr, te = _holdout_split(C.nnz, ntest, seed)

    def pick(idx):
        return scipy.sparse.coo_matrix((C.data[idx], (C.row[idx], C.col[idx])), shape=C.shape)
    return pick(tr), pick(te)


def make_train_test_df(Y, ntest, seed=None):
    """Random holdout of the rows of a DataFrame of (index columns..., value) records; ntest as
    in make_train_test.  Returns the train and test frames (macau.pyx:132-152)."""
    if type(Y) != pd.core.frame.DataFrame:
        raise TypeError("Y should be DataFrame.")
    tr, te = _holdout_split(Y.shape[0], ntest, seed)
    return Y.iloc[tr], Y.iloc[te]


def remove_nan(Y):
    """Drops the cells of a COO matrix whose value is NaN (returns Y itself when none is)."""
    keep = ~np.isnan(Y.data)
    if keep.all():
        return Y
    return scipy.sparse.coo_matrix((Y.data[keep], (Y.row[keep], Y.col[keep])), shape=Y.shape)


class Data:
    """Training and test data as index arrays and values, from a sparse matrix pair or a
    DataFrame pair; the checks and their messages are those of the reference's Python entry
    (macau.pyx:242-306).  A number for Ytest holds out that fraction / count of Y."""

    def __init__(self, Y, Ytest):
        if _is_matrix(Y):
            self._from_matrices(Y, Ytest)
        elif type(Y) == pd.core.frame.DataFrame:
            self._from_frames(Y, Ytest)
        else:
            raise TypeError("Unsupported Y type: %s" % type(Y))

    def _from_matrices(self, Y, Ytest):
        if Ytest is None:
            Ytest = scipy.sparse.coo_matrix(Y.shape, dtype=np.float64)
        if isinstance(Ytest, numbers.Real):
            Y, Ytest = make_train_test(Y, Ytest)
        if not _is_matrix(Ytest):
            raise ValueError("When Y is a sparse matrix Ytest must be too.")
        if Y.shape != Ytest.shape:
            raise ValueError("Y (%d x %d) and Ytest (%d x %d) must have the same shape." %
                             (Y.shape[0], Y.shape[1], Ytest.shape[0], Ytest.shape[1]))
        tr = remove_nan(Y.tocoo(copy=False))
        te = remove_nan(Ytest.tocoo(copy=False))
        self.shape = np.array(tr.shape, dtype=np.int32)
        self.idxTrain, self.valTrain = [tr.row, tr.col], tr.data
        self.idxTest, self.valTest = [te.row, te.col], te.data
        self.colnames = np.array(["row", "col"], dtype=object)

    def _from_frames(self, Y, Ytest):
        if Ytest is None:
            Ytest = Y[0:0]
        if isinstance(Ytest, numbers.Real):
            Y, Ytest = make_train_test_df(Y, Ytest)
        if type(Ytest) != pd.core.frame.DataFrame:
            raise TypeError("When Y is a DataFrame Ytest must be too.")
        if (Y.columns != Ytest.columns).any():
            raise ValueError("Columns of Y and Ytest must be the same.")
        if (Y.dtypes != Ytest.dtypes).any():
            raise TypeError("Y.dtypes and Ytest.dtypes must be the same.")
        index_cols = [c for c in Y.columns if Y[c].dtype in (np.int64, np.int32)]
        value_cols = [c for c in Y.columns if Y[c].dtype in (np.float32, np.float64)]
        if len(index_cols) > 10:
            raise ValueError("Y has too many index(int) columns (%d), maximum is 10." % len(index_cols))
        if len(index_cols) < 2:
            raise ValueError("Y must have at least 2 index (int) columns.")
        if len(value_cols) != 1:
            raise ValueError("Y has %d float columns but must have exactly 1 value column." % len(value_cols))
        if Y.shape[0] == 0:
            raise ValueError("Ytrain must not be empty.")
        # each mode's size is one more than the largest index seen in train or test
        largest = np.array([Y[c].max() for c in index_cols])
        if Ytest.shape[0] > 0:
            largest = np.maximum(largest, [Ytest[c].max() for c in index_cols])
        self.shape = np.array(largest + 1, dtype=np.int32)
        self.colnames = index_cols
        self.idxTrain = [np.array(Y[c], dtype=np.int32) for c in index_cols]
        self.idxTest = [np.array(Ytest[c], dtype=np.int32) for c in index_cols]
        self.valTrain = np.array(Y[value_cols[0]], dtype=np.float64)
        self.valTest = np.array(Ytest[value_cols[0]], dtype=np.float64)


def _side_coo(s, nrows):
    """Side information -> (rows, cols, vals or None for binary, shape); make_prior's accepted
    types (macau.pyx:154-192)."""
    if _is_matrix(s):
        m = s.tocoo(copy=False)
        vals = np.asarray(m.data, np.float64)
        binary = bool(np.all(vals == 1.0))
        return m.row, m.col, (None if binary else vals), m.shape
    if isinstance(s, np.ndarray):
        if len(s.shape) != 2:
            raise TypeError("Side information must have 2 dimensions (got %d)." % len(s.shape))
        m = scipy.sparse.coo_matrix(s.astype(np.float64, copy=False))
        return m.row, m.col, np.asarray(m.data, np.float64), s.shape
    raise TypeError("Unsupported side information type: '%s'" % type(s).__name__)


class _StopOnInterrupt(object):
    """Ctrl-C during the sweeps: the reference's SIGINT handler (macau.cpp:30-35) prints a note
    and the run stops after the current iteration (macau.cpp:111-114), returning the results so
    far.  Installed only from the main thread; the previous handler is put back on exit (the
    reference's caller restores Python's default one, macau.pyx:421)."""

    MESSAGE = "[Received Ctrl-C. Stopping after finishing the current iteration.]"

    def __init__(self):
        self.requested = False
        self._installed = False
        self._previous = None

    def _handler(self, signum, frame):
        self.requested = True
        print(self.MESSAGE)
        sys.stdout.flush()

    def __enter__(self):
        if threading.current_thread() is threading.main_thread():
            self._previous = signal.signal(signal.SIGINT, self._handler)
            self._installed = True
        return self

    def __exit__(self, *exc):
        if self._installed:
            # None: the previous handler was not set from Python; fall back to Python's default
            prev = self._previous if self._previous is not None else signal.default_int_handler
            signal.signal(signal.SIGINT, prev)
            self._installed = False
            self._previous = None
        return False


def _compute_mode(compute):
    if compute is None:
        compute = os.environ.get("MACAU_GPU_PRECISION", "fp64")
    if compute in ("fp64", _lib.MG_COMPUTE_FP64):
        return _lib.MG_COMPUTE_FP64
    if compute in ("mixed", _lib.MG_COMPUTE_MIXED):
        return _lib.MG_COMPUTE_MIXED
    raise ValueError("compute must be 'fp64' or 'mixed' (got %r)" % (compute,))


def _write_csv(path, M):
    """writeToCSVfile (bpmfutils.h:169-173): rows of M, 6 significant digits."""
    M = np.atleast_2d(M)
    with open(path, "w") as f:
        f.write("\n".join(",".join("%.6g" % v for v in row) for row in M))


def bpmf(Y, Ytest=None, num_latent=10, precision=1.0, burnin=50, nsamples=400, **keywords):
    """BPMF without side information (macau.pyx:221-234)."""
    return macau(Y, Ytest=Ytest, num_latent=num_latent, precision=precision, burnin=burnin,
                 nsamples=nsamples, **keywords)


def macau(Y,
          Ytest=None,
          side=[],
          lambda_beta=5.0,
          num_latent=10,
          precision=1.0,
          burnin=50,
          nsamples=400,
          univariate=False,
          tol=1e-6,
          sn_max=10.0,
          save_prefix=None,
          verbose=True,
          seed=None,
          compute=None,
          autotune=False):
    """
    Matrix factorization with side information, sampled on a B200 GPU.
      Y          training data to factorize (sparse matrix or DataFrame)
      Ytest      either:
                 number below 1.0, how much training data to move to test
                 sparse matrix or DataFrame of test data
      side       list of side information matrices (one per mode, None = no side info)
      lambda_beta  initial precision (regularization) for the link matrix
      num_latent   number of latent dimensions
      precision    precision of observations of Y:
                   number     - fixed Gaussian noise
                   "adaptive" - automatically learn precision (also "sample")
      burnin       number of Gibbs samples to drop (burn-in)
      nsamples     number of Gibbs samples to collect
      univariate   whether to use univariate sampler (faster than standard sampler)
      tol          error tolerance for conjugate gradient solver
      sn_max       maximum signal-to-noise ratio for observation precision
                   only used if precision="adaptive"
      save_prefix  prefix for model files or None if not saving the model
      verbose      whether to print output for each Gibbs iteration
      seed         key of all random draws (None: drawn from the OS)
      compute      "fp64" or "mixed" (BF16/FP32 tensor-core sampler), default from
                   MACAU_GPU_PRECISION or "fp64"
      autotune     time the row samplers' work splits and CTA shapes on this data before
                   sampling and keep the fastest (choices cached per process, and in the file
                   named by MACAU_B200_TUNE_CACHE if set); the draws are unchanged
    """
    data = Data(Y, Ytest)

    if not side:
        side = [None for i in range(len(data.shape))]
    if type(side) not in [list, tuple]:
        raise ValueError("Parameter 'side' must be a tuple or a list.")
    if len(side) != len(data.shape):
        raise ValueError("Length of 'side' is %d but must be equal to the number of data dimensions (%d)." %
                         (len(side), len(data.shape)))
    if len(data.shape) != 2:
        raise ValueError("Tensor data (%d modes) is not supported by the GPU sampler." % len(data.shape))
    adaptive = False
    if isinstance(precision, str):
        if precision in ("adaptive", "sample"):  # make_macau_adaptive(Nmodes, D, 1.0, sn_max) (macau.pyx:391-392)
            adaptive = True
        elif precision == "probit":
            raise ValueError("precision='probit' is not supported by the GPU sampler (Gaussian noise only).")
        else:
            raise ValueError("Parameter 'precision' has to be either a number or \"adaptive\" for adaptive precision, or \"probit\" for binary matrices.")
    if save_prefix is not None and type(save_prefix) != str:
        raise ValueError("Parameter 'save_prefix' has to be a string (str) or None.")
    if univariate:  # make_one_prior accepts sparse matrices only (macau.pyx:194-198)
        for sd in side:
            if sd is None or (isinstance(sd, tuple) and sd == ()):
                continue
            if not _is_matrix(sd):
                raise ValueError("Unsupported side information type: '%s'" % type(sd).__name__)

    if seed is None:
        seed = int.from_bytes(os.urandom(8), "little")
    D = int(np.int32(num_latent))
    s = _lib.Sampler(D, 1.0 if adaptive else float(precision), seed=seed,
                     compute=_compute_mode(compute), verbose=False)
    try:
        if adaptive:
            s.set_noise_adaptive(1.0, float(sn_max))
        if autotune:
            s.set_option("autotune", 1)
        s.set_relation_data(data.idxTrain[0], data.idxTrain[1], data.valTrain, data.shape)
        if len(data.valTest) > 0:
            s.set_relation_data_test(data.idxTest[0], data.idxTest[1], data.valTest, data.shape)
        for mode, sd in enumerate(side):
            if sd is None:
                continue
            if univariate and isinstance(sd, tuple) and sd == ():  # make_one_prior: () = none
                continue
            r, c, v, shp = _side_coo(sd, data.shape[mode])
            if shp[0] != data.shape[mode]:
                raise ValueError("Side information for mode %d has %d rows, expected %d." %
                                 (mode, shp[0], data.shape[mode]))
            if univariate:  # MacauOnePrior<SparseFeat | SparseDoubleFeat> (macau.pyx:194-214)
                s.set_side_univariate(mode, r, c, v, shp, lambda_beta)
            else:
                s.set_side(mode, r, c, v, shp, lambda_beta, tol)
        s.set_samples(int(burnin), int(nsamples))
        s.init()
        if verbose:
            if adaptive:  # AdaptiveGaussianNoise::getInitStatus (noisemodels.h:75)
                print("Noise precision: adaptive (with max precision of %f)" % s.noise()[1])
            else:
                print("Noise precision: %f (fixed)" % float(precision))
            print("Sampling")
        if save_prefix is not None:
            _write_csv(save_prefix + "-meanvalue.csv", [[s.mean_value()]])
        import time
        with _StopOnInterrupt() as stop:
            for i in range(burnin + nsamples):
                if stop.requested:
                    break
                if verbose and i == burnin:
                    print(" ====== Burn-in complete, averaging samples ====== ")
                t0 = time.time()
                s.sweep(i, eval=True)
                if save_prefix is not None and i >= burnin:
                    _save_sample(s, save_prefix, i - burnin + 1)
                if verbose:
                    r, r1 = s.rmse()
                    norms = [np.linalg.norm(s.latents(m)) for m in range(2)]
                    links = ["%1.2e" % np.linalg.norm(s.beta(m)) if s.nfeat[m] else "nan"
                             for m in range(2)]
                    prec = "Prec:%.2g" % s.noise()[0] if adaptive else ""  # noisemodels.h:77-79
                    # getEvalString (noisemodels.h:46): 5 significant digits, C++ ostream
                    # default format = %.5g
                    print("Iter %3d: RMSE: %.5g (1samp: %.5g)  U:[%1.2e, %1.2e]\tSide:[%s]%s [took %0.1fs]" %
                          (i, r, r1, norms[0], norms[1], ", ".join(links), prec, time.time() - t0))
                    sys.stdout.flush()
        rmse_test, _ = s.rmse()
        yhat = s.predictions()
        yhat_sd = s.stds()
        testdata = s.test_data()
    finally:
        s.close()

    df = pd.DataFrame(testdata[:, :-1].astype(int), columns=list(data.colnames))
    df["y"] = pd.Series(testdata[:, -1])
    df["y_pred"] = pd.Series(yhat)
    df["y_pred_std"] = pd.Series(yhat_sd)

    result = MacauResult()
    result.rmse_test = rmse_test if len(data.valTest) > 0 else np.nan
    result.auc_test = np.nan
    result.Yshape = data.shape
    result.ntrain = data.valTrain.shape[0]
    result.ntest = data.valTest.shape[0] if Ytest is not None else 0
    result.prediction = pd.DataFrame(df)
    return result


def _save_sample(s, prefix, isample):
    """MacauX::saveModel (macau.cpp:191-198): per-sample latents, latent means and links."""
    fp = "%s-sample%d-" % (prefix, isample)
    for m in range(2):
        _write_csv(fp + "U%d-latents.csv" % (m + 1), s.latents(m).T)
        mu, _, _ = s.hyper(m)
        _write_csv(fp + "U%d-latentmean.csv" % (m + 1), mu.reshape(-1, 1))
        if s.nfeat[m]:
            _write_csv(fp + "U%d-link.csv" % (m + 1), s.beta(m).T)


def blockcg(X, B, reg, tol=1e-6, compute=None):
    """macau.blockcg (macau.pyx:67-91): solves (X'X + reg I) W' = B' on the GPU for a binary
    sparse X and an order='F' B (nrhs x nfeat).  Returns [niter, seconds] like the reference;
    the solution is available through ``blockcg_solve``."""
    if not np.isfortran(B):
        raise ValueError("B must have order='F' (fortran)")
    if B.shape[1] != X.shape[1]:
        raise ValueError("B.shape[1] must equal X.shape[1]")
    _, it, sec = blockcg_solve(X, B, reg, tol, compute)
    v = np.zeros(2)
    v[0] = it
    v[1] = sec
    return v


def blockcg_solve(X, B, reg, tol=1e-6, compute=None, binary=True):
    """Like blockcg() but returns (W, niter, seconds); binary=False keeps X's values."""
    X = X.tocoo(copy=False)
    vals = None if binary else np.asarray(X.data, np.float64)
    return _lib.blockcg_raw(X.row, X.col, vals, X.shape, B, reg, tol, _compute_mode(compute))
