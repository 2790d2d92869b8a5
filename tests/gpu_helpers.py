"""Shared set-up of GPU-vs-oracle parity tests: the same workload fed to the CUDA library (through
its C ABI) and to the CPU oracle (CSR built independently with scipy)."""
import numpy as np
import scipy.sparse as sp

from macau_b200 import _lib
from oracle import oracle as orc


def relerr(a, b):
    """Norm-wise relative error max|a-b| / max|b|."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    den = max(np.abs(b).max(), 1e-300)
    return float(np.abs(a - b).max() / den)


def train_matrix(w):
    Y = sp.coo_matrix((w["vals"], (w["rows"], w["cols"])), shape=w["shape"]).tocsc()
    Y.sum_duplicates()
    Y.sort_indices()
    return Y


def oracle_model(w, K, alpha, seed, lambda_beta=5.0, tol=1e-6):
    Y = train_matrix(w)
    mean = float(np.sum(Y.data)) / Y.nnz
    m = orc.Model(K, alpha, seed)
    m.set_train(orc.Csr.from_scipy(Y), orc.Csr.from_scipy(Y.T), mean)
    if len(w.get("tvals", [])):
        T = sp.coo_matrix((w["tvals"], (w["trows"], w["tcols"])), shape=w["shape"]).tocsc()
        T.sum_duplicates()
        T.sort_indices()
        Tc = T.tocoo()
        m.set_test(Tc.row, Tc.col, Tc.data)
    if "side" in w:
        fr, fc, fv, shp = w["side"]
        F = sp.coo_matrix((np.ones(len(fr)) if fv is None else fv, (fr, fc)), shape=shp)
        binary = fv is None
        m.set_side(0, orc.Csr.from_scipy(F, binary), orc.Csr.from_scipy(F.T, binary),
                   lambda_beta, tol)
    return m


def gpu_sampler(w, K, alpha, seed, compute=_lib.MG_COMPUTE_FP64, burnin=0, nsamples=1,
                lambda_beta=5.0, tol=1e-6, init=True):
    s = _lib.Sampler(K, alpha, seed=seed, compute=compute)
    s.set_relation_data(w["rows"], w["cols"], w["vals"], w["shape"])
    if len(w.get("tvals", [])):
        s.set_relation_data_test(w["trows"], w["tcols"], w["tvals"], w["shape"])
    if "side" in w:
        fr, fc, fv, shp = w["side"]
        s.set_side(0, fr, fc, fv, shp, lambda_beta, tol)
    s.set_samples(burnin, nsamples)
    if init:
        s.init()
    return s


def random_spd(rng, K, scale=1.0):
    A = rng.normal(size=(K, K))
    return scale * (A @ A.T / K + np.eye(K))
