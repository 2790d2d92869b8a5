"""The Python mirror of macau.macau() / macau.bpmf() on the GPU, along the lines of the
reference's own Python tests (python/macau/test_macau.py): result shapes and column names for
BPMF, Macau with sparse / binary / dense side information, the univariate sampler, adaptive
noise and empty test sets, plus a learning check on a low-rank matrix for each prior."""
import numpy as np
import pandas as pd
import pytest
import scipy.sparse as sp

import macau_b200

pytestmark = pytest.mark.gpu


def rand(nrow, ncol, density, seed):
    return sp.random(nrow, ncol, density=density, format="coo", random_state=seed)


@pytest.mark.parametrize("compute", ["fp64", "mixed"])
def test_bpmf_prediction_frame(compute):  # test_macau.py:9-16
    Y, Ytest = macau_b200.make_train_test(rand(10, 20, 0.2, 1), 0.5, seed=1)
    r = macau_b200.bpmf(Y, Ytest=Ytest, num_latent=4, verbose=False, burnin=50, nsamples=50,
                        univariate=False, seed=3, compute=compute)
    assert r.prediction.shape[0] == Ytest.nnz
    assert list(r.prediction.columns[0:2]) == ["row", "col"]
    assert np.isfinite(r.rmse_test)


def test_bpmf_numeric_test_fraction():  # test_macau.py:18-21
    macau_b200.bpmf(rand(15, 10, 0.2, 2), 0.3, num_latent=10, burnin=10, nsamples=15,
                    verbose=False, seed=1)


def test_macau_sparse_sides():  # test_macau.py:23-32
    rng = np.random.default_rng(0)
    Y, Ytest = macau_b200.make_train_test(rand(10, 20, 0.2, 3), 0.5, seed=2)
    side1 = sp.coo_matrix(rng.random((10, 2)))
    side2 = sp.coo_matrix(rng.random((20, 3)))
    r = macau_b200.macau(Y, Ytest=Ytest, side=[side1, side2], num_latent=4, verbose=False,
                         burnin=50, nsamples=50, univariate=False, seed=4)
    assert r.prediction.shape[0] == Ytest.nnz


def test_macau_binary_and_dense_sides():  # test_macau.py:34-45
    rng = np.random.default_rng(1)
    F = rand(15, 2, 0.5, 5).tocsr()
    F.data[:] = 1
    macau_b200.macau(rand(15, 10, 0.2, 6), rand(15, 10, 0.1, 7), side=[F, None], num_latent=5,
                     burnin=10, nsamples=5, verbose=False, seed=5)
    macau_b200.macau(rand(15, 10, 0.2, 8), rand(15, 10, 0.1, 9), side=[rng.normal(size=(15, 2)),
                                                                    None],
                     num_latent=5, burnin=10, nsamples=5, verbose=False, seed=6)


@pytest.mark.parametrize("compute", ["fp64", "mixed"])
def test_univariate_sides(compute):  # test_macau.py:64-73
    rng = np.random.default_rng(2)
    Y, Ytest = macau_b200.make_train_test(rand(10, 20, 0.2, 10), 0.5, seed=3)
    side1 = sp.coo_matrix(rng.random((10, 2)))
    side2 = sp.coo_matrix(rng.random((20, 3)))
    r = macau_b200.bpmf(Y, Ytest=Ytest, side=[side1, side2], num_latent=4, verbose=False,
                        burnin=50, nsamples=50, univariate=True, seed=7, compute=compute)
    assert r.prediction.shape[0] == Ytest.nnz


def test_empty_test_sets():  # test_macau.py:80-82, 209-222
    X = rand(15, 10, 0.2, 11)
    r = macau_b200.bpmf(X, Ytest=0, num_latent=10, burnin=10, nsamples=15, verbose=False, seed=8)
    assert np.isnan(r.rmse_test)
    df = pd.DataFrame({"A": X.row, "B": X.col, "value": X.data})
    r0 = macau_b200.macau(df, Ytest=0, num_latent=2, burnin=5, nsamples=5, precision=1.0,
                          verbose=False, seed=9)
    r1 = macau_b200.macau(df, Ytest=None, num_latent=2, burnin=5, nsamples=5, precision=1.0,
                          verbose=False, seed=9)
    assert np.isnan(r0.rmse_test) and np.isnan(r1.rmse_test)


def low_rank(seed, nrow=300, ncol=200, rank=3, sd=0.3, density=0.3):
    rng = np.random.default_rng(seed)
    U = rng.normal(size=(nrow, rank))
    V = rng.normal(size=(ncol, rank))
    mask = rng.random((nrow, ncol)) < density
    r, c = np.nonzero(mask)
    y = np.sum(U[r] * V[c], axis=1) + rng.normal(scale=sd, size=len(r))
    Y = sp.coo_matrix((y, (r, c)), shape=(nrow, ncol))
    F = sp.csr_matrix(np.hstack([U + rng.normal(scale=0.5, size=U.shape), np.ones((nrow, 1))]))
    return Y, F


@pytest.mark.parametrize("compute", ["fp64", "mixed"])
@pytest.mark.parametrize("variant", ["bpmf", "univariate", "adaptive"])
def test_low_rank_matrix_is_learned(variant, compute):
    Y, F = low_rank(4)
    Ytr, Yte = macau_b200.make_train_test(Y, 0.1, seed=5)
    kw = dict(num_latent=8, burnin=100, nsamples=100, verbose=False, seed=11, compute=compute)
    if variant == "univariate":
        r = macau_b200.macau(Ytr, Yte, side=[F, None], univariate=True, precision=1 / 0.09, **kw)
    elif variant == "adaptive":
        r = macau_b200.macau(Ytr, Yte, precision="adaptive", sn_max=100.0, **kw)
    else:
        r = macau_b200.bpmf(Ytr, Yte, precision=1 / 0.09, **kw)
    assert r.rmse_test < 0.45, r.rmse_test


def test_autotuned_run_draws_the_same_chain():
    # the autotuner only reshapes the work of the row samplers; with no row long enough to be
    # split, the FP64 chain is the same draw for draw
    Y, F = low_rank(4)
    Ytr, Yte = macau_b200.make_train_test(Y, 0.1, seed=5)
    kw = dict(num_latent=8, burnin=20, nsamples=20, verbose=False, seed=11, compute="fp64",
              precision=1 / 0.09)
    a = macau_b200.bpmf(Ytr, Yte, **kw)
    b = macau_b200.bpmf(Ytr, Yte, autotune=True, **kw)
    assert abs(a.rmse_test - b.rmse_test) < 1e-9
    np.testing.assert_allclose(a.prediction["y_pred"], b.prediction["y_pred"], rtol=1e-9)


def _read_csv_checked(path):
    """A model file of writeToCSVfile (bpmfutils.h:169-173): lines of ','-joined values, six
    significant digits (the %.6g form of C++'s default stream format), no trailing newline."""
    text = path.read_text()
    assert not text.endswith("\n")
    rows = [line.split(",") for line in text.split("\n")]
    for row in rows:
        for tok in row:
            assert format(float(tok), ".6g") == tok, tok
    return np.array([[float(t) for t in row] for row in rows])


def test_save_prefix_writes_the_reference_model_files(tmp_path):
    # MacauX::saveGlobalParams / saveModel (macau.cpp:191-205), BPMFPrior / MacauPrior::saveModel
    # (latentprior.cpp:307-315): file names, K x N shapes, six significant digits, and the last
    # sample's values against the same chain run through the C ABI
    from macau_b200 import _lib
    rng = np.random.default_rng(5)
    nrow, ncol, nfeat, K, burnin, nsamples, seed = 120, 80, 30, 6, 2, 3, 9
    Y, Ytest = macau_b200.make_train_test(rand(nrow, ncol, 0.25, 6), 0.2, seed=3)
    F = sp.random(nrow, nfeat, density=0.1, format="coo", random_state=7)
    F.data[:] = 1.0
    prefix = tmp_path / "model"
    macau_b200.macau(Y, Ytest=Ytest, side=[F, None], num_latent=K, precision=2.0, burnin=burnin,
                     nsamples=nsamples, save_prefix=str(prefix), verbose=False, seed=seed)
    want = {"model-meanvalue.csv"}
    for n in range(1, nsamples + 1):
        for m in (1, 2):
            want |= {f"model-sample{n}-U{m}-latents.csv", f"model-sample{n}-U{m}-latentmean.csv"}
        want.add(f"model-sample{n}-U1-link.csv")
    assert {p.name for p in tmp_path.iterdir()} == want
    last = f"model-sample{nsamples}-"
    U = _read_csv_checked(tmp_path / (last + "U1-latents.csv"))
    V = _read_csv_checked(tmp_path / (last + "U2-latents.csv"))
    mu = _read_csv_checked(tmp_path / (last + "U1-latentmean.csv"))
    link = _read_csv_checked(tmp_path / (last + "U1-link.csv"))
    mean = _read_csv_checked(tmp_path / "model-meanvalue.csv")
    assert U.shape == (K, nrow) and V.shape == (K, ncol)
    assert mu.shape == (K, 1) and link.shape == (K, nfeat) and mean.shape == (1, 1)
    Yc = Y.tocoo()
    Tc = Ytest.tocoo()
    s = _lib.Sampler(K, 2.0, seed=seed)
    s.set_relation_data(Yc.row, Yc.col, Yc.data, Y.shape)
    s.set_relation_data_test(Tc.row, Tc.col, Tc.data, Y.shape)
    s.set_side(0, F.row, F.col, None, F.shape, 5.0, 1e-6)
    s.set_samples(burnin, nsamples)
    s.init()
    s.sweeps(0, burnin + nsamples, eval=True)
    for got, ref in ((U, s.latents(0).T), (V, s.latents(1).T), (mu[:, 0], s.hyper(0)[0]),
                     (link, s.beta(0).T),
                     (mean[0, 0], s.mean_value())):
        ref = np.asarray(ref)
        assert np.all(np.abs(got - ref) <= 5.01e-6 * np.abs(ref))
    s.close()
