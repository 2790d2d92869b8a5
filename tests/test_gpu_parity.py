"""GPU parity of the CUDA library against the CPU oracle, through the C ABI.

Bar (FP64 mode): per-row samples, hyperparameters and beta within 1e-9 (norm-wise relative) of
the FP64 oracle fed the same keyed or injected N(0,1) draws.  Mixed mode: stated tolerances
against the same FP64 oracle."""
import json
from pathlib import Path

import numpy as np
import pytest
import scipy.sparse as sp

from macau_b200 import _lib, workloads
from oracle import oracle as orc
from tests.gpu_helpers import gpu_sampler, oracle_model, random_spd, relerr, train_matrix

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-9
MIXED_SAMPLE_TOL = 6e-3   # BF16 Gram + FP32 factor vs FP64, norm-wise relative per sweep


def small_uniform(seed=0, nrow=300, ncol=200, nobs=6000):
    return workloads.bpmf_uniform(nrow=nrow, ncol=ncol, nobs=nobs, seed=seed)


@pytest.mark.parametrize("K", [4, 10, 16, 32, 50, 64, 128])
@pytest.mark.parametrize("mode", [0, 1])
def test_row_sampler_fp64_injected_draws(K, mode):
    rng = np.random.default_rng(K + 100 * mode)
    w = small_uniform(seed=K)
    s = gpu_sampler(w, K, 4.0, seed=7)
    Y = train_matrix(w)
    other = 1 - mode
    Vo = rng.normal(scale=0.5, size=(w["shape"][other], K))
    s.set_latents(other, Vo)
    mu = rng.normal(size=K)
    Lam = random_spd(rng, K, 5.0)
    s.set_hyper(mode, mu, Lam)
    N = w["shape"][mode]
    z = rng.normal(size=(N, K))
    s.sample_latents(mode, 3, z)
    got = s.latents(mode)
    R = orc.Csr.from_scipy(Y if mode == 0 else Y.T)
    want, st = orc.sample_latents(K, R, Vo, s.mean_value(), 4.0, mu, Lam, z=z)
    assert st == 0
    assert relerr(got, want) < FP64_TOL


@pytest.mark.parametrize("K", [10, 32])
def test_row_sampler_fp64_keyed_draws(K):
    rng = np.random.default_rng(5)
    w = small_uniform(seed=1)
    s = gpu_sampler(w, K, 2.0, seed=12345)
    Y = train_matrix(w)
    V = rng.normal(scale=0.5, size=(w["shape"][1], K))
    s.set_latents(1, V)
    mu0, Lam0, _ = s.hyper(0)
    s.sample_latents(0, 17)
    want, _ = orc.sample_latents(K, orc.Csr.from_scipy(Y), V, s.mean_value(), 2.0, mu0, Lam0,
                                 seed=12345, sweep=17, mode=0)
    assert relerr(s.latents(0), want) < FP64_TOL


def test_row_sampler_split_heavy_rows():
    # rows with thousands of entries are split into parts and reduced by the last part
    rng = np.random.default_rng(9)
    nrow, ncol, K = 64, 4000, 32
    r, c = [], []
    for i in range(nrow):
        n = 3900 if i % 7 == 0 else rng.integers(1, 60)
        cols = rng.choice(ncol, size=n, replace=False)
        r += [i] * n
        c += list(cols)
    r = np.array(r, np.int32)
    c = np.array(c, np.int32)
    v = rng.normal(3.0, 1.0, size=len(r))
    w = dict(rows=r, cols=c, vals=v, shape=(nrow, ncol))
    s = gpu_sampler(w, K, 1.5, seed=3)
    V = rng.normal(scale=0.3, size=(ncol, K))
    s.set_latents(1, V)
    z = rng.normal(size=(nrow, K))
    mu, Lam, _ = s.hyper(0)
    s.sample_latents(0, 0, z)
    Y = train_matrix(w)
    want, _ = orc.sample_latents(K, orc.Csr.from_scipy(Y), V, s.mean_value(), 1.5, mu, Lam, z=z)
    assert relerr(s.latents(0), want) < FP64_TOL


@pytest.mark.parametrize("K", [3, 10, 32, 64])
def test_hyperprior_fp64(K):
    rng = np.random.default_rng(K)
    w = small_uniform(seed=2)
    s = gpu_sampler(w, K, 1.0, seed=99)
    U = rng.normal(0.3, 1.0, size=(w["shape"][0], K))
    s.set_latents(0, U)
    s.update_prior(0, 11)
    mu, Lam, _ = s.hyper(0)
    mu_o, Lam_o, st = orc.cond_normal_wishart(U, np.zeros(K), 2.0, np.eye(K), K, seed=99,
                                              sweep=11, mode=0)
    assert st == 0
    assert relerr(Lam, Lam_o) < FP64_TOL
    assert relerr(mu, mu_o) < FP64_TOL


def test_full_sweeps_fp64_match_oracle():
    w = workloads.bpmf_uniform(nrow=400, ncol=300, nobs=12000, seed=4)
    K, alpha, seed, burnin = 10, 4.0, 2024, 4
    s = gpu_sampler(w, K, alpha, seed, burnin=burnin, nsamples=6)
    m = oracle_model(w, K, alpha, seed)
    for it in range(10):
        s.sweep(it, eval=True)
        assert m.sweep(it, burnin) == 0
        for mode in (0, 1):
            assert relerr(s.latents(mode), m.latents(mode)) < 1e-8, (it, mode)
            mu, Lam, _ = s.hyper(mode)
            assert relerr(Lam, m.Lambda(mode)) < 1e-8
        r, r1 = s.rmse()
        ro, r1o = m.rmse()
        assert abs(r - ro) < 1e-9 and abs(r1 - r1o) < 1e-9
    np.testing.assert_allclose(s.predictions(), m.predictions(), rtol=1e-9, atol=1e-12)


def gpu_cg_parts(nfeat):
    """Number of contiguous row blocks of the CUDA block-CG's K x K reductions; the oracle is
    given the same partition (the reference's own depends on its OpenMP thread count,
    linop.cpp:280-317).  Within and across the blocks the two add in different orders, which the
    tolerances below absorb."""
    return min(296, max(1, -(-nfeat // 64)))


@pytest.fixture
def oracle_parts():
    yield orc.set_reduce_parts
    orc.set_reduce_parts(1)


def test_macau_update_prior_fp64_tight_tolerance(oracle_parts):
    # With the CG solved to 1e-12 the link matrix is determined to far below 1e-9, so the whole
    # MacauPrior::update_prior chain (Wishart, sample_beta RHS, CG, Uhat, lambda_beta) is
    # compared at the FP64 bar.
    w = workloads.macau_side(scale=0.02, seed=5)
    K, alpha, seed = 8, 1.0, 77
    s = gpu_sampler(w, K, alpha, seed, lambda_beta=5.0, tol=1e-12)
    m = oracle_model(w, K, alpha, seed, lambda_beta=5.0, tol=1e-12)
    oracle_parts(gpu_cg_parts(w["side"][3][1]))
    for it in range(2):
        for mode in (0, 1):
            s.sample_latents(mode, it)
            m.sample_mode(mode, it)
            m.set("latents", mode, s.latents(mode))  # identical inputs for the next phase
        s.update_prior(0, it)
        m.update_prior(0, it)
        mu, Lam, lb = s.hyper(0)
        assert relerr(Lam, m.Lambda(0)) < FP64_TOL
        assert relerr(mu, m.mu(0)) < FP64_TOL
        assert relerr(s.beta(0), m.beta(0)) < FP64_TOL, it
        assert relerr(s.uhat(0), m.uhat(0)) < FP64_TOL, it
        assert abs(lb - m.lambda_beta(0)[0]) / lb < FP64_TOL
        s.update_prior(1, it)
        m.update_prior(1, it)
        # carry the GPU's state into the oracle so the next sweep starts from identical inputs
        m.set("beta", 0, s.beta(0))
        m.set("uhat", 0, s.uhat(0))
        m.set("lambda_beta", 0, [lb])
        for mode in (0, 1):
            mu, Lam, _ = s.hyper(mode)
            m.set("mu", mode, mu)
            m.set("Lambda", mode, Lam)


def test_macau_side_sweeps_fp64_match_oracle(oracle_parts):
    # At the default tolerance (1e-6) block-CG's output is defined only to about the tolerance:
    # the oracle itself moves by ~1e-7 when its reduction order changes.  Full sweeps are
    # therefore compared at 1e-5 (CG-bounded), with identical iteration counts.
    w = workloads.macau_side(scale=0.02, seed=5)
    K, alpha, seed = 8, 1.0, 77
    s = gpu_sampler(w, K, alpha, seed, lambda_beta=5.0, tol=1e-6)
    m = oracle_model(w, K, alpha, seed, lambda_beta=5.0, tol=1e-6)
    oracle_parts(gpu_cg_parts(w["side"][3][1]))
    for it in range(3):
        s.sweep(it, eval=True)
        assert m.sweep(it, 10) == 0
        for mode in (0, 1):
            assert relerr(s.latents(mode), m.latents(mode)) < 1e-5, (it, mode)
        assert relerr(s.beta(0), m.beta(0)) < 1e-5, it
        assert relerr(s.uhat(0), m.uhat(0)) < 1e-5, it
        lbo, iters = m.lambda_beta(0)
        assert abs(s.hyper(0)[2] - lbo) / lbo < 1e-5
        assert abs(s.stats()["cg_iters"][0] - int(iters)) <= 1


FIX = json.loads((Path(__file__).parent / "golden" / "reference_tests_cpp.json").read_text())


def _case(name):
    env = {}
    for st in FIX["cases"][name]["statements"]:
        if st["kind"] == "array":
            env[st["name"]] = np.array(st["values"])
        elif st["kind"] == "matrix" and st["name"] not in env:
            env[st["name"]] = np.array(st["values"]).reshape(st["shape"])
    return env


@pytest.mark.parametrize("name", ["SparseFeat/solve_blockcg", "SparseFeat/solve_blockcg_1_0",
                                  "linop/solve_blockcg_dense"])
@pytest.mark.parametrize("compute", [_lib.MG_COMPUTE_FP64, _lib.MG_COMPUTE_MIXED])
def test_blockcg_golden_on_gpu(name, compute):  # tests.cpp:123-207
    env = _case(name)
    r = env["rows"].astype(np.int32)
    c = env["cols"].astype(np.int32)
    B = np.asfortranarray(env["B"])
    if name.endswith("_1_0"):  # blocksize 1: every RHS solved on its own
        X = np.vstack([_lib.blockcg_raw(r, c, None, (6, 4), B[i:i + 1], 0.5, 1e-6, compute)[0]
                       for i in range(B.shape[0])])
        it = 0
    else:
        X, it, _ = _lib.blockcg_raw(r, c, None, (6, 4), B, 0.5, 1e-6, compute)
    np.testing.assert_allclose(X, env["X_true"], rtol=2e-5, atol=2e-6)
    if name == "SparseFeat/solve_blockcg":
        assert it <= 4


@pytest.mark.parametrize("tol,bar", [(1e-12, FP64_TOL), (1e-6, 1e-5)])
def test_blockcg_matches_oracle_fp64(oracle_parts, tol, bar):
    # 32 right-hand sides over a Zipf-degree binary F.  At tol 1e-6 the solve is only defined to
    # about the tolerance (the oracle moves by ~1.5e-7 between reduction orders), so that case
    # is bounded by the CG tolerance; at tol 1e-12 the FP64 bar applies.
    w = workloads.macau_side(scale=0.05, seed=6)
    fr, fc, _, shp = w["side"]
    F = sp.coo_matrix((np.ones(len(fr)), (fr, fc)), shape=shp)
    rng = np.random.default_rng(1)
    B = rng.normal(size=(32, shp[1]))
    oracle_parts(gpu_cg_parts(shp[1]))
    Xo, ito = orc.blockcg(orc.Csr.from_scipy(F, True), orc.Csr.from_scipy(F.T, True), 3.0, B.T,
                          tol, 32, 8)
    X, it, _ = _lib.blockcg_raw(fr, fc, None, shp, B, 3.0, tol, _lib.MG_COMPUTE_FP64)
    assert abs(it - ito) <= 1
    assert relerr(X.T, Xo) < bar


def test_blockcg_iteration_cap_is_reported():
    # linop.h:279 stops at its iteration cap silently; here a solve that reaches the cap keeps
    # its last iterate, the prior update completes, and the call reports MG_ERR_CG; the context
    # carries on, and with the default cap the next sweep's solve converges
    w = workloads.macau_side(scale=0.02, seed=5)
    s = gpu_sampler(w, 8, 1.0, 77, tol=1e-10, init=False)
    s.set_option("cg_max_iter", 2)
    s.init()
    with pytest.raises(_lib.MacauError, match="did not converge within 2 iterations") as e:
        s.sweep(0, eval=False)
    assert e.value.code == _lib.MG_ERR_CG
    assert s.stats()["cg_iters"][0] == 2
    assert np.isfinite(s.beta(0)).all()
    s.set_option("cg_max_iter", 100000)
    s.sweep(1, eval=False)
    assert s.stats()["cg_iters"][0] > 2
    s.close()


def test_blockcg_fp32_with_fp64_residual_replacement():
    w = workloads.macau_side(scale=0.05, seed=6)
    fr, fc, _, shp = w["side"]
    F = sp.coo_matrix((np.ones(len(fr)), (fr, fc)), shape=shp)
    rng = np.random.default_rng(1)
    B = rng.normal(size=(32, shp[1]))
    Xd, itd, _ = _lib.blockcg_raw(fr, fc, None, shp, B, 3.0, 1e-6, _lib.MG_COMPUTE_FP64)
    Xf, itf, _ = _lib.blockcg_raw(fr, fc, None, shp, B, 3.0, 1e-6, _lib.MG_COMPUTE_MIXED)
    A = (F.T @ F).toarray() + 3.0 * np.eye(shp[1])
    res = np.linalg.norm(A @ Xf.T - B.T, axis=0) / np.linalg.norm(B.T, axis=0)
    assert res.max() < 1e-5
    assert relerr(Xf, Xd) < 1e-5
    assert itf <= 2 * itd


def test_mixed_row_sampler_within_tolerance():
    rng = np.random.default_rng(8)
    K = 32
    w = small_uniform(seed=3, nrow=500, ncol=300, nobs=20000)
    s = gpu_sampler(w, K, 2.0, seed=1, compute=_lib.MG_COMPUTE_MIXED)
    V = rng.normal(scale=0.3, size=(w["shape"][1], K))
    s.set_latents(1, V)
    mu, Lam, _ = s.hyper(0)
    z = rng.normal(size=(w["shape"][0], K))
    s.sample_latents(0, 0, z)
    Y = train_matrix(w)
    want, _ = orc.sample_latents(K, orc.Csr.from_scipy(Y), V, s.mean_value(), 2.0, mu, Lam, z=z)
    assert relerr(s.latents(0), want) < MIXED_SAMPLE_TOL


def heavy_rows_workload(rng, nrow=64, ncol=4000):
    """Rows 0, 7, 14, ... have 3,900 entries (split into parts by the samplers); the others 1-59."""
    r, c = [], []
    for i in range(nrow):
        n = 3900 if i % 7 == 0 else rng.integers(1, 60)
        cols = rng.choice(ncol, size=n, replace=False)
        r += [i] * n
        c += list(cols)
    r = np.array(r, np.int32)
    c = np.array(c, np.int32)
    return dict(rows=r, cols=c, vals=rng.normal(3.0, 1.0, size=len(r)), shape=(nrow, ncol))


@pytest.mark.parametrize("tensor_cores", [1, 0])
@pytest.mark.parametrize("mode", [0, 1])
def test_mixed_row_sampler_split_heavy_rows(tensor_cores, mode):
    # mixed precision at K = 32 through the tensor-core sampler (Gram records, split parts summed
    # by the finish kernel) and through the CUDA-core sampler, against the FP64 oracle
    rng = np.random.default_rng(19 + mode)
    K = 32
    w = heavy_rows_workload(rng)
    s = gpu_sampler(w, K, 1.5, seed=3, compute=_lib.MG_COMPUTE_MIXED)
    s.set_option("tensor_core_gram", tensor_cores)
    other = 1 - mode
    Vo = rng.normal(scale=0.3, size=(w["shape"][other], K))
    s.set_latents(other, Vo)
    z = rng.normal(size=(w["shape"][mode], K))
    mu, Lam, _ = s.hyper(mode)
    s.sample_latents(mode, 0, z)
    Y = train_matrix(w)
    R = orc.Csr.from_scipy(Y if mode == 0 else Y.T)
    want, _ = orc.sample_latents(K, R, Vo, s.mean_value(), 1.5, mu, Lam, z=z)
    assert relerr(s.latents(mode), want) < MIXED_SAMPLE_TOL


@pytest.mark.parametrize("K", [10, 32, 64])
@pytest.mark.parametrize("mode", [0, 1])
def test_mixed_row_sampler_keyed_draws(K, mode):
    # keyed draws (no injection): the mixed samplers draw the same z as the FP64 oracle
    rng = np.random.default_rng(K + 7 * mode)
    w = small_uniform(seed=5, nrow=400, ncol=250, nobs=15000)
    s = gpu_sampler(w, K, 2.0, seed=4242, compute=_lib.MG_COMPUTE_MIXED)
    other = 1 - mode
    Vo = rng.normal(scale=0.3, size=(w["shape"][other], K))
    s.set_latents(other, Vo)
    mu, Lam, _ = s.hyper(mode)
    s.sample_latents(mode, 9)
    Y = train_matrix(w)
    R = orc.Csr.from_scipy(Y if mode == 0 else Y.T)
    want, _ = orc.sample_latents(K, R, Vo, s.mean_value(), 2.0, mu, Lam, seed=4242, sweep=9,
                                 mode=mode)
    assert relerr(s.latents(mode), want) < MIXED_SAMPLE_TOL


# ---- adaptive Gaussian noise (AdaptiveGaussianNoise, noisemodels.cpp:14-33, 55-81) ----

def adaptive_pair(w, K, seed, sn_max=10.0, compute=_lib.MG_COMPUTE_FP64, burnin=0, nsamples=1):
    s = gpu_sampler(w, K, 1.0, seed, compute=compute, burnin=burnin, nsamples=nsamples,
                    init=False)
    s.set_noise_adaptive(1.0, sn_max)
    s.init()
    m = oracle_model(w, K, 1.0, seed)
    m.set_noise_adaptive(1.0, sn_max)
    return s, m


@pytest.mark.parametrize("sn_max", [10.0, 0.05])
def test_adaptive_noise_sweeps_fp64_match_oracle(sn_max):
    # whole sweeps (samplers at the current precision, priors, precision redraw, eval); with
    # sn_max = 0.05 the cap binds
    w = workloads.bpmf_uniform(nrow=400, ncol=300, nobs=12000, seed=6)
    K, seed, burnin = 10, 77, 4
    s, m = adaptive_pair(w, K, seed, sn_max, burnin=burnin, nsamples=6)
    a0, amax0, vt0 = m.noise()
    a, amax, vt = s.noise()
    assert abs(vt - vt0) <= 1e-12 * vt0 and abs(a - a0) <= 1e-12 * a0
    assert abs(amax - amax0) <= 1e-12 * amax0
    capped = 0
    for it in range(10):
        s.sweep(it, eval=True)
        assert m.sweep(it, burnin) == 0
        for mode in (0, 1):
            assert relerr(s.latents(mode), m.latents(mode)) < 1e-8, (it, mode)
            assert relerr(s.hyper(mode)[1], m.Lambda(mode)) < 1e-8
        a, ao = s.noise()[0], m.noise()[0]
        assert abs(a - ao) <= FP64_TOL * ao, (it, a, ao)
        capped += ao == amax0
        r, r1 = s.rmse()
        ro, r1o = m.rmse()
        assert abs(r - ro) < 1e-9 and abs(r1 - r1o) < 1e-9
    assert (capped > 0) == (sn_max < 1.0)


@pytest.mark.parametrize("compute", [_lib.MG_COMPUTE_FP64, _lib.MG_COMPUTE_MIXED])
def test_adaptive_noise_update_matches_oracle(compute):
    # the precision redraw alone from given latents (the mixed context keeps FP32 latents, so the
    # oracle gets the same FP32 values)
    rng = np.random.default_rng(31)
    w = small_uniform(seed=8, nrow=500, ncol=350, nobs=25000)
    K, seed = 32, 5
    s, m = adaptive_pair(w, K, seed, compute=compute)
    for it in (0, 3):
        U = rng.normal(scale=0.4, size=(w["shape"][0], K))
        V = rng.normal(scale=0.4, size=(w["shape"][1], K))
        if compute == _lib.MG_COMPUTE_MIXED:
            U = U.astype(np.float32).astype(np.float64)
            V = V.astype(np.float32).astype(np.float64)
        s.set_latents(0, U)
        s.set_latents(1, V)
        m.set("latents", 0, U)
        m.set("latents", 1, V)
        s.update_noise(it)
        m.update_noise(it)
        a, ao = s.noise()[0], m.noise()[0]
        assert abs(a - ao) <= 1e-12 * ao, (it, a, ao)


@pytest.mark.parametrize("compute,tensor_cores,K", [
    (_lib.MG_COMPUTE_FP64, 0, 10),
    (_lib.MG_COMPUTE_MIXED, 1, 32),
    (_lib.MG_COMPUTE_MIXED, 0, 32),
    (_lib.MG_COMPUTE_MIXED, 0, 10),
])
@pytest.mark.parametrize("mode", [0, 1])
def test_row_sampler_uses_device_precision(compute, tensor_cores, K, mode):
    # after a redraw the samplers read the precision from the device (mixed: unscaled packed
    # weights times that precision) and match the oracle sampled at the same alpha
    rng = np.random.default_rng(40 + K + mode)
    w = heavy_rows_workload(rng, nrow=80)
    s, _ = adaptive_pair(w, K, 12, compute=compute)
    s.set_option("tensor_core_gram", tensor_cores)
    s.set_latents(0, rng.normal(scale=0.3, size=(w["shape"][0], K)))
    s.set_latents(1, rng.normal(scale=0.3, size=(w["shape"][1], K)))
    s.update_noise(2)
    alpha = s.noise()[0]
    assert alpha > 0
    other = 1 - mode
    Vo = rng.normal(scale=0.3, size=(w["shape"][other], K))
    s.set_latents(other, Vo)
    z = rng.normal(size=(w["shape"][mode], K))
    mu, Lam, _ = s.hyper(mode)
    s.sample_latents(mode, 0, z)
    Y = train_matrix(w)
    R = orc.Csr.from_scipy(Y if mode == 0 else Y.T)
    want, _ = orc.sample_latents(K, R, Vo, s.mean_value(), alpha, mu, Lam, z=z)
    tol = FP64_TOL if compute == _lib.MG_COMPUTE_FP64 else MIXED_SAMPLE_TOL
    assert relerr(s.latents(mode), want) < tol


# ---- univariate prior (MacauOnePrior, macauoneprior.cpp:41-95, 189-290) ----

def side_matrix(rng, nrows, kind):
    """'sparse': many features of a few rows each (the link sampler gives one feature per warp);
    'dense': a few features sharing most rows (one feature at a time per block); 'binary'."""
    if kind == "dense":
        F = sp.random(nrows, 6, density=0.6, random_state=rng, format="csr")
    else:
        F = sp.random(nrows, 300, density=0.01, random_state=rng, format="csr")
    if kind == "binary":
        F.data[:] = 1.0
    else:
        F.data = rng.normal(size=F.nnz)
    return F


def univariate_pair(w, K, seed, mode, F, compute=_lib.MG_COMPUTE_FP64, lambda_beta=3.0,
                    burnin=0, nsamples=1):
    binary = bool(np.all(F.data == 1.0))
    s = gpu_sampler(w, K, 1.5, seed, compute=compute, burnin=burnin, nsamples=nsamples,
                    init=False)
    Fc = F.tocoo()
    s.set_side_univariate(mode, Fc.row, Fc.col, None if binary else Fc.data, F.shape, lambda_beta)
    s.init()
    m = oracle_model(w, K, 1.5, seed)
    m.set_side_one(mode, orc.Csr.from_scipy(F, binary), orc.Csr.from_scipy(F.T, binary),
                   lambda_beta)
    return s, m


@pytest.mark.parametrize("K", [10, 32, 64])
@pytest.mark.parametrize("mode", [0, 1])
def test_univariate_row_sampler_fp64_matches_oracle(K, mode):
    # coordinate draws from the Gram (warp finish at K <= 32, group finish at K = 64) against the
    # oracle's residual form, from random current values and hyperparameters, keyed draws
    rng = np.random.default_rng(K + 3 * mode)
    w = heavy_rows_workload(rng, nrow=70)
    F = side_matrix(rng, w["shape"][mode], "sparse")
    s, m = univariate_pair(w, K, 321, mode, F)
    for it in (0, 4):
        Ut = rng.normal(scale=0.3, size=(w["shape"][mode], K))
        Vo = rng.normal(scale=0.3, size=(w["shape"][1 - mode], K))
        mu = rng.normal(scale=0.2, size=K)
        Lam = random_spd(rng, K, 3.0)
        s.set_latents(mode, Ut)
        s.set_latents(1 - mode, Vo)
        m.set("latents", mode, Ut)
        m.set("latents", 1 - mode, Vo)
        s.set_hyper(mode, mu, Lam, None)
        m.set("mu", mode, mu)
        m.set("Lambda", mode, Lam)
        s.sample_latents(mode, it)
        assert m.sample_mode(mode, it) == 0
        assert relerr(s.latents(mode), m.latents(mode)) < FP64_TOL, it


@pytest.mark.parametrize("kind", ["sparse", "dense", "binary"])
def test_univariate_update_prior_fp64_matches_oracle(kind):
    rng = np.random.default_rng(len(kind))
    K, mode = 12, 0
    w = small_uniform(seed=2, nrow=400, ncol=250, nobs=9000)
    F = side_matrix(rng, w["shape"][mode], kind)
    s, m = univariate_pair(w, K, 55, mode, F)
    for it in (0, 1, 2):
        U = rng.normal(scale=0.5, size=(w["shape"][mode], K))
        s.set_latents(mode, U)
        m.set("latents", mode, U)
        s.update_prior(mode, it)
        assert m.update_prior(mode, it) == 0
        mu, Lam, lb_mean = s.hyper(mode)
        assert relerr(mu, m.mu(mode)) < FP64_TOL
        assert relerr(Lam, m.Lambda(mode)) < FP64_TOL
        assert relerr(s.beta(mode), m.beta(mode)) < FP64_TOL, it
        assert relerr(s.uhat(mode), m.uhat(mode)) < FP64_TOL
        lb = s.lambda_beta_univariate(mode)
        assert relerr(lb, m.lambda_beta_one(mode)) < FP64_TOL
        assert abs(lb_mean - lb.mean()) <= 1e-12 * lb.mean()


def test_univariate_update_prior_large_mode_fp64():
    # a mode with more rows than the shared-memory link sampler holds (26K) takes the
    # global-memory variant (k_beta_one, four dimensions per block)
    rng = np.random.default_rng(12)
    K, mode = 10, 0
    w = workloads.bpmf_uniform(nrow=27000, ncol=120, nobs=60000, seed=3)
    F = side_matrix(rng, w["shape"][mode], "sparse")
    s, m = univariate_pair(w, K, 66, mode, F)
    U = rng.normal(scale=0.5, size=(w["shape"][mode], K))
    s.set_latents(mode, U)
    m.set("latents", mode, U)
    s.update_prior(mode, 4)
    assert m.update_prior(mode, 4) == 0
    assert relerr(s.beta(mode), m.beta(mode)) < FP64_TOL
    assert relerr(s.uhat(mode), m.uhat(mode)) < FP64_TOL
    assert relerr(s.lambda_beta_univariate(mode), m.lambda_beta_one(mode)) < FP64_TOL


def test_univariate_sweeps_fp64_match_oracle():
    # whole sweeps: univariate prior on the rows (dense side), BPMF on the columns, evaluation
    rng = np.random.default_rng(77)
    w = workloads.bpmf_uniform(nrow=400, ncol=300, nobs=12000, seed=9)
    K, seed, burnin = 8, 2026, 4
    F = side_matrix(rng, w["shape"][0], "dense")
    s, m = univariate_pair(w, K, seed, 0, F, burnin=burnin, nsamples=6)
    for it in range(10):
        s.sweep(it, eval=True)
        assert m.sweep(it, burnin) == 0
        for mode in (0, 1):
            assert relerr(s.latents(mode), m.latents(mode)) < 1e-8, (it, mode)
        assert relerr(s.beta(0), m.beta(0)) < 1e-8
        r, r1 = s.rmse()
        ro, r1o = m.rmse()
        assert abs(r - ro) < 1e-9 and abs(r1 - r1o) < 1e-9
    np.testing.assert_allclose(s.predictions(), m.predictions(), rtol=1e-9, atol=1e-12)


@pytest.mark.parametrize("tensor_cores,K", [(1, 32), (0, 32), (0, 10)])
@pytest.mark.parametrize("mode", [0, 1])
def test_univariate_row_sampler_mixed_within_tolerance(tensor_cores, K, mode):
    rng = np.random.default_rng(90 + K + mode)
    w = heavy_rows_workload(rng, nrow=70)
    F = side_matrix(rng, w["shape"][mode], "sparse")
    s, m = univariate_pair(w, K, 8, mode, F, compute=_lib.MG_COMPUTE_MIXED)
    s.set_option("tensor_core_gram", tensor_cores)
    Ut = rng.normal(scale=0.3, size=(w["shape"][mode], K)).astype(np.float32).astype(np.float64)
    Vo = rng.normal(scale=0.3, size=(w["shape"][1 - mode], K)).astype(np.float32).astype(np.float64)
    s.set_latents(mode, Ut)
    s.set_latents(1 - mode, Vo)
    m.set("latents", mode, Ut)
    m.set("latents", 1 - mode, Vo)
    s.sample_latents(mode, 3)
    assert m.sample_mode(mode, 3) == 0
    assert relerr(s.latents(mode), m.latents(mode)) < MIXED_SAMPLE_TOL


def test_macau_mixed_cg_precision_option():
    # mixed mode runs the block-CG in FP64 unless "cg_fp32" selects FP32 with FP64 residual
    # replacement; both reach the same link matrix within the CG tolerance's reach
    w = workloads.macau_side(scale=0.05, seed=6)
    betas = []
    for opt in (0, 1):
        s = gpu_sampler(w, 16, 2.0, 17, compute=_lib.MG_COMPUTE_MIXED, init=False)
        s.set_option("cg_fp32", opt)
        s.init()
        for it in range(2):
            s.sweep(it, eval=False)
        betas.append(s.beta(0))
        assert s.stats()["cg_iters"][0] > 0
    assert relerr(betas[1], betas[0]) < 2e-2


@pytest.mark.parametrize("K", [16, 32, 64])
@pytest.mark.parametrize("gram", [1, 2])
def test_mixed_row_sampler_fp16_tf32_grams(K, gram):
    # Gram inputs in FP16 (1) or TF32 (2) instead of BF16: the CUDA-core sampler at every K
    # (K = 32 included), against the FP64 oracle under the same keyed draws; TF32 and FP16 keep
    # 10-11 mantissa bits against BF16's 8, so their error stays below the BF16 run's
    rng = np.random.default_rng(K + 50 * gram)
    w = small_uniform(seed=5, nrow=400, ncol=250, nobs=15000)
    Vo = rng.normal(scale=0.3, size=(w["shape"][1], K))
    Y = train_matrix(w)
    errs = []
    for g in (0, gram):
        s = gpu_sampler(w, K, 2.0, seed=4242, compute=_lib.MG_COMPUTE_MIXED, init=False)
        s.set_option("gram_precision", g)
        s.init()
        s.set_latents(1, Vo)
        mu, Lam, _ = s.hyper(0)
        s.sample_latents(0, 9)
        want, _ = orc.sample_latents(K, orc.Csr.from_scipy(Y), Vo, s.mean_value(), 2.0, mu, Lam,
                                     seed=4242, sweep=9, mode=0)
        errs.append(relerr(s.latents(0), want))
    assert errs[1] < MIXED_SAMPLE_TOL
    assert errs[1] < errs[0], errs


# ---- many independent chains in one set of launches (mg_batch) ----

def test_batch_matches_single_problem_contexts():
    # each problem of the batch follows the chain of a single mixed context with its seed: the
    # same keyed draws and arithmetic except the order of the FP32 Gram sums (tensor cores at a
    # padded K = 32 in the batch, the CUDA-core sampler for K < 32 alone); a last-bit difference
    # can move a BF16 rounding of a gathered latent, so the chains agree to the mixed tolerance
    # (a row of the wrong problem, or a wrong draw, would differ at O(1))
    problems, Ks, seeds = workloads.batched_uneven(nprob=7, rows=(40, 300), cols=(30, 200),
                                                   density=(0.05, 0.2))
    alpha = 4.0
    for sweeps, tol in ((1, 5e-3), (6, 5e-2)):
        b = _lib.Batch(problems, Ks, seeds, alpha)
        b.init(2)
        b.sweeps(0, sweeps, eval=True)
        rb = b.rmse()
        assert b.info()["nnz"] == sum(len(pr["vals"]) for pr in problems)
        for p, (pr, K, sd) in enumerate(zip(problems, Ks, seeds)):
            s = gpu_sampler(pr, K, alpha, sd, compute=_lib.MG_COMPUTE_MIXED, burnin=2,
                            nsamples=max(1, sweeps - 2))
            for it in range(sweeps):
                s.sweep(it, eval=True)
            for mode in (0, 1):
                assert relerr(b.latents(p, mode), s.latents(mode)) < tol, (sweeps, p, mode)
            r, r1 = s.rmse()
            assert abs(rb[p, 0] - r) < tol * r and abs(rb[p, 1] - r1) < tol * r1
        b.close()


def test_batch_matches_oracle_per_problem():
    # the reference runs one Macau object per problem (macau.pyx:221-234); here every problem of
    # one batch is compared after each of its first sweeps with an FP64 oracle chain of that
    # problem and seed (same keyed draws): latents of both modes, hyperparameters and the
    # running RMSE.  K = 8, 16 and 32 all occur.
    problems, Ks, seeds = workloads.batched_uneven(nprob=10, rows=(60, 400), cols=(40, 260),
                                                   density=(0.04, 0.2))
    assert {8, 16, 32} <= set(Ks), Ks
    alpha, burnin = 4.0, 1
    b = _lib.Batch(problems, Ks, seeds, alpha)
    b.init(burnin)
    models = [oracle_model(pr, K, alpha, sd) for pr, K, sd in zip(problems, Ks, seeds)]
    for it, tol in enumerate((MIXED_SAMPLE_TOL, 2 * MIXED_SAMPLE_TOL, 4 * MIXED_SAMPLE_TOL)):
        b.sweeps(it, 1, eval=True)
        rb = b.rmse()
        for p, m in enumerate(models):
            assert m.sweep(it, burnin) == 0
            for mode in (0, 1):
                err = relerr(b.latents(p, mode), m.latents(mode))
                assert err < tol, (it, p, Ks[p], mode, err)
            ro = m.rmse()
            assert abs(rb[p, 0] - ro[0]) < tol * ro[0], (it, p, rb[p], ro)
            assert abs(rb[p, 1] - ro[1]) < tol * ro[1], (it, p, rb[p], ro)
    b.close()


def test_batch_learns_every_problem():
    problems, Ks, seeds = workloads.batched_uneven(nprob=24, rows=(200, 600), cols=(100, 300),
                                                   density=(0.05, 0.1))
    b = _lib.Batch(problems, Ks, seeds, 4.0)
    b.init(30)
    b.sweeps(0, 60, eval=True)
    rm = b.rmse()
    # the data noise is 0.5: every problem's posterior-mean RMSE lands near it
    assert np.all(rm[:, 0] < 0.75), rm[:, 0]
    assert rm[:, 0].mean() < rm[:, 1].mean()  # averaging over samples helps on the whole
    b.close()


def test_cholesky_failure_is_reported_and_context_survives():
    w = small_uniform(seed=4)
    K = 6
    s = gpu_sampler(w, K, 1.0, seed=1)
    s.set_hyper(0, np.zeros(K), -10.0 * np.eye(K))
    with pytest.raises(_lib.CholeskyError, match="Cholesky Decomposition failed"):
        s.sample_latents(0, 0)
    s.init()
    s.sweep(0)
    assert np.isfinite(s.latents(0)).all()


def test_eval_rmse_golden_on_gpu():  # tests.cpp:552-591 through mg_eval
    w = dict(rows=np.array([0], np.int32), cols=np.array([0], np.int32), vals=np.array([2.0]),
             trows=np.array([0], np.int32), tcols=np.array([0], np.int32),
             tvals=np.array([4.5]), shape=(1, 1))
    s = gpu_sampler(w, 2, 1.0, seed=0)
    steps = [([1.0, 0.0], [1.0, 0.0], 3.0, 0.0, 1.5, 1.5),
             ([2.0, 0.0], [1.0, 0.0], 3.5, 0.5, 0.5, 1.0),
             ([2.0, 0.0], [3.0, 0.0], 5.0, 14.0, 3.5, 0.5)]
    for n, (u, v, pred, var, r1, ravg) in enumerate(steps):
        s.set_latents(0, np.array([u]))
        s.set_latents(1, np.array([v]))
        s.eval(n)
        got_r, got_r1 = s.rmse()
        assert got_r1 == pytest.approx(r1) and got_r == pytest.approx(ravg)
        assert s.predictions()[0] == pytest.approx(pred)
    s.set_samples(0, 3)
    assert s.stds()[0] == pytest.approx(np.sqrt(14.0 / 2))


@pytest.mark.parametrize("compute", [_lib.MG_COMPUTE_FP64, _lib.MG_COMPUTE_MIXED])
def test_two_mode_prior_update_matches_one_mode_at_a_time(compute):
    """A sweep updates both modes' BPMF priors together (three launches for the two modes'
    statistics, reductions and Normal-Wishart draws); the phase-timed sweeps update them one mode
    after the other.  The chains must agree bit for bit."""
    w = small_uniform(seed=12)
    out = []
    for phased in (False, True):
        s = gpu_sampler(w, 16, 2.0, 31, compute=compute)
        s.time_sweeps(0, 3, eval=False, phase_events=phased)
        out.append([s.latents(0), s.latents(1)] + [np.asarray(x) for m in (0, 1)
                                                   for x in s.hyper(m)[:2]])
        s.close()
    for a, b in zip(out[0], out[1]):
        np.testing.assert_array_equal(a, b)


def test_row_and_column_arrays_give_the_same_context_as_the_idx_form():
    """mg_set_relation_data_rc / _test_rc (macau.h:37-38: separate row and column arrays) build
    the same training and test data as the nnz x 2 idx forms (macau.h:39-40): two sweeps from the
    same seed agree bit for bit, and so do the test sets."""
    w = small_uniform(seed=8)
    nr, nc = w["shape"]
    rows, cols = np.asarray(w["rows"], np.int32), np.asarray(w["cols"], np.int32)
    rows = np.concatenate([rows, rows[:50]])  # duplicates, summed in input order
    cols = np.concatenate([cols, cols[:50]])
    vals = np.concatenate([np.asarray(w["vals"], np.float64), np.linspace(-1, 1, 50)])
    lib = _lib.lib()
    dims = np.array([nr, nc], np.int32)
    out = []
    for form in ("idx", "rc"):
        s = _lib.Sampler(8, 2.0, seed=4, compute=_lib.MG_COMPUTE_MIXED)
        if form == "idx":
            idx = np.concatenate([rows, cols])
            s._chk(lib.mg_set_relation_data(s.h, _lib.ptr(idx), 2, _lib.ptr(vals), len(vals),
                                            _lib.ptr(dims)))
            tidx = np.concatenate([np.asarray(w["trows"], np.int32),
                                   np.asarray(w["tcols"], np.int32)])
            tv = np.ascontiguousarray(w["tvals"], np.float64)
            s._chk(lib.mg_set_relation_data_test(s.h, _lib.ptr(tidx), 2, _lib.ptr(tv), len(tv),
                                                 _lib.ptr(dims)))
            s.dims = (nr, nc)
            n = np.zeros(1, np.int64)
            s._chk(lib.mg_get_dims(s.h, None, None, None, _lib.ptr(n), None))
            s.ntest = int(n[0])
        else:
            s.set_relation_data(rows, cols, vals, w["shape"])
            s.set_relation_data_test(w["trows"], w["tcols"], w["tvals"], w["shape"])
        s.set_samples(0, 2)
        s.init()
        for it in range(2):
            s.sweep(it, eval=True)
        out.append((s.latents(0), s.latents(1), s.test_data(), s.rmse()))
    for a, b in zip(out[0], out[1]):
        np.testing.assert_array_equal(np.asarray(a), np.asarray(b))
    with pytest.raises(ValueError):
        _lib.Sampler(8, 2.0).set_relation_data(rows, cols[:-1], vals, w["shape"])


def test_device_index_checks_and_test_set_order():
    """Training and test indices are checked on the device during the CSR builds; the test set
    comes back in column-major order with duplicates summed (sparseFromIJV, bpmfutils.h:57-82),
    and a rejected training set leaves a context that accepts a valid one."""
    w = small_uniform(seed=6)
    nr, nc = w["shape"]
    s = _lib.Sampler(4, 1.0, seed=1)
    bad_rows = np.array(w["rows"], np.int32)
    bad_rows[len(bad_rows) // 2] = nr
    with pytest.raises(_lib.MacauError, match="training index out of range"):
        s.set_relation_data(bad_rows, w["cols"], w["vals"], w["shape"])
    bad_cols = np.array(w["cols"], np.int32)
    bad_cols[-1] = -1
    with pytest.raises(_lib.MacauError, match="training index out of range"):
        s.set_relation_data(w["rows"], bad_cols, w["vals"], w["shape"])
    with pytest.raises(_lib.MacauError):
        s.init()
    s.set_relation_data(w["rows"], w["cols"], w["vals"], w["shape"])
    with pytest.raises(_lib.MacauError, match="test index out of range"):
        s.set_relation_data_test(np.array([0, nr]), np.array([0, 0]), np.array([1.0, 2.0]),
                                 w["shape"])
    rng = np.random.default_rng(3)
    tr = rng.integers(0, nr, 400).astype(np.int32)
    tc = rng.integers(0, nc, 400).astype(np.int32)
    tr[200:260], tc[200:260] = tr[:60], tc[:60]  # duplicates, summed in input order
    tv = rng.integers(-4, 5, 400).astype(np.float64)
    s.set_relation_data_test(tr, tc, tv, w["shape"])
    got = s.test_data()
    key = tc.astype(np.int64) * nr + tr
    order = np.argsort(key, kind="stable")
    uk, first = np.unique(key[order], return_index=True)
    want_v = np.add.reduceat(tv[order], first)
    assert got.shape == (len(uk), 3)
    np.testing.assert_array_equal(got[:, 0], uk % nr)
    np.testing.assert_array_equal(got[:, 1], uk // nr)
    np.testing.assert_array_equal(got[:, 2], want_v)
    s.set_samples(0, 2)
    s.init()
    s.sweep(0, eval=True)
    assert np.isfinite(s.rmse()[0])
