"""Parity on the shape of the benchmark workload: the power-law matrix generator of the
138,000 x 27,000 benchmark at 5% scale (6,900 x 1,350, about 0.9M training entries; row degrees
up to 1,350 and column degrees up to ~4,500 from the truncated 1/k law), K = 32, alpha = 2.

At this scale the default split threshold of the row samplers is 256 entries, so the tensor-core
sampler sees the benchmark's mix: length-sorted 4-row MMA groups of very uneven lengths, heavy
rows cut into parts whose partial Grams are summed, and (with the autotuner) the tuned
threshold and bucketed task lists.

  * one keyed-draw half-sweep per mode against the oracle's sample_latent_blas restatement
    (latentprior.cpp:361-385): FP64 within 1e-9, mixed (tensor cores) within the mixed bar;
  * the posterior-mean test RMSE of whole chains (the same burn-in and sample counts as the
    oracle's FP64 chain, eval_rmse of bpmfutils.h:86-114) within 0.002, mixed and FP64.
"""
import numpy as np
import pytest

from macau_b200 import _lib, workloads
from oracle import oracle as orc
from tests.gpu_helpers import gpu_sampler, oracle_model, random_spd, relerr, train_matrix
from tests.test_gpu_parity import FP64_TOL, MIXED_SAMPLE_TOL

pytestmark = pytest.mark.gpu

K, ALPHA, SEED = 32, 2.0, 31
RMSE_GATE = 0.002
BURNIN, NSAMPLES = 50, 50


@pytest.fixture(scope="module")
def powerlaw():
    return workloads.bpmf_powerlaw(scale=0.05, seed=2)


def test_powerlaw_workload_has_split_rows(powerlaw):
    # the half-sweep tests below cover heavy rows only if the workload has rows past the
    # default threshold clamp(nnz / (2 * 148 * 16), 256, 16384) in both modes
    Y = train_matrix(powerlaw)
    thr = min(16384, max(256, Y.nnz // (2 * 148 * 16)))
    assert np.diff(Y.tocsr().indptr).max() > thr
    assert np.diff(Y.indptr).max() > thr


@pytest.mark.parametrize("tuned", [False, True])
@pytest.mark.parametrize("compute", [_lib.MG_COMPUTE_FP64, _lib.MG_COMPUTE_MIXED])
@pytest.mark.parametrize("mode", [0, 1])
def test_powerlaw_half_sweep_matches_oracle(powerlaw, mode, compute, tuned):
    rng = np.random.default_rng(100 + 10 * mode + compute)
    s = gpu_sampler(powerlaw, K, ALPHA, SEED, compute=compute)
    if tuned:
        s.autotune(use_cache=False)
    other = 1 - mode
    Vo = rng.normal(scale=0.4, size=(powerlaw["shape"][other], K))
    s.set_latents(other, Vo)
    mu = rng.normal(scale=0.2, size=K)
    Lam = random_spd(rng, K, 4.0)
    s.set_hyper(mode, mu, Lam)
    s.sample_latents(mode, 13)
    Y = train_matrix(powerlaw)
    R = orc.Csr.from_scipy(Y if mode == 0 else Y.T)
    want, st = orc.sample_latents(K, R, Vo, s.mean_value(), ALPHA, mu, Lam, seed=SEED, sweep=13,
                                  mode=mode)
    assert st == 0
    got = s.latents(mode)
    s.close()
    tol = FP64_TOL if compute == _lib.MG_COMPUTE_FP64 else MIXED_SAMPLE_TOL
    err = relerr(got, want)
    assert err < tol, err


@pytest.fixture(scope="module")
def oracle_chain_rmse(powerlaw):
    m = oracle_model(powerlaw, K, ALPHA, SEED)
    for it in range(BURNIN + NSAMPLES):
        assert m.sweep(it, BURNIN) == 0
    return m.rmse()[0]


@pytest.mark.parametrize("compute", [_lib.MG_COMPUTE_MIXED, _lib.MG_COMPUTE_FP64])
def test_powerlaw_posterior_mean_rmse_matches_oracle(powerlaw, oracle_chain_rmse, compute):
    s = gpu_sampler(powerlaw, K, ALPHA, SEED, compute=compute, burnin=BURNIN,
                    nsamples=NSAMPLES)
    s.autotune()
    s.sweeps(0, BURNIN + NSAMPLES, eval=True)
    r = s.rmse()[0]
    s.close()
    assert abs(r - oracle_chain_rmse) < RMSE_GATE, (r, oracle_chain_rmse)
    if compute == _lib.MG_COMPUTE_FP64:
        # the FP64 chain draws what the oracle draws; only the split rows' summation order
        # (autotuned threshold) and the reduction orders differ
        assert abs(r - oracle_chain_rmse) < 1e-4, (r, oracle_chain_rmse)
