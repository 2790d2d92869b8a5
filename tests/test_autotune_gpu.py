"""The row samplers' autotuner (mg_autotune) and its two knobs, the work split ("split_threshold")
and the CUDA-core sampler's CTA shape ("cta_groups").

Every knob setting must draw the same samples as the FP64 oracle under injected draws (1e-9 in
FP64, the mixed tolerance in mixed mode), and a tuned context must continue the chain of an
untuned one: only the summation order of split rows may differ."""
import numpy as np
import pytest

from macau_b200 import _lib, workloads
from oracle import oracle as orc
from tests.gpu_helpers import gpu_sampler, relerr, train_matrix
from tests.test_gpu_parity import FP64_TOL, MIXED_SAMPLE_TOL, heavy_rows_workload

pytestmark = pytest.mark.gpu

FP64 = _lib.MG_COMPUTE_FP64
MIXED = _lib.MG_COMPUTE_MIXED


@pytest.mark.parametrize("K,groups", [(10, 2), (32, 2), (32, 4), (64, 1)])
@pytest.mark.parametrize("compute", [FP64, MIXED])
@pytest.mark.parametrize("thr", [256, 1024])
@pytest.mark.parametrize("mode", [0, 1])
def test_knobs_match_oracle(K, groups, compute, thr, mode):
    # rows of 3,900 entries are split into 4 or 16 parts; the CUDA-core sampler at both shapes
    rng = np.random.default_rng(K + 7 * groups + thr + mode)
    w = heavy_rows_workload(rng)
    s = gpu_sampler(w, K, 1.5, seed=3, compute=compute)
    s.set_option("tensor_core_gram", 0)
    s.set_option("split_threshold", thr)
    s.set_option("cta_groups", groups)
    t = s.tuning()[mode]
    assert t["split_threshold"] == thr and t["cta_groups"] == groups and not t["tensor_core"]
    other = 1 - mode
    Vo = rng.normal(scale=0.3, size=(w["shape"][other], K))
    s.set_latents(other, Vo)
    z = rng.normal(size=(w["shape"][mode], K))
    mu, Lam, _ = s.hyper(mode)
    s.sample_latents(mode, 0, z)
    Y = train_matrix(w)
    R = orc.Csr.from_scipy(Y if mode == 0 else Y.T)
    want, _ = orc.sample_latents(K, R, Vo, s.mean_value(), 1.5, mu, Lam, z=z)
    tol = FP64_TOL if compute == FP64 else MIXED_SAMPLE_TOL
    assert relerr(s.latents(mode), want) < tol


@pytest.mark.parametrize("thr", [256, 2048])
@pytest.mark.parametrize("mode", [0, 1])
def test_split_threshold_tensor_core_sampler_matches_oracle(thr, mode):
    rng = np.random.default_rng(thr + mode)
    K = 32
    w = heavy_rows_workload(rng)
    s = gpu_sampler(w, K, 1.5, seed=3, compute=MIXED)
    s.set_option("split_threshold", thr)
    assert s.tuning()[mode]["tensor_core"]
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


def test_knob_validation():
    w = workloads.bpmf_uniform(nrow=100, ncol=80, nobs=2000, seed=1)
    s = gpu_sampler(w, 10, 2.0, seed=1)
    with pytest.raises(_lib.MacauError):
        s.set_option("split_threshold", 100)
    with pytest.raises(_lib.MacauError):
        s.set_option("cta_groups", 3)
    m = gpu_sampler(w, 10, 2.0, seed=1, compute=MIXED)
    m.set_option("gram_precision", 1)  # FP16 Grams offer only the default shape
    with pytest.raises(_lib.MacauError):
        m.set_option("cta_groups", 2)


@pytest.fixture(scope="module")
def powerlaw():
    # 20,700 x 4,050 with about 2.7M training entries: four distinct split thresholds
    return workloads.bpmf_powerlaw(scale=0.15, seed=7)


@pytest.mark.parametrize("K,compute,tc", [(10, FP64, True), (32, MIXED, True),
                                          (32, MIXED, False), (64, FP64, True)])
def test_autotuned_chain_continues_the_untuned_one(powerlaw, K, compute, tc):
    w = powerlaw
    seed, burnin = 11, 1
    ref = gpu_sampler(w, K, 2.0, seed, compute=compute, burnin=burnin, nsamples=2)
    tun = gpu_sampler(w, K, 2.0, seed, compute=compute, burnin=burnin, nsamples=2)
    for s in (ref, tun):
        s.set_option("tensor_core_gram", int(tc))
        s.init()
    ref.sweep(0, eval=True)
    tun.sweep(0, eval=True)
    info = tun.autotune(use_cache=False)
    for m, t in enumerate(info):
        assert t["state"] == "timed"
        assert t["candidates"] >= 3, t  # at least 3 distinct thresholds at this size
        assert 256 <= t["split_threshold"] <= 16384
        assert t["ms_best"] <= t["ms_default"] + 1e-9
        assert t["tensor_core"] == (compute == MIXED and K == 32 and tc)
    assert tun.stats()["sweeps"] == ref.stats()["sweeps"]
    for it in (1, 2):
        ref.sweep(it, eval=True)
        tun.sweep(it, eval=True)
    # mixed: a split row's Gram summed in another order can move the BF16 rounding of a
    # gathered latent, so the chains agree to the mixed tolerance
    tol = FP64_TOL if compute == FP64 else MIXED_SAMPLE_TOL
    for m in (0, 1):
        assert relerr(tun.latents(m), ref.latents(m)) < tol, m
    assert abs(tun.rmse()[0] - ref.rmse()[0]) < (FP64_TOL if compute == FP64 else 1e-3)
    # a later context on the same data takes the choice from the cache
    again = gpu_sampler(w, K, 2.0, seed, compute=compute, init=False)
    again.set_option("tensor_core_gram", int(tc))
    again.set_option("autotune", 1)
    again.init()
    cached = again.tuning()
    for m in (0, 1):
        assert cached[m]["state"] == "cached"
        assert cached[m]["split_threshold"] == info[m]["split_threshold"]
        assert cached[m]["cta_groups"] == info[m]["cta_groups"]
    # with the option set before the training data, the cached choice shapes the task lists
    # built there, and mg_init keeps them
    early = _lib.Sampler(K, 2.0, seed=seed, compute=compute)
    early.set_option("tensor_core_gram", int(tc))
    early.set_option("autotune", 1)
    early.set_relation_data(w["rows"], w["cols"], w["vals"], w["shape"])
    pre = early.tuning()
    early.set_samples(burnin, 2)
    early.init()
    post = early.tuning()
    for m in (0, 1):
        assert pre[m]["state"] == post[m]["state"] == "cached"
        assert pre[m]["split_threshold"] == post[m]["split_threshold"] == info[m]["split_threshold"]
    for s in (ref, tun, again, early):
        s.close()


def test_batch_autotune_keeps_the_chains():
    problems, Ks, seeds = workloads.batched_uneven(nprob=40)
    alpha = 4.0
    tuned = _lib.Batch(problems, Ks, seeds, alpha)
    tuned.init(2)
    info = tuned.autotune(use_cache=False)
    for t in info:
        assert t["state"] == "timed" and t["candidates"] >= 3, t
        assert t["finish_ctas_per_sm"] in (4, 8, 16)
        assert t["ms_best"] <= t["ms_default"] + 1e-9
    plain = _lib.Batch(problems, Ks, seeds, alpha)
    plain.init(2)
    for b in (tuned, plain):
        b.sweeps(0, 4, eval=True)
    # no row of these problems is long enough to be split, so only the launch shape changed
    for p in range(0, len(problems), 7):
        for mode in (0, 1):
            assert relerr(tuned.latents(p, mode), plain.latents(p, mode)) < 5e-3, (p, mode)
    np.testing.assert_allclose(tuned.rmse(), plain.rmse(), rtol=1e-3)
    again = _lib.Batch(problems, Ks, seeds, alpha)
    again.init(2)
    cached = again.autotune(use_cache=True)
    for m in (0, 1):
        assert cached[m]["state"] == "cached"
        assert cached[m]["split_threshold"] == info[m]["split_threshold"]
        assert cached[m]["finish_ctas_per_sm"] == info[m]["finish_ctas_per_sm"]
    for b in (tuned, plain, again):
        b.close()
