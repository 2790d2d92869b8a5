"""The tensor-core sampler's fused epilogue (k_gram_tc<true>: each row factored, solved and drawn
in the Gram kernel) against the two-kernel path it replaces (Gram records in HBM, then
k_finish_tc): the same FP32 arithmetic, so the latents agree to the last bit; its FP64 retry of
rows whose FP32 factor fails, against the oracle; the order of the row groups in the work queue
(option group_mix), which changes no result; and the bounded waits of the kernel, made to run
out through a test hook, reported as MG_ERR_TIMEOUT with the context still usable."""
import numpy as np
import pytest

from macau_b200 import _lib, workloads
from oracle import oracle as orc
from tests.gpu_helpers import gpu_sampler, random_spd, relerr, train_matrix
from tests.test_gpu_parity import MIXED_SAMPLE_TOL, heavy_rows_workload, small_uniform

pytestmark = pytest.mark.gpu

K = 32


def _half_sweep(w, fused, mode, seed=11, alpha=2.0):
    rng = np.random.default_rng(50 + mode)
    s = gpu_sampler(w, K, alpha, seed, compute=_lib.MG_COMPUTE_MIXED)
    s.set_option("fused_finish", fused)
    other = 1 - mode
    s.set_latents(other, rng.normal(scale=0.4, size=(w["shape"][other], K)))
    s.set_hyper(mode, rng.normal(scale=0.2, size=K), random_spd(rng, K, 4.0))
    s.sample_latents(mode, 6)
    out = s.latents(mode)
    s.close()
    return out


@pytest.mark.parametrize("name", ["heavy_rows", "powerlaw"])
@pytest.mark.parametrize("mode", [0, 1])
def test_fused_finish_matches_the_record_path(name, mode):
    # heavy_rows: rows split into parts (finished by k_finish_tc after the fused kernel) beside
    # unsplit ones; powerlaw: the benchmark generator at 5% scale
    w = (heavy_rows_workload(np.random.default_rng(19)) if name == "heavy_rows"
         else workloads.bpmf_powerlaw(scale=0.05, seed=2))
    a = _half_sweep(w, 1, mode)
    b = _half_sweep(w, 0, mode)
    assert np.array_equal(a, b), float(np.abs(a - b).max())


@pytest.mark.parametrize("mix", [0, 4])
def test_group_order_changes_no_result(mix):
    # the row groups' order in the work queue (option group_mix, default 16) decides which CTA
    # finishes which row and when, not the row's arithmetic: the same sweeps bit for bit
    w = workloads.bpmf_powerlaw(scale=0.05, seed=2)
    out = []
    for m in (16, mix):
        s = gpu_sampler(w, K, 2.0, 23, compute=_lib.MG_COMPUTE_MIXED)
        s.set_option("group_mix", m)
        for it in range(2):
            s.sweep(it)
        out.append((s.latents(0), s.latents(1)))
        s.close()
    for a, b in zip(out[0], out[1]):
        np.testing.assert_array_equal(a, b)


@pytest.mark.parametrize("adaptive", [False, True])
def test_fused_finish_sweeps_match_the_record_path(adaptive):
    # whole sweeps: a Macau prior on the rows (the finish adds Lambda (mu + Uhat)), BPMF on the
    # columns, and optionally adaptive noise (the precision read from the device)
    w = workloads.macau_side(scale=0.02, seed=5)
    lat = []
    for fused in (1, 0):
        s = gpu_sampler(w, K, 1.0, 21, compute=_lib.MG_COMPUTE_MIXED, init=False)
        s.set_option("fused_finish", fused)
        if adaptive:
            s.set_noise_adaptive(1.0, 10.0)
        s.init()
        for it in range(3):
            s.sweep(it, eval=False)
        lat.append([s.latents(0), s.latents(1)])
        s.close()
    for mode in (0, 1):
        assert np.array_equal(lat[0][mode], lat[1][mode])


@pytest.mark.parametrize("fused", [1, 0])
def test_fp32_factor_failures_are_redone_in_fp64(fused):
    # Lambda = 1e-7 I and rows with fewer entries than K: MM = Lambda + alpha G is singular up to
    # 1e-7 in the directions the row's latents leave free, so every FP32 factor loses its pivot
    # (below 2^-20 of its diagonal) and the row is redone in FP64.  The other factor's values are
    # multiples of 1/8 (exact in BF16, their products and sums exact in FP32), so the Gram the
    # FP64 redo factors is the oracle's.  The fused redo also re-accumulates the right-hand side
    # in FP64 from the FP32 weights, so its samples agree to FP64 rounding amplified by the
    # conditioning; the record path redoes the factor from the record, whose right-hand side
    # carries the tensor-core sum's 16-bit weights, so it is held to the mixed bar.
    rng = np.random.default_rng(77)
    w = small_uniform(seed=9, nrow=300, ncol=200, nobs=3000)
    Y = train_matrix(w)
    assert np.diff(Y.tocsr().indptr).max() < K
    s = gpu_sampler(w, K, 2.0, seed=5, compute=_lib.MG_COMPUTE_MIXED)
    s.set_option("fused_finish", fused)
    V = rng.integers(-8, 9, size=(w["shape"][1], K)) / 8.0
    s.set_latents(1, V)
    mu, Lam = np.zeros(K), 1e-7 * np.eye(K)
    s.set_hyper(0, mu, Lam)
    before = s.stats()["retries"][0]
    s.sample_latents(0, 4)
    retried = s.stats()["retries"][0] - before
    got = s.latents(0)
    want, st = orc.sample_latents(K, orc.Csr.from_scipy(Y), V, s.mean_value(), 2.0, mu, Lam,
                                  seed=5, sweep=4, mode=0)
    s.close()
    assert st == 0
    assert retried >= 0.9 * w["shape"][0], retried
    assert relerr(got, want) < (1e-6 if fused else MIXED_SAMPLE_TOL), relerr(got, want)


@pytest.mark.parametrize("fused", [1, 0])
def test_wait_that_runs_out_is_reported_and_the_context_survives(fused):
    # the MMA warp waits on a barrier that nothing arrives on, with a 1 ms budget: the launch
    # aborts (every role leaves, the MMAs drain, TMEM is freed) and reports MG_ERR_TIMEOUT; after
    # mg_init the same context samples normally (a later launch allocates TMEM again)
    rng = np.random.default_rng(3)
    w = small_uniform(seed=5, nrow=400, ncol=250, nobs=15000)
    s = gpu_sampler(w, K, 2.0, seed=4242, compute=_lib.MG_COMPUTE_MIXED)
    s.set_option("fused_finish", fused)
    s.set_option("tc_wait_us", 1000)
    s.set_option("tc_wait_test", 1)
    with pytest.raises(_lib.MacauError, match="timed out") as e:
        s.sample_latents(0, 9)
    assert e.value.code == _lib.MG_ERR_TIMEOUT
    s.set_option("tc_wait_test", 0)
    s.set_option("tc_wait_us", 0)
    s.init()
    Vo = rng.normal(scale=0.3, size=(w["shape"][1], K))
    s.set_latents(1, Vo)
    mu, Lam, _ = s.hyper(0)
    s.sample_latents(0, 9)
    want, _ = orc.sample_latents(K, orc.Csr.from_scipy(train_matrix(w)), Vo, s.mean_value(), 2.0,
                                 mu, Lam, seed=4242, sweep=9, mode=0)
    assert relerr(s.latents(0), want) < MIXED_SAMPLE_TOL
    s.close()
