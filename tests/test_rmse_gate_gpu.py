"""The statistical gate on the 2,000 x 1,500 uniform matrix (60,000 entries at random positions,
rank-10 signal + N(0, 0.5^2), 10% random holdout, alpha = 4, seed 0): after 200 burn-in and 200
collected sweeps, the posterior-mean test RMSE of the GPU chain matches the FP64 oracle's within
0.002, in FP64 mode, in mixed mode on the CUDA-core sampler (K = 10), and in mixed mode on the
tensor-core sampler (K = 32).  The FP64 chain draws what the oracle draws, so it matches far more
tightly; the mixed chains differ by rounding, which the gate bounds."""
import pytest

from macau_b200 import _lib, workloads
from tests.gpu_helpers import gpu_sampler, oracle_model

pytestmark = pytest.mark.gpu

RMSE_GATE = 0.002
BURNIN, NSAMPLES = 200, 200


@pytest.fixture(scope="module")
def uniform():
    return workloads.bpmf_uniform(seed=0)


@pytest.fixture(scope="module")
def oracle_rmse(uniform):
    out = {}

    def get(K):
        if K not in out:
            m = oracle_model(uniform, K, 4.0, 0)
            for it in range(BURNIN + NSAMPLES):
                assert m.sweep(it, BURNIN) == 0
            out[K] = m.rmse()[0]
        return out[K]
    return get


@pytest.mark.parametrize("K,compute", [(10, _lib.MG_COMPUTE_FP64), (10, _lib.MG_COMPUTE_MIXED),
                                       (32, _lib.MG_COMPUTE_MIXED)])
def test_posterior_mean_rmse_matches_oracle(uniform, oracle_rmse, K, compute):
    s = gpu_sampler(uniform, K, 4.0, 0, compute=compute, burnin=BURNIN, nsamples=NSAMPLES)
    s.sweeps(0, BURNIN + NSAMPLES, eval=True)
    r = s.rmse()[0]
    ro = oracle_rmse(K)
    s.close()
    assert abs(r - ro) < RMSE_GATE, (r, ro)
    if compute == _lib.MG_COMPUTE_FP64:
        assert abs(r - ro) < 1e-4, (r, ro)
