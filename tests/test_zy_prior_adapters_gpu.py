"""The C++ adapters of include/macau_b200_priors.hpp on the GPU.  A compiled program runs one
chain with MacauGpuX::run() (the whole loop on the device) and one through the reference's
ILatentPrior calls on host Eigen matrices in MacauX::run's order (sample mode 0, mode 1, update
both priors); both draw the same keyed numbers from the same device code, so their latents and
Lambdas agree to the last bit, and the device run's RMSE equals the ctypes binding's mg_run for
the same data and seed.  Run with BPMF priors on both modes and with a binary side matrix on
mode 0 (GpuMacauPrior)."""
import numpy as np
import pytest

from macau_b200 import workloads
from tests import cpp_host
from tests.gpu_helpers import gpu_sampler

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("with_side", [False, True])
def test_prior_adapters_match_the_device_run(tmp_path, with_side):
    exe = cpp_host.build(tmp_path, "prior_adapter_check")
    w = workloads.bpmf_uniform(nrow=300, ncol=200, nobs=6000, seed=3)
    K, burnin, nsamples, seed = 8, 4, 4, 17
    side = None
    if with_side:
        rng = np.random.default_rng(2)
        nfeat = 50
        key = np.unique(rng.integers(0, 300 * nfeat, size=1500))
        side = ((key // nfeat).astype(np.int32), (key % nfeat).astype(np.int32), nfeat)
        w = dict(w, side=(side[0], side[1], None, (300, nfeat)))
    cpp_host.write_data(tmp_path / "d.bin", w, K, burnin, nsamples, side)
    code, out, err = cpp_host.run(exe, tmp_path / "d.bin", seed)
    assert code == 0, (out, err)
    assert float(out["LATENT_DIFF"]) == 0.0, out
    assert float(out["LAMBDA_DIFF"]) == 0.0, out
    assert int(out["CHECKS"]) == 3, out
    s = gpu_sampler(w, K, 2.0, seed, burnin=burnin, nsamples=nsamples, init=False)
    s.run()
    r = s.rmse()[0]
    link = float(np.linalg.norm(s.beta(0))) if with_side else float("nan")
    s.close()
    assert abs(float(out["RMSE"]) - r) <= 1e-12 * r, (out["RMSE"], r)
    if with_side:
        assert abs(float(out["LINKNORM"]) - link) <= 1e-12 * link
    else:
        assert np.isnan(float(out["LINKNORM"]))
