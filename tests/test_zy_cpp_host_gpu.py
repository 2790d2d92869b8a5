"""The C++ host class (include/macau_b200.hpp) on the GPU: a compiled C++ program runs a BPMF
chain through MacauGpu (the reference's Macau-shaped interface) and gets the chain that the
ctypes binding gets for the same data and seed."""
import numpy as np
import pytest

from macau_b200 import workloads
from tests import cpp_host
from tests.gpu_helpers import gpu_sampler

pytestmark = pytest.mark.gpu


def test_cpp_host_matches_the_ctypes_binding(tmp_path):
    exe = cpp_host.build(tmp_path)
    w = workloads.bpmf_uniform(nrow=300, ncol=200, nobs=6000, seed=3)
    K, burnin, nsamples, seed = 8, 5, 5, 5
    cpp_host.write_data(tmp_path / "d.bin", w, K, burnin, nsamples)
    code, out, err = cpp_host.run(exe, tmp_path / "d.bin", seed)
    assert code == 0, (out, err)
    s = gpu_sampler(w, K, 2.0, seed, burnin=burnin, nsamples=nsamples, init=False)
    s.run()
    want = {"RMSE": s.rmse()[0], "PRED": float(np.sum(s.predictions())),
            "STDS": float(np.sum(s.stds())), "TEST": float(np.sum(s.test_data()))}
    s.close()
    for k, v in want.items():
        assert abs(float(out[k]) - v) <= 1e-9 * max(1.0, abs(v)), (k, out[k], v)
