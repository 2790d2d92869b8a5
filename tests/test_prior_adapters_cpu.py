"""The C++ adapters of include/macau_b200_priors.hpp (GpuBPMFPrior / GpuMacauPrior behind the
reference's ILatentPrior, MacauGpuX behind its Macau class) compile against a stand-in of those
two interfaces (tests/cpp/standin) and link against the library; without a GPU the program
reports the library's error instead of running."""
import pytest

from macau_b200 import workloads
from tests import cpp_host


def test_prior_adapters_compile_and_report_a_missing_gpu(tmp_path):
    exe = cpp_host.build(tmp_path, "prior_adapter_check")
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a GPU is present: tests/test_zy_prior_adapters_gpu.py runs the program")
    except ImportError:
        pass
    w = workloads.bpmf_uniform(nrow=60, ncol=40, nobs=600, seed=1)
    cpp_host.write_data(tmp_path / "d.bin", w, 4, 1, 1)
    code, out, _ = cpp_host.run(exe, tmp_path / "d.bin", 3)
    assert code == 2
    assert "ERROR" in out
