"""The hyperprior entry point that allocates no device memory (mg_normal_wishart_noalloc).

It is for callers that cannot call cudaMalloc when they resample the hyperparameters: a process
whose memory pool already owns the device memory, or a loop that cannot take cudaMalloc's
implicit synchronisation.  Its scratch lives in a fixed array inside the library.  These tests
call it through the C ABI and check it against the context entry point mg_update_prior, on two
calls in a row (so the second call runs on the array the first one left behind), at K on both
sides of 32 (the K <= 32 kernels and the generic ones, whose workspace is carved from the array)
and at row counts on both sides of its 64-part reduction cap (beyond 8,192 rows its partition
differs from the context's, so the sums differ by rounding only), and check that sizes beyond
its fixed scratch and invalid prior parameters are refused.
"""
import ctypes as C

import numpy as np
import pytest

from macau_b200 import _lib, workloads
from tests.gpu_helpers import gpu_sampler, relerr

FP64_TOL = 1e-9  # the FP64 parity bar of the other GPU tests


def call_noalloc(U, N, K, mu0, T, seed, sweep, mode, mu_out, Lambda_out, stream):
    err = C.create_string_buffer(256)
    code = _lib.lib().mg_normal_wishart_noalloc(U, N, K, K, mu0, 2.0, T, K, seed, sweep, mode,
                                                mu_out, Lambda_out, stream, err, 256)
    return code, err.value.decode()


@pytest.mark.gpu
@pytest.mark.parametrize("N", [300, 20000])
@pytest.mark.parametrize("K", [10, 48, 64])
def test_noalloc_hyperprior_matches_update_prior_on_two_calls(K, N):
    import torch

    seed = 21 + K
    w = workloads.bpmf_uniform(nrow=N, ncol=200, nobs=max(6000, 3 * N), seed=11)
    s = gpu_sampler(w, K, 4.0, seed=seed)  # BPMF prior: mu0 = 0, kappa = 2, T = I, nu = K
    dev = torch.device("cuda:0")
    mu0 = torch.zeros(K, dtype=torch.float64, device=dev)
    T = torch.eye(K, dtype=torch.float64, device=dev)
    mu = torch.empty(K, dtype=torch.float64, device=dev)
    Lam = torch.empty((K, K), dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream().cuda_stream
    rng = np.random.default_rng(4)
    for sweep in (5, 6):
        U = rng.normal(0.2, 1.0, size=(N, K))
        s.set_latents(0, U)
        s.update_prior(0, sweep)  # the existing entry point
        mu_ref, Lam_ref, _ = s.hyper(0)
        Ud = torch.from_numpy(U).to(dev)
        code, msg = call_noalloc(Ud.data_ptr(), N, K, mu0.data_ptr(), T.data_ptr(), seed, sweep,
                                 0, mu.data_ptr(), Lam.data_ptr(), stream)
        assert code == 0, msg
        torch.cuda.synchronize()
        # both write K x K column-major; compare the raw memory the same way
        assert relerr(Lam.cpu().numpy(), Lam_ref) < FP64_TOL
        assert relerr(mu.cpu().numpy(), mu_ref) < FP64_TOL
    s.close()


def test_noalloc_rejects_sizes_beyond_its_scratch():
    code, msg = call_noalloc(None, 10, 65, None, None, 0, 0, 0, None, None, None)
    assert code == -1
    assert "K must be in [1, 64]" in msg


@pytest.mark.parametrize("nu,kappa", [(9, 2.0), (10, 0.0), (10, -1.0), (10, float("nan"))])
def test_noalloc_rejects_invalid_prior_parameters(nu, kappa):
    # checked before any device work: the pointers are never dereferenced
    fake = 256
    err = C.create_string_buffer(256)
    code = _lib.lib().mg_normal_wishart_noalloc(fake, 100, 10, 10, fake, kappa, fake, nu, 0, 0,
                                                0, fake, fake, None, err, 256)
    assert code == -1
    assert "nu >= K and kappa > 0" in err.value.decode()
