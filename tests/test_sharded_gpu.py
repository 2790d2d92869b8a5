"""The row-sharded chain's library side on one GPU: two contexts play two ranks (each samples
its row range of every half-sweep, mg_set_row_range), the new rows are exchanged between their
latent buffers on the device (mg_latents_device, then mg_latents_changed), and each updates its
hyperparameters locally.  Both must follow a single context's chain bit for bit, in FP64 mode
and in mixed mode (the tensor-core sampler at K = 32).  The contexts run one after the other; no
kernel waits on another."""
import numpy as np
import pytest

from macau_b200 import _lib, sharded, workloads
from tests.gpu_helpers import gpu_sampler, train_matrix

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("compute,K", [(_lib.MG_COMPUTE_FP64, 10), (_lib.MG_COMPUTE_MIXED, 32)])
def test_two_row_ranges_follow_the_single_context_chain(compute, K):
    import torch
    w = workloads.bpmf_powerlaw(scale=0.02, seed=4)
    Y = train_matrix(w)
    lengths = [np.diff(Y.tocsr().indptr), np.diff(Y.indptr)]
    ranges = [sharded.balanced_row_ranges(lengths[m], 2) for m in (0, 1)]
    thr = 512  # one split threshold for every context (split rows included)
    ref = gpu_sampler(w, K, 2.0, 7, compute=compute, init=False)
    ref.set_option("split_threshold", thr)
    ref.init()
    ranks = []
    for r in range(2):
        s = gpu_sampler(w, K, 2.0, 7, compute=compute, init=False)
        s.set_option("split_threshold", thr)
        s.init()
        for m in (0, 1):
            s.set_row_range(m, *ranges[m][r])
        ranks.append(sharded.LibraryBackend(s, torch.device("cuda:0")))
    for it in range(3):
        for mode in (0, 1):
            ref.sample_latents(mode, it)
            for b in ranks:
                b.sample_rows(mode, it)
            torch.cuda.synchronize()
            views = [b.latent_view(mode) for b in ranks]
            for r, (lo, hi) in enumerate(ranges[mode]):
                views[1 - r][lo:hi] = views[r][lo:hi]
            torch.cuda.synchronize()
            for b in ranks:
                b.latents_written(mode)
        for mode in (0, 1):
            ref.update_prior(mode, it)
            for b in ranks:
                b.update_prior(mode, it)
        for mode in (0, 1):
            want = ref.latents(mode)
            for b in ranks:
                np.testing.assert_array_equal(b.s.latents(mode), want)
            for b in ranks:
                np.testing.assert_array_equal(b.s.hyper(mode)[1], ref.hyper(mode)[1])
    for b in ranks:
        b.s.close()
    ref.close()


def test_row_range_is_checked():
    w = workloads.bpmf_uniform(nrow=100, ncol=80, nobs=1500, seed=1)
    s = gpu_sampler(w, 4, 1.0, 1)
    with pytest.raises(_lib.MacauError):
        s.set_row_range(0, 50, 101)
    with pytest.raises(_lib.MacauError):
        s.set_row_range(1, 30, 20)
    s.set_row_range(0, 0, 0)  # an empty range samples nothing
    before = s.latents(0)
    s.sample_latents(0, 0)
    np.testing.assert_array_equal(s.latents(0), before)
    s.close()
