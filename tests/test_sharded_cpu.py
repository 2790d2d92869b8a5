"""The row-sharded chain (macau_b200/sharded.py) on CPU: two gloo ranks each sample their row
range of every half-sweep with the CPU oracle, all-gather the new rows, and update the
hyperparameters locally; the result must be the single-rank oracle chain, bit for bit (the
draws are keyed by the global row index and every rank sees the same latents).  Also the
entry-balanced row partition."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from macau_b200 import sharded, workloads


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _workload():
    return workloads.bpmf_uniform(nrow=300, ncol=220, nobs=7000, seed=21)


def _row_lengths(w):
    from tests.gpu_helpers import train_matrix
    Y = train_matrix(w)
    return [np.diff(Y.tocsr().indptr), np.diff(Y.indptr)]


K, ALPHA, SEED, SWEEPS = 8, 3.0, 99, 3


def _rank_main(rank, world, port, out):
    import datetime

    import torch.distributed as dist

    from oracle import oracle as orc
    from tests.gpu_helpers import oracle_model
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    orc.set_threads(1)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        w = _workload()
        m = oracle_model(w, K, ALPHA, SEED)
        chain = sharded.ShardedChain(sharded.OracleBackend(m), dist, rank, world,
                                     _row_lengths(w))
        for it in range(SWEEPS):
            chain.sweep(it)
        out[rank] = (m.latents(0), m.latents(1), m.Lambda(0), m.Lambda(1), chain.ranges)
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(180)
def test_two_gloo_ranks_reproduce_the_single_rank_chain():
    from oracle import oracle as orc
    from tests.gpu_helpers import oracle_model
    world = 2
    port = _free_port()
    with mp.Manager() as mgr:
        out = mgr.dict()
        mp.spawn(_rank_main, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    orc.set_threads(1)
    w = _workload()
    m = oracle_model(w, K, ALPHA, SEED)
    for it in range(SWEEPS):
        for mode in (0, 1):
            assert m.sample_mode(mode, it) == 0
        for mode in (0, 1):
            assert m.update_prior(mode, it) == 0
    want = (m.latents(0), m.latents(1), m.Lambda(0), m.Lambda(1))
    for r in range(world):
        for got, ref in zip(res[r][:4], want):
            np.testing.assert_array_equal(got, ref)
    # the two ranks really split the rows
    for mode in (0, 1):
        (a0, b0), (a1, b1) = res[0][4][mode]
        assert a0 == 0 and b0 == a1 and b1 == w["shape"][mode] and 0 < b0 < b1


def test_balanced_row_ranges():
    rng = np.random.default_rng(3)
    lengths = rng.integers(1, 200, size=1000)
    lengths[10] = 50000  # one heavy row
    for world in (1, 2, 3, 8):
        ranges = sharded.balanced_row_ranges(lengths, world)
        assert len(ranges) == world
        assert ranges[0][0] == 0 and ranges[-1][1] == len(lengths)
        for (a, b), (c, d) in zip(ranges, ranges[1:]):
            assert b == c and a <= b
        if world > 1:
            light = lengths.copy()
            light[10] = 100
            shares = [light[a:b].sum() for a, b in sharded.balanced_row_ranges(light, world)]
            assert max(shares) <= light.sum() / world + 200  # within one row of the target
    assert sharded.balanced_row_ranges([], 3) == [(0, 0), (0, 0), (0, 0)]
