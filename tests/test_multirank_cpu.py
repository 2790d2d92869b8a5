"""The N > 1 path of bench.py on CPU: two processes with the gloo backend (one per rank, as
torchrun launches them on GPUs).  Each rank runs an independent chain; the ranks agree on the
maximum of their timings and on the whole-job rate, and their chains have distinct seeds."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    os.environ.update(RANK=str(rank), LOCAL_RANK=str(rank), WORLD_SIZE=str(world),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import bench
    r = bench.Ranks("gloo", device="cpu", timeout_s=60)
    try:
        r.barrier()
        seconds = 1.0 + rank  # rank 1 is the slow one
        t_max = r.max(seconds)
        out[rank] = (r.chain_seed(), t_max, r.rate(200, t_max), r.world)
    finally:
        r.close()


@pytest.mark.timeout(120)
def test_two_gloo_ranks_agree_on_max_time_and_whole_job_rate():
    world = 2
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_rank_main, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    seeds = {res[r][0] for r in range(world)}
    assert seeds == {1000, 1001}  # independent chains
    for r in range(world):
        _, t_max, rate, w = res[r]
        assert w == world
        assert t_max == 2.0  # the maximum over ranks, on every rank
        assert rate == pytest.approx(world * 200 / 2.0)  # every rank's sweeps in the slowest time


def test_single_process_needs_no_process_group():
    import bench
    for k in ("RANK", "LOCAL_RANK", "WORLD_SIZE"):
        os.environ.pop(k, None)
    r = bench.Ranks("gloo", device="cpu")
    assert r.world == 1 and r.dist is None and r.chain_seed() == 1000
    assert r.max(3.5) == 3.5 and r.rate(10, 2.0) == 5.0
    r.close()


def test_reference_arm_under_torchrun_prints_one_line():
    # bench.py --impl reference launched like the N > 1 runs: rank 0 times the CPU oracle and
    # prints the one JSON line, the other rank exits 0 without work
    import json
    import socket
    import subprocess
    import sys
    from pathlib import Path

    root = Path(__file__).resolve().parent.parent
    with socket.socket() as so:
        so.bind(("127.0.0.1", 0))
        port = so.getsockname()[1]
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(port), str(root / "bench.py"),
           "--impl", "reference", "--gpus", "2", "--steps", "1", "--warmup", "1",
           "--scale", "0.01"]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=240, cwd=root)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, r.stdout
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["n_gpus"] == 2 and d["value"] > 0
    assert d["cpu_baseline"]["kind"] == "port" and d["e2e"]["h2d_bytes_per_step"] == 0
