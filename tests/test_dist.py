"""The multi-GPU path of bench.py on CPU ranks (gloo, world size 2).

The step does not shard (one lattice per GPU, "replicas only"): what runs
across ranks is the barrier around the timed region, the max of the per-rank
times and the whole-job throughput computed from it. Each rank here plays a
GPU with a made-up time; both must agree on the max and on the throughput,
and a rank that is slower must set it.
"""
import os
import socket
import sys
from pathlib import Path

import pytest
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parents[1]


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank: int, world: int, port: int, q) -> None:
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    sys.path.insert(0, str(ROOT))
    import bench
    d = bench.Dist(backend="gloo")
    d.init()
    try:
        d.barrier()
        ms = 100.0 + 25.0 * rank          # rank 1 is the slow one
        ms_max = d.max(ms)
        value = bench.whole_job_mlups(d.world, 4_194_304, 1000, ms_max)
        d.barrier()
        q.put((rank, ms_max, value))
    finally:
        d.close()


@pytest.mark.timeout(120)
def test_two_gloo_ranks_agree_on_the_max_time_and_the_throughput():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(90)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    got = sorted(q.get(timeout=5) for _ in range(world))
    for rank, ms_max, value in got:
        assert ms_max == 125.0
        assert value == pytest.approx(2 * 4_194_304 * 1000 / 0.125 / 1e6)


def test_single_rank_needs_no_process_group():
    sys.path.insert(0, str(ROOT))
    import bench
    d = bench.Dist(backend="gloo")
    assert d.world == int(os.environ.get("WORLD_SIZE", "1"))
    if d.world == 1:
        d.init()
        assert not d.pg and d.max(3.5) == 3.5
        d.barrier()
        d.close()
