"""The replica path of `bench.py --gpus N` on CPU: two gloo ranks check the
max-over-ranks timing, the whole-job rate and the round-robin sharding of
independent designs (no GPU, no collective on a data path)."""

import os
import socket

import pytest

torch = pytest.importorskip("torch")
import torch.multiprocessing as mp  # noqa: E402

from toptimization_b200 import replicas  # noqa: E402


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank: int, world: int, port: int, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    r = replicas.from_env()
    replicas.init(r, backend="gloo", timeout_s=60)
    try:
        replicas.barrier(r)
        t = replicas.max_over_ranks(1.0 + rank, r)  # rank 1 is the slow one
        mine = replicas.shard(list(range(10)), r)
        rate = replicas.job_rate(5, t, r)
        out.put((rank, t, mine, rate))
    finally:
        replicas.finish(r)


def test_two_gloo_ranks():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(i, world, port, q)) for i in range(world)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, t0, s0, v0), (r1, t1, s1, v1) = res
    assert t0 == t1 == 2.0                       # both ranks see the slowest time
    assert s0 == [0, 2, 4, 6, 8] and s1 == [1, 3, 5, 7, 9]
    assert v0 == v1 == pytest.approx(2 * 5 / 2.0)


def test_single_rank_needs_no_group():
    r = replicas.Ranks(0, 1, 0)
    replicas.init(r, backend="gloo")
    assert replicas.max_over_ranks(3.5, r) == 3.5
    assert replicas.shard([1, 2, 3], r) == [1, 2, 3]
    assert replicas.job_rate(4, 2.0, r) == 2.0
