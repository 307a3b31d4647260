"""The multi-rank bench path on CPU: two gloo ranks shard frames with no overlap
and reduce their step times to the slowest rank's."""
import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from topos_codec_b200 import sharding


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        mine = sharding.rank_frames(rank, 4)
        times = [10.0 + rank, 5.0 - rank]
        red = sharding.max_over_ranks(times)
        q.put((rank, mine, red))
    finally:
        dist.destroy_process_group()


def test_two_rank_sharding_and_max_reduction():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, f0, red0), (r1, f1, red1) = res
    assert not set(f0) & set(f1)
    assert red0 == red1 == [11.0, 5.0]


def test_single_process_reduction_is_identity():
    assert sharding.max_over_ranks([1.5, 2.5]) == [1.5, 2.5]
