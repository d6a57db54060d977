"""The multi-process host path on CPU: two gloo ranks shard a mixed batch of sequences (the
48-sequence batching configuration) by voxels x sources, agree on the max-over-ranks timing the
bench reports, and gather per-rank statistics.  No GPU and no collective on the data path."""
import os
import socket

import pytest

torch = pytest.importorskip("torch")

from probabilistic_mapping_b200.shard import sequence_weight, shard_sequences   # noqa: E402

S = 4
MIXED = ([dict(width=320, height=240, num_planes=64)] * 16 + [dict(width=640, height=480, num_planes=128)] * 16 +
         [dict(width=1280, height=720, num_planes=192)] * 16)


def test_shards_cover_all_and_balance():
    for world in (1, 2, 4, 8):
        groups = shard_sequences(MIXED, world, S)
        flat = sorted(i for g in groups for i in g)
        assert flat == list(range(len(MIXED)))
        loads = [sum(sequence_weight(MIXED[i], S) for i in g) for g in groups]
        big = sequence_weight(MIXED[-1], S)
        assert max(loads) - min(loads) <= big   # within one largest job
    assert shard_sequences(MIXED, 2, S) == shard_sequences(MIXED, 2, S)   # deterministic


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, q):
    import sys
    from datetime import timedelta
    import torch.distributed as dist
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    import bench
    from probabilistic_mapping_b200.shard import gather_stats, shard_sequences
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        mine = shard_sequences(MIXED, world, S)[rank]
        t_local = 10.0 + rank   # this rank's timed region (ms)
        t_max = bench.max_over_ranks([t_local, 2.0 * t_local], world)
        stats = gather_stats([len(mine), sum(sequence_weight(MIXED[i], S) for i in mine)])
        q.put((rank, mine, t_max, stats))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_shard_and_reduce():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    out.sort()
    (r0, m0, t0, s0), (r1, m1, t1, s1) = out
    assert sorted(m0 + m1) == list(range(len(MIXED))) and not set(m0) & set(m1)
    assert t0 == t1 == [11.0, 22.0]     # the slowest rank's times, on every rank
    assert s0 == s1 and sum(v[0] for v in s0) == len(MIXED)
