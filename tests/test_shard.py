"""Multi-rank host logic (shard.py) on the CPU with gloo, world size 2: the
scan partition is deterministic, covers every scan once and is balanced;
the max / sum over ranks and the end-of-run gather behave (no GPU)."""
import os
import socket

import pytest
import torch.multiprocessing as mp

import shard


def test_partition_covers_and_balances():
    rng = __import__("numpy").random.default_rng(0)
    work = list(rng.integers(10, 200, size=64) * rng.choice([19200, 76800, 307200], size=64))
    for world in (1, 2, 3, 8):
        parts = shard.partition(work, world)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(work)))
        loads = [sum(work[i] for i in p) for p in parts]
        assert max(loads) <= sum(work) / world + max(work)
        assert parts == shard.partition(work, world)  # deterministic
    with pytest.raises(ValueError):
        shard.partition(work, 0)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank, world, port, work, q):
    import datetime

    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    mine = shard.partition(work, world)[rank]
    local = float(sum(work[i] for i in mine))
    mx = shard.max_over_ranks(local, dist)
    tot = shard.sum_over_ranks(local, dist)
    stats = shard.gather_stats({"rank": rank, "scans": mine, "load": local}, dist)
    dist.barrier()
    dist.destroy_process_group()
    q.put((rank, mine, mx, tot, stats))


def test_two_gloo_ranks_shard_without_overlap():
    work = [5.0, 3.0, 9.0, 1.0, 7.0, 2.0, 8.0]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_rank, args=(r, 2, port, work, q)) for r in range(2)]
    for p in ps:
        p.start()
    res = sorted(q.get(timeout=120) for _ in ps)
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, m0, mx0, t0, s0), (r1, m1, mx1, t1, s1) = res
    assert sorted(m0 + m1) == list(range(len(work))) and not set(m0) & set(m1)
    loads = [sum(work[i] for i in m0), sum(work[i] for i in m1)]
    assert mx0 == mx1 == max(loads) and t0 == t1 == sum(work)
    assert [d["rank"] for d in s0] == [0, 1] and s0 == s1
