"""CPU tests of the multi-rank path with the gloo backend (world size 2):
row shards cover the table exactly, the all-reduce of the shards' group
vectors equals the star-join of the whole table (shards computed by the
oracle on CPU), and a rank that dies before the exchange makes the other
rank's collective fail within the process-group timeout instead of hanging."""
import datetime
import multiprocessing as mp
import os
import socket

import numpy as np
import pytest

from memory_database_b200.distributed import reduce_group_sums, shard_range


def test_shard_ranges_cover_every_row_once():
    for n in (0, 1, 7, 1000, 600_000_001):
        for world in (1, 2, 3, 8):
            spans = [shard_range(n, r, world) for r in range(world)]
            assert spans[0][0] == 0 and spans[-1][1] == n
            assert all(spans[r][1] == spans[r + 1][0] for r in range(world - 1))
            sizes = [e - b for b, e in spans]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        shard_range(10, 2, 2)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _table():
    rng = np.random.default_rng(77)
    sizes, groups = [3000, 200, 1400, 255], [4, 4, 4, 4]
    dv = []
    for s_, g in zip(sizes, groups):
        c = rng.integers(0, g, s_).astype(np.int8)
        c[rng.random(s_) < 0.4] = 127
        dv.append(c)
    n = 200_003
    fk = [rng.integers(0, s_, n).astype(np.int32) for s_ in sizes]
    m1 = rng.integers(1, 10000, n).astype(np.int32)
    m2 = rng.integers(-100, 100, n).astype(np.int32)
    return dv, fk, [64, 16, 4, 1], m1, m2, 256


def _rank_main(rank, world, port, mode, q):
    import torch
    import torch.distributed as dist
    import oracle
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=5))
    try:
        dv, fk, factor, m1, m2, G = _table()
        b, e = shard_range(len(m1), rank, world)
        gs, tot, _ = oracle.starjoin(dv, fk, factor, m1, m2, G, aggs=(1, 3), row_range=(b, e))
        t = torch.from_numpy(np.ascontiguousarray(gs))
        if mode == "die" and rank == 1:
            q.put((rank, "left"))
            q.close()
            q.join_thread()  # the message is out before the process goes
            os._exit(0)  # leaves between steps, before the exchange
        try:
            reduce_group_sums(t)
            q.put((rank, t.numpy().tolist()))
        except Exception as ex:  # the peer is gone: the collective fails
            q.put((rank, "error: " + type(ex).__name__))
    finally:
        if mode != "die":
            dist.destroy_process_group()


def _run(mode):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_rank_main, args=(r, 2, port, mode, q)) for r in range(2)]
    for p in ps:
        p.start()
    out = dict(q.get(timeout=120) for _ in ps)
    for p in ps:
        p.join(timeout=60)
        if p.is_alive():
            p.kill()
    return out


def test_allreduce_of_shards_equals_whole_table():
    import oracle
    out = _run("ok")
    dv, fk, factor, m1, m2, G = _table()
    whole, _, _ = oracle.starjoin(dv, fk, factor, m1, m2, G, aggs=(1, 3))
    for r in (0, 1):
        assert np.array_equal(np.array(out[r], dtype=np.int64), whole)


def test_rank_that_leaves_makes_the_exchange_fail_not_hang():
    out = _run("die")
    assert out[1] == "left"
    assert out[0].startswith("error")
