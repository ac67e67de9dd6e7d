"""Multi-rank host logic on CPU with the gloo backend (world size 2): the
render partition every rank computes independently covers every render once
and balances rays; the bench's max-over-ranks timing reduction; a rank that
raises is seen by the other as a collective error, not a hang."""
import os
import socket
import sys

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _init(rank, world, port):
    sys.path.insert(0, ROOT)
    import datetime
    dist.init_process_group("gloo", init_method="tcp://127.0.0.1:%d" % port, rank=rank,
                            world_size=world, timeout=datetime.timedelta(seconds=20))


def _partition_worker(rank, world, port, q):
    _init(rank, world, port)
    from gray_b200 import configs, shard
    cfgs = configs.survey()
    sizes = [c["n_width"] * c["n_height"] for c in cfgs]
    mine = shard.partition(sizes, world)[rank]
    got = [None] * world
    dist.all_gather_object(got, mine)
    import bench
    t = bench.max_over_ranks(torch, dist, 1.5 + rank)
    dist.barrier()
    dist.destroy_process_group()
    if rank == 0:
        q.put((got, sizes, t))


def test_partition_and_timing_reduction():
    world, port = 2, free_port()
    ctx = mp.get_context("spawn")
    q = ctx.SimpleQueue()
    ps = [ctx.Process(target=_partition_worker, args=(r, world, port, q)) for r in range(world)]
    for p in ps:
        p.start()
    for p in ps:
        p.join(60)
        assert p.exitcode == 0
    got, sizes, t = q.get()
    allidx = sorted(i for s in got for i in s)
    assert allidx == list(range(len(sizes)))  # disjoint cover
    loads = [sum(sizes[i] for i in s) for s in got]
    assert max(loads) / (sum(loads) / world) < 1.02
    assert t == 2.5  # max over ranks


def _failing_worker(rank, world, port, q):
    _init(rank, world, port)
    try:
        if rank == 1:
            raise RuntimeError("rank 1 fails before its collective")
        import datetime
        t = torch.tensor([1.0])
        work = dist.all_reduce(t, async_op=True)
        ok = work.wait(timeout=datetime.timedelta(seconds=5))
        q.put(("no-error", ok))
    except Exception as e:  # noqa: BLE001 - the point is to see the error
        q.put((type(e).__name__, rank))


def test_failed_rank_is_detected_not_hung():
    """Failure detection on the host: rank 1 dies without joining the
    collective; rank 0's collective ends with an error within its timeout."""
    world, port = 2, free_port()
    ctx = mp.get_context("spawn")
    q = ctx.SimpleQueue()
    ps = [ctx.Process(target=_failing_worker, args=(r, world, port, q)) for r in range(world)]
    for p in ps:
        p.start()
    for p in ps:
        p.join(60)
    res = [q.get() for _ in range(world)]
    assert ("RuntimeError", 1) in res
    other = [r for r in res if r != ("RuntimeError", 1)]
    assert other and other[0][0] != "no-error"


def test_partition_is_deterministic_and_handles_edges():
    from gray_b200 import shard
    assert shard.partition([], 3) == [[], [], []]
    assert shard.partition([5], 2) == [[0], []]
    a = shard.partition([3, 3, 2, 2, 2], 2)
    assert a == shard.partition([3, 3, 2, 2, 2], 2)
    with pytest.raises(ValueError):
        shard.partition([1], 0)


def _rows_worker(rank, world, port, q):
    """Each rank traces its row block of a small torus render with the CPU
    oracle (standing in for its GPU), rank 0 gathers; the GPU side of the
    row window is checked by test_row_blocks_concatenate_to_the_render."""
    _init(rank, world, port)
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import numpy as np
    import oracle as O
    from gray_b200 import configs, shard
    cfg = dict(configs.scaled(configs.TORUS_RT_1024, 6), n_width=7, n_height=5, n_dump=3)
    begin, rows = shard.row_block(cfg["n_height"], rank, world)
    rays = begin * cfg["n_width"] + np.arange(rows * cfg["n_width"], dtype=np.int64)
    st, _, _ = O.trace(cfg, rays)
    full = shard.gather_rows(dist, st.T, cfg["n_width"], cfg["n_height"])
    blocks = [None] * world
    dist.all_gather_object(blocks, (begin, rows))
    dist.barrier()
    dist.destroy_process_group()
    if rank == 0:
        ref, _, _ = O.trace(cfg, np.arange(cfg["n_width"] * cfg["n_height"], dtype=np.int64))
        q.put((blocks, bool(np.array_equal(full, ref.T)), full.shape))


def test_row_partition_gathers_to_the_one_rank_layout():
    world, port = 2, free_port()
    ctx = mp.get_context("spawn")
    q = ctx.SimpleQueue()
    ps = [ctx.Process(target=_rows_worker, args=(r, world, port, q)) for r in range(world)]
    for p in ps:
        p.start()
    for p in ps:
        p.join(120)
        assert p.exitcode == 0
    blocks, same, shape = q.get()
    assert blocks == [(0, 3), (3, 2)]  # every row once, in rank order
    assert same and shape == (16, 35)


def test_row_block_edges():
    from gray_b200 import shard
    assert [shard.row_block(10, r, 3) for r in range(3)] == [(0, 4), (4, 3), (7, 3)]
    assert [shard.row_block(2, r, 4) for r in range(4)] == [(0, 1), (1, 1), (2, 0), (2, 0)]
    with pytest.raises(ValueError):
        shard.row_block(4, 2, 2)
