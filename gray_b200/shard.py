"""Sharding of independent renders across GPUs (one process per GPU).

Rays and renders are independent (driver.cl:47-51: one work-item per ray,
no communication), so multi-GPU runs need no data-path collective: every
rank integrates its own share and results are gathered on the host.
"""


def partition(sizes, world):
    """Assign items of the given sizes (ray counts) to `world` ranks by the
    greedy longest-processing-time rule; deterministic, ties broken by index.
    Returns one sorted index list per rank."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(sizes)), key=lambda i: (-sizes[i], i))
    load = [0] * world
    share = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        share[r].append(i)
        load[r] += sizes[i]
    return [sorted(s) for s in share]


def my_share(items, sizes, rank, world):
    """The items this rank renders."""
    return [items[i] for i in partition(sizes, world)[rank]]


def row_block(n_rows, rank, world):
    """The contiguous camera rows [begin, begin + count) that `rank` of
    `world` integrates when one render is split by rows: counts differ by
    at most one, earlier ranks take the extra rows.  A render's rays are
    row-major (driver.cl:47-51), so a row block is a contiguous ray range
    and the blocks concatenate, in rank order, into the whole render."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("rank must be in [0, world)")
    base, extra = divmod(n_rows, world)
    return rank * base + min(rank, extra), base + (1 if rank < extra else 0)


def gather_rows(dist, block, n_width, n_height, group=None):
    """Rank 0 assembles a render's SoA state [n_data, n_width * n_height]
    from every rank's row block [n_data, n_width * rows]; the other ranks
    get None.  Host memory, over `group` (a gloo group when the default
    process group is NCCL)."""
    import numpy as np
    import torch
    world, rank = dist.get_world_size(group), dist.get_rank(group)
    counts = [row_block(n_height, k, world)[1] * n_width for k in range(world)]
    if block.shape[1] != counts[rank]:
        raise ValueError("block has %d rays, rank %d owns %d" % (block.shape[1], rank, counts[rank]))
    t = torch.zeros((block.shape[0], max(counts)), dtype=torch.float64)
    t[:, :block.shape[1]] = torch.from_numpy(np.ascontiguousarray(block, dtype=np.float64))
    bufs = [torch.zeros_like(t) for _ in range(world)] if rank == 0 else None
    dist.gather(t, bufs, dst=0, group=group)
    if rank != 0:
        return None
    return np.concatenate([b[:, :c].numpy() for b, c in zip(bufs, counts)], axis=1)
