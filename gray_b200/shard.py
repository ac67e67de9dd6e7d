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
