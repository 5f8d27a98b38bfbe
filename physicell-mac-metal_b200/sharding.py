"""Instance sharding across GPUs (one process per GPU).

Independent simulations need no exchange between GPUs: the instance set is
split once, before any device work, and every rank builds a batch from its
own shard.  The split is a greedy longest-processing-time packing on each
instance's predicted bytes per step: heaviest first, each to the rank with
the least load so far (ties to the lower rank).  It depends only on the
weights, so every rank computes the same split without communicating.
"""


def partition(weights, world):
    """Split range(len(weights)) into 'world' shards (sorted index lists)
    with near-equal total weight; every index lands in exactly one shard."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(weights)), key=lambda i: (-weights[i], i))
    loads = [0] * world
    parts = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (loads[k], k))
        parts[r].append(i)
        loads[r] += weights[i]
    return [sorted(p) for p in parts]


def shard_loads(weights, parts):
    return [sum(weights[i] for i in p) for p in parts]
