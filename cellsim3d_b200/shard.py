"""Sharding of ensembles across ranks (one process per GPU).

Instances of an ensemble are independent simulations, so they shard with no
data-path collective: each rank builds one ensemble context from its share of
the instances and steps it alone.  The only communication is at the end
(timing reductions and a gather of per-instance results).  Single systems do
not shard; under several ranks they run as replicas.
"""
import heapq


def partition(costs, world):
    """Greedy bin-packing of instances onto `world` ranks by predicted cost
    (largest first onto the least-loaded rank; ties by rank).  Returns, for
    each rank, its instance indices in ascending order.  Deterministic, so
    every rank computes the same partition without communicating."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(costs)), key=lambda k: (-float(costs[k]), k))
    heap = [(0.0, r) for r in range(world)]
    parts = [[] for _ in range(world)]
    for k in order:
        load, r = heapq.heappop(heap)
        parts[r].append(k)
        heapq.heappush(heap, (load + float(costs[k]), r))
    return [sorted(p) for p in parts]


def predicted_cost(state, steps=1, growth=0.0):
    """Cost model of one instance: node-steps, with the population growing
    linearly at `growth` cells per cell per step (0 for non-dividing runs)."""
    n0 = float(state["n"])
    return n0 * 180.0 * steps * (1.0 + 0.5 * growth * steps)


def gather_results(local, group=None):
    """All ranks' per-instance results (dicts keyed by instance index),
    merged; one object all-gather over the default process group."""
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return dict(local)
    out = [None] * dist.get_world_size(group)
    dist.all_gather_object(out, dict(local), group=group)
    merged = {}
    for part in out:
        for k, v in part.items():
            if k in merged:
                raise RuntimeError("instance %r reported by two ranks" % (k,))
            merged[k] = v
    return merged
