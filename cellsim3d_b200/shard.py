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


# Population model of a dividing instance, fitted on a B200 to 2000-step runs
# of 15 instances of the 256-instance ensemble (1..511 initial cells, box of
# side 30) and to the whole ensemble's count after 10,000 steps (48,304 cells
# after step 1, 463,487 at the end):
#  * the unit-radius initial cells exceed every division volume, so every
#    cell divides at step 1;
#  * afterwards the population grows as a Richards (generalised logistic)
#    curve, dn/dt = r n (1 - (n / K)^nu), with r = 6.91e-4 per step, a
#    capacity K of 0.0705 cells per unit of box volume and a crowding
#    exponent nu = 1.79: growth slows later, and then faster, than a plain
#    logistic (nu = 1) does.  Fitted counts are within 12 % of the measured
#    ones at step 2000 (most within 7 %) and the ensemble's total within 1 %
#    at step 10,000.  A daughter divides once its shape has relaxed (the
#    sphericity test), about 450 steps after its birth when it has room; the
#    pressure growth rate and the division volume barely change that
#    (single-cell runs of the oracle at growth rates 0.001 to 0.004 and
#    division volumes 2.6 to 3.2 divide at the same steps to within 1 %), and
#    crowding slows it.
GROWTH_RATE = 6.91e-4
CAPACITY_PER_VOLUME = 0.0705
CROWDING_EXPONENT = 1.79


def predicted_population(n0, steps, box, dividing=True, div_steps=None):
    """Expected cell count after each of `steps` steps (array of length
    steps) of an instance of n0 cells in a box of sides `box`."""
    import numpy as np
    t = np.arange(1, steps + 1, dtype=np.float64)
    if not dividing or n0 <= 0:
        return np.full(steps, float(n0))
    K = max(CAPACITY_PER_VOLUME * float(box[0]) * float(box[1]) * float(box[2]), 2.0 * n0)
    n1 = 2.0 * n0
    nu = CROWDING_EXPONENT
    n = K / (1.0 + ((K / n1) ** nu - 1.0) * np.exp(-GROWTH_RATE * nu * (t - 1.0))) ** (1.0 / nu)
    if div_steps is not None and div_steps < steps:
        n[max(div_steps, 1):] = n[max(div_steps, 1) - 1]   # no division after div_steps
    return n


def predicted_cost(state, steps=1, params=None):
    """Cost model of one instance: node-steps over `steps` steps.  Without
    params, or for a non-dividing instance (growth rate 0), the cell count
    stays n0; a dividing instance follows predicted_population."""
    n0 = float(state["n"])
    if params is None or not params.get("growth_rate", 0.0) or steps <= 0:
        return n0 * 180.0 * steps
    pop = predicted_population(n0, int(steps), params["box_len"], True, params.get("div_time_steps"))
    return 180.0 * float(pop.sum())


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
