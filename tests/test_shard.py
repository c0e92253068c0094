"""Ensemble sharding across ranks: the partition (every instance on exactly
one rank, balanced, identical on every rank) and the end-of-run gather, with
two gloo ranks on the CPU."""
import os
import socket

import numpy as np

from cellsim3d_b200 import shard
from cellsim3d_b200 import workloads as W


def test_partition_covers_every_instance_once():
    rng = np.random.default_rng(3)
    costs = rng.lognormal(3.0, 1.5, size=257)
    for world in (1, 2, 3, 8):
        parts = shard.partition(costs, world)
        assert len(parts) == world
        flat = sorted(k for p in parts for k in p)
        assert flat == list(range(len(costs)))
        loads = [costs[p].sum() for p in parts]
        # greedy largest-first: no rank exceeds the mean by more than the largest item
        assert max(loads) <= np.mean(loads) + costs.max() + 1e-9
        assert shard.partition(costs, world) == parts


def test_partition_of_the_256_instance_ensemble():
    insts = W.config4()
    costs = [shard.predicted_cost(st) for _, st in insts]
    parts = shard.partition(costs, 8)
    loads = np.array([sum(costs[k] for k in p) for p in parts])
    assert sorted(k for p in parts for k in p) == list(range(256))
    assert loads.max() / loads.mean() < 1.05


# Cell counts after 2000 steps of the 16-instance stratified subset of the
# 256-instance ensemble, measured on a B200 by
# tests/test_gpu_fullsize.py::test_ensemble256_subset_full_size (initial
# cells -> cells after 2000 steps).
MEASURED_2000 = {1: 9, 511: 1963, 47: 372, 275: 1428, 67: 515, 10: 77, 4: 31, 22: 166, 123: 815, 2: 15,
                 32: 267, 398: 1753, 15: 123, 175: 1044, 5: 41}


# the whole 256-instance ensemble on a B200: cells after step 1 and after step 10,000
MEASURED_10K_TOTAL = (48304, 463487)


def test_population_model_matches_measured_growth():
    errs = {}
    for p, st in W.config4():
        n0 = st["n"]
        if n0 not in MEASURED_2000:
            continue
        pred = shard.predicted_population(n0, 2000, p["box_len"])[-1]
        errs[n0] = abs(pred - MEASURED_2000[n0]) / MEASURED_2000[n0]
        assert abs(pred - MEASURED_2000[n0]) <= max(2.0, 0.12 * MEASURED_2000[n0]), (n0, pred)
    assert set(errs) == set(MEASURED_2000) and np.median(list(errs.values())) < 0.07


def test_population_model_matches_the_ensemble_after_10k_steps():
    insts = W.config4()
    after1 = sum(shard.predicted_population(st["n"], 1, p["box_len"])[-1] for p, st in insts)
    total = sum(shard.predicted_population(st["n"], 10000, p["box_len"])[-1] for p, st in insts)
    assert after1 == MEASURED_10K_TOTAL[0]
    assert abs(total - MEASURED_10K_TOTAL[1]) < 0.02 * MEASURED_10K_TOTAL[1], total


def test_cost_model_uses_growth_and_steps():
    insts = W.config4()
    p, st = insts[0]
    flat = dict(p, growth_rate=0.0)
    assert shard.predicted_cost(st, 100, flat) == st["n"] * 180.0 * 100
    assert shard.predicted_cost(st, 100) == st["n"] * 180.0 * 100
    # dividing: every cell divides at step 1, then more
    assert shard.predicted_cost(st, 100, p) > 2 * st["n"] * 180.0 * 99
    # a growing ensemble: small instances grow proportionally more than large ones
    costs = {st["n"]: shard.predicted_cost(st, 10000, p) / (st["n"] * 180.0 * 10000) for p, st in insts}
    assert costs[min(costs)] > costs[max(costs)]
    # 8 ranks over the 10k-step run stay balanced under the growth model
    c = [shard.predicted_cost(st, 10000, p) for p, st in insts]
    loads = np.array([sum(c[k] for k in part) for part in shard.partition(c, 8)])
    assert loads.max() / loads.mean() < 1.05


def test_partition_more_ranks_than_instances():
    parts = shard.partition([5.0, 1.0], 4)
    assert sorted(k for p in parts for k in p) == [0, 1]
    assert sum(1 for p in parts if not p) == 2


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, costs, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        mine = shard.partition(costs, world)[rank]
        local = {k: {"rank": rank, "cells": 10 * k} for k in mine}
        merged = shard.gather_results(local)
        q.put((rank, mine, sorted(merged), {k: v["rank"] for k, v in merged.items()}))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_shard_and_gather():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    costs = [float(c) for c in np.random.default_rng(7).integers(1, 500, size=37)]
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, costs, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(2)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    res.sort()
    (r0, mine0, all0, owner0), (r1, mine1, all1, owner1) = res
    assert set(mine0).isdisjoint(mine1)
    assert sorted(mine0 + mine1) == list(range(len(costs)))
    assert all0 == all1 == list(range(len(costs)))
    assert owner0 == owner1
    assert all(owner0[k] == 0 for k in mine0) and all(owner0[k] == 1 for k in mine1)
