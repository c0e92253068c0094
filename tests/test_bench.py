"""bench.py's accounting, on the CPU: node-steps and time per population
decade of a colony run, from its division events; and the whole-job figures
under several ranks (slowest rank's time, work summed), with two gloo ranks."""
import os
import sys

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
import bench  # noqa: E402


def test_colony_decades_counts_cells_at_the_start_of_each_step():
    # one cell; divisions at steps 5 (-> 2 cells) and 8 (-> 3 cells)
    d = bench.colony_decades([(5, 0, 1), (8, 0, 2)], 1, [10], [2.0])["1-10"]
    assert d["steps"] == 10
    assert d["node_steps"] == 180 * (5 * 1 + 3 * 2 + 2 * 3)
    assert np.isclose(d["node_steps_per_s"], d["node_steps"] / 0.002)


def test_colony_decades_split_at_the_bounds():
    # doubling every 10 steps from one cell: 2, 4, 8, 16 cells after steps 10, 20, 30, 40
    ev, n, k = [], 1, 0
    for s in (10, 20, 30, 40):
        for _ in range(n):
            ev.append((s, 0, n + len(ev)))
        n *= 2
    d = bench.colony_decades(ev, 1, [40, 45], [4.0, 5.0])
    first, second = d["1-10"], d["10-100"]
    assert first["steps"] == 40 and second["steps"] == 5
    assert first["node_steps"] == 180 * 10 * (1 + 2 + 4 + 8)
    assert second["node_steps"] == 180 * 5 * 16
    assert np.isclose(second["seconds"], 1e-3)


def _reduce_rank(rank, world, port, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        # rank r: device time 10 + r ms, 100 * (r + 1) node-steps, an end-to-end time of 2 - r s
        q.put((rank, bench.reduce_over_ranks(dist, "cpu", [10.0 + rank, 2.0 - rank],
                                             [100.0 * (rank + 1), 7.0])))
    finally:
        dist.destroy_process_group()


def test_whole_job_figures_are_max_time_and_summed_work_over_two_gloo_ranks():
    import socket
    import torch.multiprocessing as mp
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_reduce_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in range(2))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for _, (mx, sm) in res:
        assert mx == [11.0, 2.0]
        assert sm == [300.0, 14.0]


def test_single_process_figures_pass_through():
    assert bench.reduce_over_ranks(None, "cpu", [3.5, 0.0], [1e12, 2.0]) == ([3.5, 0.0], [1e12, 2.0])
