"""bench.py's accounting, on the CPU: node-steps and time per population
decade of a colony run, from its division events."""
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
