"""bench.py's accounting, on the CPU: node-steps and time per population
decade of a colony run, from its division events; and the whole-job figures
under several ranks (slowest rank's time, work summed), with two gloo ranks."""
import json
import os
import sys

import numpy as np
import pytest

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


_REF_INPUTS = r'''
import os, sys, tempfile
sys.path.insert(0, sys.argv[1])
import bench
from oracle import ref
insts = bench.build_workload("small8", 100000, steps=8)
cfg = bench.workload_config("small8", insts)
mesh = bench.workloads().load_mesh()
p, st, cap = insts[0]
with tempfile.TemporaryDirectory() as d:
    ref._write_input(os.path.join(d, "in.bin"), ref.pack_params(p), ref.pack_mesh(mesh), st, cap, 3, 0, 0)
    assert os.path.getsize(os.path.join(d, "in.bin")) > 0
if ref.available():
    r0, th = ref.tables(p, mesh, st)
    assert r0.shape == (576,) and th.shape == (576,)
assert not any(m == "cellsim3d_b200" or m.startswith("cellsim3d_b200.") for m in sys.modules), "package imported"
maps = open("/proc/self/maps").read()
assert "libcs3d" not in maps, "libcs3d.so mapped"
print("CFG", sorted(cfg.items()))
'''


def test_reference_arm_inputs_do_not_load_the_library():
    """The reference arm builds its inputs (workload arrays, parameter struct,
    mesh tables, the reference's own R0/theta0) without importing
    cellsim3d_b200 or mapping libcs3d.so."""
    import subprocess
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    p = subprocess.run([sys.executable, "-c", _REF_INPUTS, root], capture_output=True, text=True, timeout=300)
    assert p.returncode == 0, p.stderr[-3000:]
    assert "CFG" in p.stdout


def test_both_arms_print_the_same_config():
    """Both arms take `config` from workload_config of the same generated
    workload, before any sharding or sampling."""
    for name in ("small8", "packed100k"):
        a = bench.workload_config(name, bench.build_workload(name, 2000, steps=10))
        b = bench.workload_config(name, bench.build_workload(name, 2000, steps=10))
        assert a == b
        assert set(a) == {"workload", "cells", "nodes", "instances", "parallelism", "l2"}


def test_reference_arm_counts_node_steps_from_the_cells_after_the_warmup(monkeypatch):
    """The reference arm's node-steps start from the cells present after the
    warm-up (initial cells plus the warm-up's divisions), as the CUDA arm's
    do, and its sims/hr cover warmup + steps steps.  The harness run is
    stubbed: 8 initial cells, all dividing at step 1 of a 3-step warm-up,
    then 2 more divisions; 10 timed steps of 1 ms each."""
    from oracle import ref
    monkeypatch.setattr(ref, "available", lambda: True)

    def fake_run(p, mesh, st, cap, steps, warmup=0, **kw):
        ev = [(1, c, 8 + c) for c in range(st["n"])] + [(6, 0, 2 * st["n"]), (9, 1, 2 * st["n"] + 1)]
        return {"steps": steps, "n": 2 * st["n"] + 2, "total_ms": 10.0, "guard_ms": 0.0, "events": np.array(ev),
                "status_text": "ok", "max_bin": 1, "max_local_nn": 1}
    monkeypatch.setattr(ref, "run", fake_run)
    monkeypatch.setattr(bench.workloads(), "load_mesh", lambda: None)
    args = bench.argparse.Namespace(workload="small8", cells=8, warmup=3, steps=10, ref_sample=0,
                                    ref_concurrency=1, gpus=1, cpu_cells=8, cpu_steps=1)
    monkeypatch.setattr(bench, "build_workload",
                        lambda *a, **k: [({}, {"n": 8}, 64)])
    line = bench.run_reference(args)
    # 16 cells after the warm-up, 18 at the end: 17 on average over 10 steps in 10 ms
    assert line["value"] == pytest.approx(17 * 180 * 10 / 10e-3)
    args.workload = "het64"
    line = bench.run_reference(args)
    assert line["ensemble"]["sims_per_hour_sequential"] == pytest.approx(3600.0 / (10e-3 * 13 / 10))


def test_skin_schedule_selection(tmp_path):
    """--skin-schedule: 'none', and 'auto' (the default) without a tuned
    file or with a fixed --skin, give no schedule; 'auto' picks the
    workload's tuned file; a path is taken as given.  The default packed
    workload has no tuned file (its pick did not carry over between
    windows)."""
    ns = bench.argparse.Namespace
    assert bench.schedule_path(ns(skin_schedule="none", skin=None, workload="packed100k")) is None
    assert bench.schedule_path(ns(skin_schedule="auto", skin=None, workload="no_such_workload")) is None
    assert bench.schedule_path(ns(skin_schedule="auto", skin=None, workload="packed100k")) is None
    tuned = os.path.join(bench.SCHEDULES, "colony.json")
    assert bench.schedule_path(ns(skin_schedule="auto", skin=None, workload="colony")) == tuned
    assert bench.schedule_path(ns(skin_schedule="auto", skin=0.08, workload="colony")) is None
    p = str(tmp_path / "s.json")
    assert bench.schedule_path(ns(skin_schedule=p, skin=None, workload="colony")) == p
    from cellsim3d_b200 import autotune
    mc, sk = autotune.load_schedule(tuned)
    assert mc and len(mc) == len(sk) and all(0.002 < s <= 1.0 for s in sk)
    info = bench.skin_info(ns(skin_schedule="auto", skin=None, workload="colony"))
    assert info["schedule"]["min_cells"] == mc and info["schedule"]["file"] == "cellsim3d_b200/schedules/colony.json"


def test_autotune_mode_writes_a_schedule(monkeypatch, tmp_path):
    """bench.py --autotune: one range for an ensemble, a schedule file in the
    format of cellsim3d_b200/schedules/ (stand-in ensemble, no GPU)."""
    import cellsim3d_b200 as cs
    from cellsim3d_b200 import autotune

    class FakeEns:
        def __init__(self, params, topo, caps):
            self.n, self.skin, self.last = [2] * len(params), None, 0.0

        def load_state(self, *a, **k):
            pass

        def set_option(self, opt, v):
            self.skin = v * 1e-6

        def n_cells(self, k):
            return self.n[k]

        def step(self, m, raise_on_error=True):
            self.last = m * (1.0 + abs(self.skin - 0.07))
            return 0

        def last_step_ms(self):
            return self.last

        def close(self):
            pass

    monkeypatch.setattr(cs, "Ensemble", FakeEns)
    monkeypatch.setattr(bench, "make_topology", lambda insts: None)
    st = {"X": None, "Y": None, "Z": None, "n": 2}
    monkeypatch.setattr(bench, "build_workload", lambda *a, **k: [({}, st, 8), ({}, st, 8)])
    out = str(tmp_path / "ens.json")
    args = bench.argparse.Namespace(workload="ensemble256", cells=0, steps=100, instances=0, autotune=out,
                                    tune_skins="0.05,0.07,0.1", tune_chunk=25)
    text = bench.run_autotune(args)
    assert autotune.load_schedule(out) == ([1], [0.07])
    assert json.loads(text)["bounds"] == [1]
