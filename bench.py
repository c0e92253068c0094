"""Benchmark of the CellSim3D timestep on B200 (node-steps/s).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl cs3d|reference]
                    [--workload packed100k|colony|ensemble256|het64|small8] [--cells C]

Default workload: the packed large system (100,000 non-dividing cells, FCC
packing at volume fraction 0.5, pressure 200, Gaussian node velocities
sigma 0.01, seed 123), the configuration the headline target is quoted on.
One "step" is one full timestep of the reference's loop
(src/GPUbounce.cu:1055-1338) over every cell.  Inputs are larger than L2
(positions + velocities of 18M nodes = 576 MB), so no L2 flush is needed.

--impl cs3d (default): the CUDA path through libcs3d.so.  Under torchrun
each rank steps its own replica (the single-system path does not shard;
ensembles shard by instance), timed with CUDA events, max over ranks.
--impl reference: the reference has no CPU implementation of the timestep;
its own CUDA kernels, compiled unmodified for sm_100a (oracle/ref.mk) and
driven through its step sequence, step the same workload on rank 0's GPU.
Without that build the FP64 oracle port steps a bounded sample on the host.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

NODE_BYTES = 48  # algorithmic bytes per node-step: float32 x and v, read and written once
# DRAM bytes (read + write) per node of one k_s1 launch: ncu's dram__bytes_read.sum
# and dram__bytes_write.sum of one launch on 30k packed cells (5.4M nodes: 387.5 MB
# + 213.7 MB), scaled by the nodes of the launch
S1_TRAFFIC_PER_NODE = 112.0
ENSEMBLES = ("ensemble256", "het64")
_WORKLOADS = {}


def _peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            pk = json.load(f)
        return float(pk["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index=0):
        self.idx = device_index
        self.proc = None
        self.lines = []   # (arrival time, line)
        self.t0 = self.t1 = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.idx), "--query-gpu=" + self.FIELDS,
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
            # the timed region starts once nvidia-smi is sampling
            t = time.perf_counter()
            while not self.lines and time.perf_counter() - t < 5.0 and self.proc.poll() is None:
                time.sleep(0.01)
        except Exception:
            self.proc = None
        self.t0 = time.perf_counter()
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append((time.perf_counter(), line.strip()))

    def __exit__(self, *a):
        self.t1 = time.perf_counter()
        if self.proc:
            # one more sample after the region (a short region may hold none)
            n = len(self.lines)
            t = time.perf_counter()
            while len(self.lines) == n and time.perf_counter() - t < 0.5 and self.proc.poll() is None:
                time.sleep(0.01)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        # samples taken during the timed region, plus the first one after it
        # (nvidia-smi reports the state at the sample time)
        inside = [ln for t, ln in self.lines if self.t0 is not None and self.t0 <= t <= self.t1]
        after = [ln for t, ln in self.lines if self.t1 is not None and t > self.t1][:1]
        for ln in inside + after:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for k, nm in enumerate(names):
                if parts[5 + k].lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


SCHEDULES = os.path.join(ROOT, "cellsim3d_b200", "schedules")


def schedule_path(args):
    """The skin schedule of the run: --skin-schedule FILE, or with "auto"
    the autotuner's schedule for the workload (cellsim3d_b200/schedules/,
    tuned on a B200) when one exists and no fixed --skin is given; "none"
    for the library's fixed skin."""
    s = args.skin_schedule
    if not s or s == "none":
        return None
    if s == "auto":
        p = os.path.join(SCHEDULES, args.workload + ".json")
        return p if args.skin is None and os.path.exists(p) else None
    return s


def apply_skin_schedule(ens, args):
    """The neighbour-list skin by population range (a schedule written by
    `bench.py --autotune`).  It changes the time only, not
    the results."""
    p = schedule_path(args)
    if p:
        from cellsim3d_b200 import autotune
        ens.set_skin_schedule(*autotune.load_schedule(p))


def skin_info(args):
    """The neighbour-list skin of the run, for the JSON line."""
    out = {"skin": args.skin if args.skin is not None else 0.1}
    p = schedule_path(args)
    if p:
        from cellsim3d_b200 import autotune
        mc, sk = autotune.load_schedule(p)
        out["schedule"] = {"min_cells": mc, "skins": sk, "file": os.path.relpath(p, ROOT)}
    return out


def run_autotune(args):
    """--autotune FILE: the skin autotuner (cellsim3d_b200/autotune.py) on
    this workload: `--steps` steps per candidate skin (`--tune-skins`) in
    cs3d_step calls of `--tune-chunk` steps, by population range for a
    single system, as one range for an ensemble.  Writes the schedule with
    its timing table to FILE (the format of cellsim3d_b200/schedules/)."""
    import cellsim3d_b200 as cs
    from cellsim3d_b200 import autotune
    insts = build_workload(args.workload, args.cells, steps=args.steps, instances=args.instances)
    topo = make_topology(insts)

    def make():
        ens = cs.Ensemble([p for p, _, _ in insts], topo, [cap for _, _, cap in insts])
        for k, (p, st, cap) in enumerate(insts):
            ens.load_state(k, st["X"], st["Y"], st["Z"], st.get("VX"), st.get("VY"), st.get("VZ"), n_cells=st["n"])
        return ens

    def total(ens):
        return sum(ens.n_cells(k) for k in range(len(insts)))

    skins = [float(x) for x in args.tune_skins.split(",")]
    bounds = (1,) if args.workload in ENSEMBLES else autotune.DEFAULT_BOUNDS
    res = autotune.tune(make, args.steps, skins=skins, bounds=bounds, chunk=args.tune_chunk, population=total)
    text = res.to_json()
    with open(args.autotune, "w") as f:
        f.write(text + "\n")
    return text


def dist_env():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def reduce_over_ranks(dist, device, maxes, sums):
    """The maximum of each of `maxes` and the sum of each of `sums` over all
    ranks (one all-reduce each, the same two calls on every rank); without a
    process group (`dist` None), the values themselves."""
    import torch
    mx = torch.tensor([float(v) for v in maxes], dtype=torch.float64, device=device)
    sm = torch.tensor([float(v) for v in sums], dtype=torch.float64, device=device)
    if dist is not None:
        dist.all_reduce(mx, op=dist.ReduceOp.MAX)
        dist.all_reduce(sm, op=dist.ReduceOp.SUM)
    return mx.tolist(), sm.tolist()


def _subset(insts, k):
    """A stratified subset by initial cell count: every (n / k)-th instance in size order."""
    if not k or k >= len(insts):
        return insts
    order = sorted(range(len(insts)), key=lambda q: (insts[q][1]["n"], q))
    pick = sorted({order[int(round(q * (len(insts) - 1) / max(k - 1, 1)))] for q in range(k)})
    return [insts[q] for q in pick]


def _config(gen):
    """The instances of an ensemble generator, generated once per process."""
    if gen.__name__ not in _WORKLOADS:
        _WORKLOADS[gen.__name__] = gen()
    return _WORKLOADS[gen.__name__]


def build_workload(name, cells, seed=123, steps=0, instances=0):
    key = (name, cells, seed, steps, instances)
    if key not in _WORKLOADS:
        _WORKLOADS[key] = _build_workload(name, cells, seed, steps, instances)
    return _WORKLOADS[key]


def workloads():
    """The seeded input generators (cellsim3d_b200/workloads.py, numpy only),
    loaded from their file without running the package's __init__, so that
    the reference arm builds its inputs without importing cellsim3d_b200 or
    mapping libcs3d.so.  Both arms step the same generated arrays."""
    mod = sys.modules.get("cs3d_workloads")
    if mod is None:
        import importlib.util
        spec = importlib.util.spec_from_file_location(
            "cs3d_workloads", os.path.join(ROOT, "cellsim3d_b200", "workloads.py"))
        mod = importlib.util.module_from_spec(spec)
        sys.modules["cs3d_workloads"] = mod
        spec.loader.exec_module(mod)
    return mod


def workload_config(name, insts):
    """The `config` object of both arms' JSON lines: the workload as generated
    (initial cells and nodes, instances), the same keys and values in both."""
    cells = int(sum(st["n"] for _, st, _ in insts))
    nodes = 180 * cells
    return {"workload": name, "cells": cells, "nodes": nodes, "instances": len(insts),
            "parallelism": "instances sharded" if name in ENSEMBLES else "replicas",
            "l2": "inputs larger than L2 (no flush)" if nodes * 24 > 126e6 else "L2 resident"}


PRECISION = ("FP32 state (positions, velocities, forces stored as float); every force term evaluated in "
             "FP64 from the float state and rounded to float once; FP64 centre of mass, volume and division "
             "test; float contact decisions with the reference's expressions")


def _build_workload(name, cells, seed, steps, instances):
    W = workloads()
    if name == "packed100k":
        c, vel, L = W.packed_fcc(cells, phi=0.5, seed=seed)
        p = W.base_params(box_len=(L, L, L), growth_rate=0.0, min_pressure=200.0, max_pressure=200.0,
                          div_time_steps=5000, rng_ij=seed, rng_kl=100 * seed)
        return [(p, W.state(c, velocities=vel), cells)]
    if name == "colony":
        p, st, cap = W.config2()
        return [(p, st, cap)]
    if name == "small8":
        # 8 cells on a 2x2x2 lattice, pressure ramp, all divide at step 1
        p, st, _ = W.config1()
        return [(p, st, 4096)]
    if name == "ensemble256":
        # capacity per instance: 10k steps grow the largest instance to ~4500 cells
        cap = 1024 if steps <= 500 else 6000
        return _subset([(p, st, cap) for p, st in _config(W.config4)], instances)
    if name == "het64":
        # 64 instances of 256..8192 cells at packing 0.4, own bond stiffness;
        # every cell divides at step 1, so the capacity is a multiple of N0
        grow = 4 if steps > 500 else 2
        return _subset([(p, st, grow * st["n"] + 64) for p, st in _config(W.config5)], instances)
    raise ValueError(name)


def make_topology(insts):
    import cellsim3d_b200 as cs
    W = workloads()
    st = insts[0][1]
    return cs.build_topology(cs.mesh_from_arrays(W.load_mesh()), st["X"][:192], st["Y"][:192], st["Z"][:192])


def run_cs3d(args, world, rank, local):
    import torch
    import cellsim3d_b200 as cs
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300), device_id=torch.device("cuda", local))
    insts = build_workload(args.workload, args.cells, steps=args.warmup + args.steps, instances=args.instances)
    n_total = len(insts)
    config = workload_config(args.workload, insts)
    if args.workload in ENSEMBLES and world > 1:
        # instances shard across ranks by predicted cost, no data-path collective
        from cellsim3d_b200 import shard
        mine = shard.partition([shard.predicted_cost(st, args.warmup + args.steps, p) for p, st, _ in insts],
                               world)[rank]
        insts = [insts[k] for k in mine]
    topo = make_topology(insts)
    ens = cs.Ensemble([p for p, _, _ in insts], topo, [cap for _, _, cap in insts], device=local)
    if args.skin is not None:
        ens.set_option(cs.OPT_SKIN, int(round(args.skin * 1e6)))
    apply_skin_schedule(ens, args)
    for k, (p, st, cap) in enumerate(insts):
        ens.load_state(k, st["X"], st["Y"], st["Z"], st.get("VX"), st.get("VY"), st.get("VZ"), n_cells=st["n"])
    n_nodes0 = sum(st["n"] for _, st, _ in insts) * 180
    ens.step(args.warmup)
    cells_before = sum(ens.n_cells(k) for k in range(len(insts)))
    # the state at the start of the timed region, on the host (pinned): the
    # end-to-end leg below restarts from it, so that both legs cover the same
    # steps of the run
    keys = ("X", "Y", "Z", "VX", "VY", "VZ")
    host0 = []
    if not args.no_e2e:
        for k in range(len(insts)):
            s = ens.state(k)
            host0.append((s["n"], {q: torch.from_numpy(s[q]).pin_memory().numpy() for q in keys},
                          s["pressure"].copy(), s["youngs"].copy()))
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        ens.step(args.steps)
    torch.cuda.synchronize()
    ms = ens.last_step_ms()
    cells_after = sum(ens.n_cells(k) for k in range(len(insts)))
    node_steps = 0.5 * (cells_before + cells_after) * 180 * args.steps
    stats = ens.stats()
    # per-kernel device times (profiling pass after the timed region)
    prof = ens.profile_step(3)
    # end to end through the C ABI with host buffers: upload the state, K
    # synchronous cs3d_step(1) calls (each returns the status word), read the
    # final state back
    e2e = None
    if not args.no_e2e:
        # every instance's state at the start of the timed region from pinned
        # host memory, K steps, every instance's state back into pinned
        # buffers with room for the capacity
        res = [{q: torch.empty(cap * 192, dtype=torch.float32).pin_memory().numpy() for q in keys}
               for _, _, cap in insts]
        host = host0
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for k, (n, h, pr, yg) in enumerate(host):
            ens.load_state(k, h["X"], h["Y"], h["Z"], h["VX"], h["VY"], h["VZ"], pressure=pr, youngs=yg, n_cells=n)
        t_load = time.perf_counter()
        for _ in range(args.steps):
            ens.step(1)
        t_steps = time.perf_counter()
        outs = [ens.state(k, out=res[k]) for k in range(len(insts))]
        t1 = time.perf_counter()
        n_in = sum(h[0] for h in host)
        n_out = sum(o["n"] for o in outs)
        # node-steps at the starting cell counts (divisions during the K steps not counted)
        # wall-clock split (rank 0's): the upload, the K calls (the first
        # one re-initialises: list build and initial forces), the read-back
        split_ms = {"load": 1e3 * (t_load - t0), "steps": 1e3 * (t_steps - t_load), "read": 1e3 * (t1 - t_steps)}
        e2e = {"seconds": t1 - t0, "node_steps": n_in * 180 * args.steps,
               "h2d": (6 * 4 * n_in * 192 + 8 * n_in) / args.steps,
               "d2h": (6 * 4 * n_out * 192 + 4 * len(insts)) / args.steps + 4 * len(insts)}
    # whole job: node-steps summed over ranks, times the slowest rank's; the
    # end-to-end leg the same way, its copies summed
    ee = e2e or {"seconds": 0.0, "node_steps": 0.0, "h2d": 0.0, "d2h": 0.0}
    (ms_max, e2e_s), (total_node_steps, e2e_ns, e2e_h2d, e2e_d2h) = reduce_over_ranks(
        dist, "cuda", [ms, ee["seconds"]], [node_steps, ee["node_steps"], ee["h2d"], ee["d2h"]])
    result = None
    if rank == 0:
        peak, peak_kind = _peaks()
        value = total_node_steps / (ms_max * 1e-3)
        top = max(prof, key=lambda kv: kv[1])
        n_nodes = 0.5 * (cells_before + cells_after) * 180
        s1 = dict(prof).get("s1_con_dis", top[1])
        achieved = NODE_BYTES * n_nodes / (s1 * 1e-3) / 1e9
        step_ms = sum(v for _, v in prof)
        result = {
            "metric": "node-steps/s (cells x 180 x steps / s)",
            "value": value,
            "unit": "node-steps/s",
            "n_gpus": world,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": ms_max / args.steps,
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f32",
            "data": "synthetic (seeded generator, cellsim3d_b200/workloads.py)",
            "config": config,
            "precision": PRECISION,
            "timed_cells": {"start": cells_before, "end": cells_after},
            "roofline": {"bound": "hbm", "kernel": "s1_con_dis", "achieved": achieved, "peak": peak,
                         "unit": "GB/s", "frac": achieved / peak,
                         "traffic": S1_TRAFFIC_PER_NODE * n_nodes if args.workload == "packed100k" else None,
                         "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of one k_s1 launch "
                                           "on 30k cells, scaled by nodes (profiles/k_s1_packed30k.md)",
                         "peak_source": peak_kind + " (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured"
                         else peak_kind,
                         "algorithmic_bytes_per_node": NODE_BYTES},
            "step_roofline": {"achieved": NODE_BYTES * value / 1e9 / world, "frac": NODE_BYTES * value / 1e9 / world / peak},
            "kernels_ms": {k: round(v, 4) for k, v in prof},
            "profiled_step_ms": step_ms,
            # every rank launches the same kernel sequence: the whole job's count
            "gpu_launches": int(stats["launches_per_step"]) * args.steps * world,
            "nl_rebuilds": stats["rebuilds"],
            "nl_rebuilds_div_rule": stats["rebuilds_div_rule"],
            "max_entries": stats["max_entries"],
            "max_cand": stats["max_cand"],
            "list_skin": skin_info(args),
            "clocks": clk.summary(),
        }
        if args.workload in ENSEMBLES:
            # whole simulations per hour: the timed steps stand for the run of
            # warmup + steps steps of every instance.  Every instance advances
            # one step per ensemble step, so each instance's step time is the
            # ensemble's step time (p50 = p99).
            secs = ms_max * 1e-3 * (args.warmup + args.steps) / args.steps
            result["ensemble"] = {"instances": n_total, "steps_per_sim": args.warmup + args.steps,
                                  "cells_start": cells_before, "cells_end": cells_after,
                                  "sims_per_hour": n_total * 3600.0 / secs,
                                  "instance_step_ms_p50": ms_max / args.steps,
                                  "instance_step_ms_p99": ms_max / args.steps}
        if e2e:
            result["e2e"] = {"value": e2e_ns / e2e_s,
                             "unit": "node-steps/s", "h2d_bytes_per_step": int(e2e_h2d),
                             "d2h_bytes_per_step": int(e2e_d2h),
                             "how": "cs3d_load_state of the timed region's starting state from pinned host, "
                                    "K x cs3d_step(1) with status read-back, cs3d_get_state to host",
                             "split_ms_rank0": {k: round(v, 3) for k, v in split_ms.items()}}
    ens.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return result


DECADES = ((1, 10), (10, 100), (100, 1000), (1000, 4096))


def colony_decades(events, n0, bounds, times_ms):
    """Node-steps and device time per population decade of a colony run.

    events: (step, parent, daughter) of the run; bounds: the steps at which
    the population first reached 10, 100, 1000 and 4096 cells (the end of a
    decade); times_ms: the device time up to each bound.  The cells stepped
    in step t are those present at its start: n0 plus the divisions of
    steps < t."""
    ev_steps = np.asarray([e[0] for e in events], dtype=np.int64)
    out = {}
    prev_s, prev_ms = 0, 0.0
    for (lo, hi), s, ms in zip(DECADES, bounds, times_ms):
        t = np.arange(prev_s + 1, s + 1)
        n_start = n0 + np.searchsorted(np.sort(ev_steps), t, side="left")
        node_steps = float(180 * n_start.sum())
        dt = (ms - prev_ms) * 1e-3
        out["%d-%d" % (lo, hi)] = {"steps": int(s - prev_s), "node_steps": node_steps, "seconds": dt,
                                   "node_steps_per_s": node_steps / dt if dt > 0 else None}
        prev_s, prev_ms = s, ms
    return out


def run_colony(args):
    """Config 2: one cell in a box of side 60 grown by division until 4096
    cells, timed in launches of a few steps (CUDA events); throughput per
    population decade.  A first pass of args.warmup steps (the step-1
    division included) captures the step graphs; the colony then starts
    again from one cell."""
    import torch
    import cellsim3d_b200 as cs
    torch.cuda.set_device(0)
    (p, st, cap), = build_workload("colony", args.cells)
    topo = make_topology([(p, st, cap)])
    sim = cs.Simulation(p, topo, cap)
    if args.skin is not None:
        sim.set_option(cs.OPT_SKIN, int(round(args.skin * 1e6)))
    apply_skin_schedule(sim, args)
    sim.load_state(st["X"], st["Y"], st["Z"], n_cells=st["n"])
    sim.step(max(args.warmup, 3))
    sim.load_state(st["X"], st["Y"], st["Z"], n_cells=st["n"])
    chunk, total, elapsed = 10, 0, 0.0
    bounds, times = [], []
    with ClockSampler(0) as clk:
        while total < args.colony_max_steps and len(bounds) < len(DECADES):
            sim.step(chunk)
            total += chunk
            elapsed += sim.last_step_ms()
            n = sim.n_cells()
            while len(bounds) < len(DECADES) and n >= DECADES[len(bounds)][1]:
                bounds.append(total)
                times.append(elapsed)
    events = sim.events()
    cells_end = sim.n_cells()
    sim.close()
    dec = colony_decades(events, st["n"], bounds, times)
    # every step of the run (a run that stops short of 4096 cells included)
    node_steps = colony_decades(events, st["n"], [total], [elapsed])["1-10"]["node_steps"]
    return {"metric": "node-steps/s (cells x 180 x steps / s)", "value": node_steps / (elapsed * 1e-3),
            "unit": "node-steps/s", "n_gpus": 1, "steps": total, "warmup": args.warmup,
            "ms_per_step": elapsed / total, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic (one cell, cellsim3d_b200/workloads.py config2)",
            "list_skin": skin_info(args),
            "config": {"workload": "colony", "cells_end": int(cells_end), "capacity": cap,
                       "timing": "launches of %d steps, CUDA events" % chunk},
            "decades": dec, "clocks": clk.summary()}


def cpu_baseline(args, steps=None, cells=None):
    """The FP64 oracle stepping a bounded sample of the workload on the host."""
    import oracle
    W = workloads()
    cells = cells or args.cpu_cells
    insts = build_workload(args.workload, cells)
    # ensembles: the instance of median initial size
    p, st, cap = sorted(insts, key=lambda t: t[1]["n"])[len(insts) // 2]
    mesh = W.load_mesh()
    r0, th = oracle.r0_theta0(st["X"][:192], st["Y"][:192], st["Z"][:192], mesh["nn"])
    topo = oracle.make_topo(mesh["nn"], mesh["sign"], r0, th, mesh["faces"])
    S = oracle.System(max(cap, st["n"]), p, topo)
    S.load(st["X"], st["Y"], st["Z"], st.get("VX"), st.get("VY"), st.get("VZ"), n=st["n"])
    S.seed(p["rng_ij"], p["rng_kl"])
    S.init()
    steps = steps or args.cpu_steps
    t0 = time.perf_counter()
    S.step(steps)
    dt = time.perf_counter() - t0
    ns = S.n * 180 * steps
    S.close()
    return {"value": ns / dt, "unit": "node-steps/s", "cores": os.cpu_count(), "kind": "port",
            "sample": "%d full timesteps of a %d-cell system of the same generator (FP64 oracle, OpenMP %d threads)"
                      % (steps, st["n"], os.cpu_count())}


def run_reference(args):
    """The reference arm.  The reference has no CPU implementation of the
    timestep: its own CUDA kernels, compiled unmodified for sm_100a from the
    reference sources (oracle/ref.mk) and driven through the reference's step
    sequence (oracle/ref_harness.cu), step the same workload on this GPU.
    Without that build, the FP64 oracle port steps a bounded sample on the
    host cores instead."""
    from oracle import ref
    if args.workload == "colony" and ref.available():
        return run_reference_colony(args)
    line = {"impl": "reference", "metric": "node-steps/s (cells x 180 x steps / s)", "unit": "node-steps/s",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "data": "synthetic (seeded generator, cellsim3d_b200/workloads.py)"}
    if not ref.available():
        base = cpu_baseline(args, steps=max(1, min(args.steps, args.cpu_steps)))
        line.update({"value": base["value"], "dtype": "f64", "config": {"workload": args.workload, "cells": args.cpu_cells},
                     "cpu_baseline": base,
                     "e2e": {"value": base["value"], "unit": "node-steps/s", "h2d_bytes_per_step": 0,
                             "d2h_bytes_per_step": 0}})
        return line
    from concurrent.futures import ThreadPoolExecutor
    insts = build_workload(args.workload, args.cells, steps=args.warmup + args.steps)
    config = workload_config(args.workload, insts)
    mesh = workloads().load_mesh()
    n_all = len(insts)
    insts = _subset(insts, args.ref_sample)
    total_ms, node_steps, cells0 = 0.0, 0.0, 0
    statuses, max_bin, max_nn, guard = set(), 0, 0, 0.0
    inst_ms = []

    def one(inst):
        p, st, cap = inst
        return st, ref.run(p, mesh, st, cap, args.warmup + args.steps, warmup=args.warmup)

    with ClockSampler(0) as clk:
        # one simulation after another (device time of each timed region)
        for st, r in map(one, insts):
            timed = r["steps"] - args.warmup
            if timed <= 0:
                raise RuntimeError("reference stopped in the warm-up: " + r["status_text"])
            total_ms += r["total_ms"] - r["guard_ms"]
            inst_ms.append((r["total_ms"] - r["guard_ms"]) / timed)
            # cell count grows by division: the trapezoid between the counts at
            # the start of the timed steps (after the warm-up's divisions) and
            # at the end, as the CUDA arm counts
            ev = np.asarray(r["events"]).reshape(-1, 3)
            n_t0 = st["n"] + int(np.count_nonzero(ev[:, 0] <= args.warmup))
            node_steps += 0.5 * (n_t0 + r["n"]) * 180 * timed
            cells0 += st["n"]
            statuses.add(r["status_text"])
            max_bin, max_nn = max(max_bin, r["max_bin"]), max(max_nn, r["max_local_nn"])
            guard += r["guard_ms"]
        conc = None
        if len(insts) > 1 and args.ref_concurrency > 1:
            # the same simulations as concurrent processes sharing the GPU
            # (wall time of the whole batch, process start-up included)
            t0 = time.perf_counter()
            with ThreadPoolExecutor(args.ref_concurrency) as ex:
                list(ex.map(one, insts))
            conc = time.perf_counter() - t0
    value = node_steps / (total_ms * 1e-3)
    extra = {}
    if args.workload in ENSEMBLES:
        # whole simulations per hour, the timed steps standing for the run of
        # warmup + steps steps (as the CUDA arm reports it)
        run_s = total_ms * 1e-3 * (args.warmup + args.steps) / args.steps
        extra = {"steps_per_sim": args.warmup + args.steps, "sims_per_hour_sequential": len(insts) * 3600.0 / run_s}
    if conc is not None:
        extra.update({"sequential_node_steps_per_s": value, "concurrent_node_steps_per_s": node_steps / conc,
                      "concurrent_processes": args.ref_concurrency,
                      "sims_per_hour_concurrent": len(insts) * 3600.0 / conc})
        value = max(value, node_steps / conc)
    if len(inst_ms) > 1:
        extra["instance_step_ms_p50"] = float(np.percentile(inst_ms, 50))
        extra["instance_step_ms_p99"] = float(np.percentile(inst_ms, 99))
    line.update({
        "value": value, "ms_per_step": total_ms / args.steps, "dtype": "f32",
        "config": config,
        "precision": "FP32 (the reference's kernels)",
        "instances_run": {"instances": len(insts), "cells": cells0, "of": n_all,
                          "how": ("a stratified sample, " if len(insts) < n_all else "") +
                                 ("one after another and %d at a time (best kept)" % args.ref_concurrency
                                  if conc is not None else "single system")},
        "ensemble": extra,
        "reference_build": {"kernels": "src/propagate.cu, centermass.cu, volume.cu, propagatebound.cu, "
                                       "PressureKernels.cu, postscriptinit.cu compiled unmodified for sm_100a "
                                       "(oracle/ref.mk)",
                            "driver": "oracle/ref_harness.cu: the step sequence of src/GPUbounce.cu:1055-1338",
                            "status": sorted(statuses), "max_bin_count": max_bin, "max_cells_per_node_filter": max_nn,
                            "guard_ms_excluded": guard},
        "cpu_baseline": {"value": value, "unit": "node-steps/s", "cores": 0, "kind": "reference",
                         "sample": "no CPU implementation exists: the reference's CUDA kernels on this GPU, "
                                   "%d timed steps after %d warm-up steps" % (args.steps, args.warmup)},
        "e2e": {"value": value, "unit": "node-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "clocks": clk.summary(),
    })
    return line


def run_reference_colony(args):
    """Config 2 through the reference's own kernels: the harness stops at 4096
    cells and reports the device time (its guard kernels excluded) at the first
    step of each population decade."""
    from oracle import ref
    (p, st, cap), = build_workload("colony", args.cells)
    mesh = workloads().load_mesh()
    with ClockSampler(0) as clk:
        r = ref.run(p, mesh, st, cap, args.colony_max_steps, decades=True)
    bounds = [m[0] for m in r["marks"]]
    times = [m[2] for m in r["marks"]]
    dec = colony_decades(r["events"], st["n"], bounds, times)
    node_steps = sum(v["node_steps"] for v in dec.values())
    secs = times[-1] * 1e-3 if times else float("nan")
    value = node_steps / secs
    return {"impl": "reference", "metric": "node-steps/s (cells x 180 x steps / s)", "value": value,
            "unit": "node-steps/s", "n_gpus": args.gpus, "steps": r["steps"], "warmup": 0,
            "ms_per_step": times[-1] / max(r["steps"], 1) if times else None, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (one cell, cellsim3d_b200/workloads.py config2)",
            "config": {"workload": "colony", "cells_end": int(r["n"]), "capacity": cap},
            "decades": dec,
            "reference_build": {"status": r["status_text"], "max_bin_count": r["max_bin"],
                                "max_cells_per_node_filter": r["max_local_nn"]},
            "cpu_baseline": {"value": value, "unit": "node-steps/s", "cores": 0, "kind": "reference",
                             "sample": "no CPU implementation exists: the reference's CUDA kernels on this GPU"},
            "e2e": {"value": value, "unit": "node-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "clocks": clk.summary()}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="cs3d", choices=["cs3d", "reference"])
    ap.add_argument("--workload", default="packed100k", choices=["packed100k", "colony", "ensemble256", "het64", "small8"])
    ap.add_argument("--cells", type=int, default=100_000)
    ap.add_argument("--cpu-cells", type=int, default=10_000)
    ap.add_argument("--cpu-steps", type=int, default=10)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--skin", type=float, default=None,
                    help="neighbour-list skin (default: the library's, 0.1)")
    ap.add_argument("--autotune", default=None, metavar="FILE",
                    help="tune the list skin on this workload (--steps steps per candidate) and write the schedule")
    ap.add_argument("--tune-skins", default="0.05,0.07,0.1,0.13")
    ap.add_argument("--tune-chunk", type=int, default=50)
    ap.add_argument("--skin-schedule", default="auto",
                    help="skin by population range: a file written by --autotune, "
                         "'auto' (the tuned schedule of the workload in cellsim3d_b200/schedules/) or 'none'")
    ap.add_argument("--colony-max-steps", type=int, default=40000,
                    help="colony: stop after this many steps if 4096 cells are not reached")
    ap.add_argument("--instances", type=int, default=0,
                    help="ensembles: a stratified subset of this many instances (0: all)")
    ap.add_argument("--ref-sample", type=int, default=0,
                    help="reference arm, ensembles: run a stratified sample of this many instances (0: all)")
    ap.add_argument("--ref-concurrency", type=int, default=8,
                    help="reference arm, ensembles: also run the simulations this many at a time")
    args = ap.parse_args()
    world, rank, local = dist_env()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        if rank != 0:
            return
        print(json.dumps(run_reference(args)))
        return
    if args.autotune:
        if rank == 0:
            print(run_autotune(args))
        return
    if args.workload == "colony":
        if rank == 0:
            print(json.dumps(run_colony(args)))
        return
    res = run_cs3d(args, world, rank, local)
    if rank == 0:
        if not args.no_cpu and world == 1:
            res["cpu_baseline"] = cpu_baseline(args)
        print(json.dumps(res))


if __name__ == "__main__":
    main()
