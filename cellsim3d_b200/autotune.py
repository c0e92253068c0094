"""Neighbour-list skin autotuner by population range.

The list skin (the margin of the list radius over the attraction range, and
with it the edge of the node-hash bins) trades the length of the contact
lists that every step sweeps against the frequency of list rebuilds.  The
best value depends on how fast the nodes move and how densely the cells
pack, and both change as a colony grows.  The skin changes no result: the
contact-pair sets and the order of every force sum are the same for any
skin.  So the tuner steps the SAME trajectory once per candidate skin, times
each chunk of steps on the device (CUDA events, Simulation.last_step_ms),
credits the chunk to the population range it started in, and keeps per range
the fastest skin.  It checks on the way that the runs do pass through the
same populations at the same steps.

    sched = tune(make_sim, steps=4000)          # e.g. a colony from one cell
    sim.set_skin_schedule(*sched.schedule())    # applied per instance by the device

`python bench.py --workload colony --steps 28000 --autotune FILE` tunes a
benchmark workload and writes the schedule with its timing table.

The device applies a schedule to each instance of an ensemble by the
instance's own cell count.  An ensemble's step times cannot be split by
instance, so an ensemble is tuned as one range (bounds=(1,)): one skin for
all its instances, picked on its own trajectory.
"""
import json

from . import OPT_SKIN

DEFAULT_SKINS = (0.05, 0.07, 0.1, 0.13)
DEFAULT_BOUNDS = (1, 10, 100, 1000, 10000, 100000)


def range_of(n, bounds):
    """Index of the population range of n cells: the last bound <= n
    (0 below the first)."""
    r = 0
    for q, b in enumerate(bounds):
        if n >= b:
            r = q
    return r


class Result:
    """Device time per (population range, skin) of a tuning run."""

    def __init__(self, bounds, skins):
        self.bounds = tuple(int(b) for b in bounds)
        self.skins = tuple(float(s) for s in skins)
        self.ms = {}      # (range, skin) -> summed device ms
        self.steps = {}   # (range, skin) -> steps timed
        self.failed = {}  # skin -> {step, range, status} of its failure (e.g. list capacity)

    def add(self, r, skin, ms, steps):
        self.ms[(r, skin)] = self.ms.get((r, skin), 0.0) + ms
        self.steps[(r, skin)] = self.steps.get((r, skin), 0) + steps

    def best(self):
        """{range: fastest skin} over the ranges timed (every run covers the
        same steps of a range, the runs being the same trajectory)."""
        out = {}
        for r in sorted({r for r, _ in self.ms}):
            cand = []
            for s in self.skins:
                if (r, s) not in self.ms:
                    continue
                cand.append((self.ms[(r, s)], s))
            if cand:
                out[r] = min(cand)[1]
        return out

    def schedule(self):
        """(min_cells, skins) for set_skin_schedule: one entry per range
        whose best skin differs from the previous range's."""
        mc, sk = [], []
        for r, s in sorted(self.best().items()):
            if sk and sk[-1] == s:
                continue
            mc.append(max(1, self.bounds[r]))
            sk.append(s)
        return mc, sk

    def to_json(self):
        mc, sk = self.schedule()
        table = {}
        for (r, s), ms in sorted(self.ms.items()):
            table.setdefault(str(self.bounds[r]), {})[repr(s)] = {
                "ms": round(ms, 4), "steps": self.steps[(r, s)],
                "ms_per_step": round(ms / max(self.steps[(r, s)], 1), 5)}
        return json.dumps({"min_cells": mc, "skins": sk, "bounds": list(self.bounds),
                           "candidates": list(self.skins), "failed": {repr(k): v for k, v in self.failed.items()},
                           "table": table}, indent=1)


def tune(make, steps, skins=DEFAULT_SKINS, bounds=DEFAULT_BOUNDS, chunk=10, population=None):
    """Run `steps` steps of the system that make() returns (a fresh,
    loaded Simulation), once per candidate skin, in cs3d_step calls of
    `chunk` steps.  population(sim) gives the cell count (default
    sim.n_cells()).  Returns a Result.  Raises if two runs disagree on the
    population at the start of a chunk (the runs must be the same
    trajectory)."""
    if population is None:
        def population(sim):
            return sim.n_cells()
    res = Result(bounds, skins)
    ref_pop = None
    for s in res.skins:
        sim = make()
        try:
            sim.set_option(OPT_SKIN, int(round(s * 1e6)))
            pops = []
            k = 0
            while k < steps:
                m = min(chunk, steps - k)
                n = population(sim)
                pops.append(n)
                if ref_pop is not None and len(ref_pop) >= len(pops) and ref_pop[len(pops) - 1] != n:
                    raise RuntimeError("skin %g: %d cells at step %d, the first run had %d"
                                       % (s, n, k, ref_pop[len(pops) - 1]))
                st = sim.step(m, raise_on_error=False)
                if st != 0:
                    # e.g. a list over its capacity: out from this range on
                    res.failed[s] = {"step": k, "range": range_of(n, res.bounds), "status": int(st)}
                    break
                res.add(range_of(n, res.bounds), s, sim.last_step_ms(), m)
                k += m
            if ref_pop is None or len(pops) > len(ref_pop):
                ref_pop = pops
        finally:
            sim.close()
    # a skin that failed part-way is kept only for the ranges before the one it failed in
    for s, f in res.failed.items():
        for key in [key for key in res.ms if key[1] == s and key[0] >= f["range"]]:
            del res.ms[key]
            del res.steps[key]
    return res


def load_schedule(path):
    """(min_cells, skins) from a file written by Result.to_json()."""
    with open(path) as f:
        d = json.load(f)
    return list(d["min_cells"]), [float(x) for x in d["skins"]]
