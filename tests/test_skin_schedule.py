"""The skin schedule (cs3d_set_skin_schedule) changes the time, not the
results: runs with a schedule that switches the skin several times as the
population grows are bit-identical to a run at a fixed skin (positions,
velocities, forces, pressures and division events), for a growing colony and
for an ensemble of uneven instances.  Argument checks of the entry point."""
import numpy as np
import pytest

import cellsim3d_b200 as cs
from cellsim3d_b200 import _lib
from cellsim3d_b200 import workloads as W

from parity import topo_for

pytestmark = pytest.mark.gpu

KEYS = ("X", "Y", "Z", "VX", "VY", "VZ", "pressure", "youngs")


def _colony(mesh, schedule, steps):
    p, st, cap = W.config2(capacity=256)
    topo, _ = topo_for(st, mesh)
    sim = cs.Simulation(p, topo, cap)
    sim.load_state(st["X"], st["Y"], st["Z"], n_cells=st["n"])
    if schedule:
        sim.set_skin_schedule(*schedule)
    for k in range(0, steps, 250):
        sim.step(min(250, steps - k))
    out = sim.state()
    out["F"] = sim.forces()
    out["events"] = sim.events()
    out["rebuilds"] = sim.stats()["rebuilds"]
    sim.close()
    return out


def _same(a, b):
    for k in KEYS:
        assert np.array_equal(np.asarray(a[k]).view(np.uint32), np.asarray(b[k]).view(np.uint32)), k
    for k in a["F"]:
        assert np.array_equal(np.asarray(a["F"][k]).view(np.uint32), np.asarray(b["F"][k]).view(np.uint32)), k


def test_colony_with_a_skin_schedule_is_bit_identical(mesh):
    """One cell grown for 2500 steps (to ~16 cells); the schedule switches the
    skin at 2, 4 and 8 cells."""
    fixed = _colony(mesh, None, 2500)
    sched = _colony(mesh, ([2, 4, 8], [0.05, 0.13, 0.07]), 2500)
    assert fixed["n"] >= 8
    assert fixed["n"] == sched["n"]
    assert np.array_equal(fixed["events"], sched["events"])
    _same(fixed, sched)
    # the schedule was in force: other skins rebuild at other steps (with
    # the same skin throughout, the identical trajectories would rebuild at
    # the same steps)
    assert sched["rebuilds"] != fixed["rebuilds"]


def test_ensemble_with_a_skin_schedule_is_bit_identical(mesh):
    """Three instances of 1, 8 and 40 initial cells: each switches by its own
    cell count."""
    insts = []
    for k, n0 in enumerate((1, 8, 40)):
        sm = W.SplitMix(11 + k)
        c = W.random_centres(n0, 30.0, sm)
        ij, kl = W.seed_pair(k)
        p = W.base_params(box_len=(30.0, 30.0, 30.0), growth_rate=0.003, div_time_steps=10 ** 9,
                          rng_ij=ij, rng_kl=kl)
        insts.append((p, W.state(c), 4 * n0 + 64))
    topo, _ = topo_for(insts[0][1], mesh)

    def run(schedule):
        ens = cs.Ensemble([p for p, _, _ in insts], topo, [cap for _, _, cap in insts])
        for k, (p, st, cap) in enumerate(insts):
            ens.load_state(k, st["X"], st["Y"], st["Z"], st.get("VX"), st.get("VY"), st.get("VZ"), n_cells=st["n"])
        if schedule:
            ens.set_skin_schedule(*schedule)
        ens.step(300)
        ens.step(300)
        out = [ens.state(k) for k in range(len(insts))]
        ev = [ens.events(k) for k in range(len(insts))]
        ens.close()
        return out, ev

    a, ea = run(None)
    b, eb = run(([1, 16, 64], [0.06, 0.12, 0.08]))
    for k in range(len(insts)):
        assert a[k]["n"] == b[k]["n"]
        assert np.array_equal(ea[k], eb[k])
        for q in KEYS:
            assert np.array_equal(np.asarray(a[k][q]).view(np.uint32), np.asarray(b[k][q]).view(np.uint32)), (k, q)


def test_schedule_arguments_are_checked(mesh):
    p, st, cap = W.config2(capacity=64)
    topo, _ = topo_for(st, mesh)
    sim = cs.Simulation(p, topo, cap)
    bad = [([4, 2], [0.1, 0.1]), ([0, 2], [0.1, 0.1]), ([1], [0.0]), ([1], [2.0]),
           (list(range(1, 10)), [0.1] * 9)]
    for mc, sk in bad:
        with pytest.raises(_lib.CS3DError):
            sim.set_skin_schedule(mc, sk)
    sim.set_skin_schedule([1, 5], [0.08, 0.12])
    sim.set_skin_schedule()   # clears
    sim.close()
