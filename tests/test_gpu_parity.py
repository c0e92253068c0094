"""CUDA path (through the C ABI) against the FP64 oracle.

Single steps from identical float states: conservative/dissipative forces and
velocities within the 1e-5 relative bar, positions (drift and division
geometry), centres of mass, grids, boxes, contact-pair sets and division
events bit-exact.  Over longer runs the division events of the CUDA path and
of an independently stepped oracle must agree."""
import numpy as np
import pytest

import cellsim3d_b200 as cs
import oracle
from cellsim3d_b200 import workloads as W

from parity import (TOL, force_errors, make_pair, oracle_from, rel_err, single_step_check, sorted_pairs,
                    topo_for)

pytestmark = pytest.mark.gpu


def _check_init(tag, sim, orc):
    mm, dv = sim.grid()
    assert np.array_equal(mm.view(np.uint32), orc.minmax.view(np.uint32)), tag
    assert tuple(dv) == orc.divs, tag
    cells = sim.cells()
    n = orc.n
    assert np.array_equal(cells["aabb"].view(np.uint32), orc.aabb[:n].view(np.uint32)), tag
    assert np.array_equal(cells["cm"].view(np.uint32), orc.CM[:, :n].T.copy().view(np.uint32)), tag
    for kind in (0, 1):
        g = sorted_pairs(sim.pairs(kind))
        r = sorted_pairs(orc.recorded_pairs(kind))
        assert g.shape == r.shape and np.array_equal(g, r), (tag, "pair set", kind)
    ec, ed = force_errors(sim, orc)
    print("%-26s Fc max %.2e glob %.2e | Fd max %.2e glob %.2e" % (tag, ec[0], ec[1], ed[0], ed[1]))
    assert ec[0] < TOL and ec[1] < TOL and ed[0] < TOL and ed[1] < TOL, (tag, ec, ed)


def test_config1_initial_forces(mesh):
    p, st, _ = W.config1()
    sim, orc = make_pair(p, st, mesh, capacity=64)
    _check_init("config1 init", sim, orc)


def test_config1_single_steps(mesh):
    p, st, _ = W.config1()
    sim, orc = make_pair(p, st, mesh, capacity=256)
    r = single_step_check(sim, "config1 step 1")
    assert r["n"] == 16                      # all eight cells divide at step 1
    for target in (2, 3, 10, 40, 120):
        cur = sim.stats()["steps"]
        if target - 1 > cur:
            sim.step(target - 1 - cur)
        single_step_check(sim, "config1 step %d" % target)


def test_config1_division_events_2000_steps(mesh):
    """Division events (step, parent, daughter) of the CUDA path and of the
    independently stepped oracle over the first 2000 steps."""
    p, st, _ = W.config1()
    sim, orc = make_pair(p, st, mesh, capacity=1024, record_pairs=False)
    for chunk in range(20):
        sim.step(100)
        orc.step(100)
        assert sim.n_cells() == orc.n, (chunk, sim.n_cells(), orc.n)
    eg, eo = sim.events(), orc.events()
    print("config1 2000 steps: %d cells, %d division events" % (sim.n_cells(), len(eg)))
    assert np.array_equal(eg, eo)
    assert sim.last_error() == 0


@pytest.mark.parametrize("n_cells", [64, 500])
def test_packed_single_steps(mesh, n_cells):
    c, vel, L = W.packed_fcc(n_cells, phi=0.5, seed=11)
    p = W.base_params(box_len=(L, L, L), growth_rate=0.0, min_pressure=200.0, max_pressure=200.0,
                      div_time_steps=5000)
    st = W.state(c, velocities=vel)
    sim, orc = make_pair(p, st, mesh, capacity=n_cells)
    assert orc.err() == 0
    _check_init("packed %d init" % n_cells, sim, orc)
    for target in (1, 2, 10, 30):
        cur = sim.stats()["steps"]
        if target - 1 > cur:
            sim.step(target - 1 - cur)
        single_step_check(sim, "packed %d step %d" % (n_cells, target))
    assert sim.last_error() == 0


def test_colony_growth_single_steps(mesh):
    """One cell in a box of side 60 growing by division: checks across the
    first divisions (every 400 steps a single-step comparison)."""
    p, st, cap = W.config2(capacity=256)
    sim, orc = make_pair(p, st, mesh, capacity=cap)
    single_step_check(sim, "colony step 1")
    for k in range(6):
        sim.step(399)
        single_step_check(sim, "colony step %d" % sim.stats()["steps"])


def _ensemble_check(mesh, insts, cap, steps):
    """Instances of one ensemble against one oracle each: initial forces,
    `steps` steps (cell counts and division events exact), then one step of
    every instance from the ensemble's own state (positions bit-exact, forces
    and velocities within the bar)."""
    topo, otopo = topo_for(insts[0][1], mesh)
    ens = cs.Ensemble([p for p, _ in insts], topo, [cap] * len(insts))
    orcs = []
    for k, (p, st) in enumerate(insts):
        ens.load_state(k, st["X"], st["Y"], st["Z"], n_cells=st["n"])
        o = oracle.System(cap, p, otopo)
        o.load(st["X"], st["Y"], st["Z"], n=st["n"])
        o.seed(p["rng_ij"], p["rng_kl"])
        o.init()
        orcs.append(o)
    for k, o in enumerate(orcs):
        f = ens.forces(k)
        ec = rel_err([f["FCX"], f["FCY"], f["FCZ"]], [o.FC[0], o.FC[1], o.FC[2]], o.n)
        assert ec[0] < TOL, (k, ec)
    ens.step(steps)
    for k, o in enumerate(orcs):
        o.step(steps)
        assert ens.n_cells(k) == o.n
        assert np.array_equal(ens.events(k), o.events())
    # single step of every instance from the ensemble's own state
    snaps = []
    for k in range(len(insts)):
        s = ens.state(k)
        s.update(ens.forces(k))
        s.update(ens.random_force(k))
        s["cm"] = ens.cells(k)["cm"]
        s["rng"] = ens.get_rng(k)
        s["step"] = steps
        snaps.append(s)
    Os = [oracle_from(snaps[k], insts[k][0], otopo, cap, record=False) for k in range(len(insts))]
    ens.step(1)
    for k, O in enumerate(Os):
        O.step(1)
        n = ens.n_cells(k)
        assert n == O.n
        s = ens.state(k)
        f = ens.forces(k)
        assert np.array_equal(s["X"][: n * 192].view(np.uint32), O.X[: n * 192].view(np.uint32))
        ec = rel_err([f["FCX"], f["FCY"], f["FCZ"]], [O.FC[0], O.FC[1], O.FC[2]], n)
        ev = rel_err([s["VX"], s["VY"], s["VZ"]], [O.VX, O.VY, O.VZ], n)
        print("ensemble inst %d n %d Fc %s V %s" % (k, n, ec, ev))
        assert ec[0] < TOL and ev[0] < TOL
    for o in orcs + Os:
        o.close()
    ens.close()


def test_ensemble_instances_single_step(mesh):
    """Instances in the manner of the 256-instance ensemble: own cell counts,
    growth rates, division volumes and seeds."""
    insts = []
    for k, (n, gr) in enumerate([(3, 0.002), (1, 0.004), (8, 0.001)]):
        c = W.random_centres(n, 12.0, W.SplitMix(100 + k))
        p = W.base_params(box_len=(12.0, 12.0, 12.0), growth_rate=gr, division_vol=2.9 - 0.1 * k,
                          rng_ij=k, rng_kl=100 * k)
        insts.append((p, W.state(c)))
    _ensemble_check(mesh, insts, 32, 30)


def test_ensemble_packed_stiffness_instances(mesh):
    """Instances in the manner of the 64-instance heterogeneous ensemble:
    packing 0.4, own bond stiffness (stiffFactor1 = k/1000, contact stays at
    Young's modulus), own boxes, seeds above 300 folded into RANMAR's range;
    every cell divides at step 1."""
    insts = []
    for k, (n, stiff, seed) in enumerate([(12, 500.0, 1000), (20, 1250.0, 1031), (30, 2000.0, 1063)]):
        box = (n * (4.0 / 3.0) * np.pi / 0.4) ** (1.0 / 3.0) + 2.1
        c = W.rsa_centres(n, box, np.random.default_rng([7, k]))
        ij, kl = W.seed_pair(seed)
        p = W.base_params(box_len=(box, box, box), stiffness1=stiff, div_time_steps=10 ** 9, rng_ij=ij, rng_kl=kl)
        insts.append((p, W.state(c)))
    _ensemble_check(mesh, insts, 96, 40)


def test_nan_input_raises_error_bit(mesh):
    p, st, _ = W.config1()
    topo, _ = topo_for(st, mesh)
    X = st["X"].copy()
    X[5] = np.nan
    sim = cs.Simulation(p, topo, 64)
    sim.load_state(X, st["Y"], st["Z"], n_cells=st["n"])
    rc = sim.step(1, raise_on_error=False)
    assert rc != 0
    assert sim.last_error() & 0x1


def test_capacity_overflow_reports(mesh):
    p, st, _ = W.config1()
    topo, _ = topo_for(st, mesh)
    sim = cs.Simulation(p, topo, 12)
    sim.load_state(st["X"], st["Y"], st["Z"], n_cells=st["n"])
    rc = sim.step(1, raise_on_error=False)
    assert rc == -69
    assert sim.n_cells() == 12


def _multi_step_cases():
    c, vel, L = W.packed_fcc(64, phi=0.5, seed=5)
    packed = W.base_params(box_len=(L, L, L), growth_rate=0.0, min_pressure=200.0, max_pressure=200.0,
                           div_time_steps=5000)
    p1, st1, _ = W.config1()
    colony = [(W.base_params(box_len=(12.0, 12.0, 12.0), growth_rate=gr, division_vol=2.9 - 0.1 * k,
                             rng_ij=k, rng_kl=100 * k), W.state(W.random_centres(n, 12.0, W.SplitMix(100 + k))))
              for k, (n, gr) in enumerate([(3, 0.002), (1, 0.004), (8, 0.001)])]
    return {
        "packed": ([(packed, W.state(c, velocities=vel))], 64, 25),
        # every cell divides at step 1, more divisions follow
        "dividing": ([(p1, st1)], 64, 60),
        "dividing_langevin": ([(dict(p1, add_rands=1, rand_scale_factor=0.5, rand_seed=9), st1)], 64, 60),
        "ensemble": (colony, 32, 40),
    }


@pytest.mark.parametrize("case", ["packed", "dividing", "dividing_langevin", "ensemble"])
def test_multi_step_launch_equals_single_steps(mesh, case):
    """cs3d_step(n) fuses the first half kick and drift of each step into the
    previous step's S2 (on division steps: into S2 for the cells that do not
    divide, and into a kernel after the division for the two cells of each
    division); n single-step calls do not.  The two must give bit-identical
    states, forces, division events and list rebuilds (same float operations)."""
    insts, cap, steps = _multi_step_cases()[case]
    topo, _ = topo_for(insts[0][1], mesh)
    runs = []
    for mode in ("fused", "single"):
        ens = cs.Ensemble([p for p, _ in insts], topo, [cap] * len(insts))
        for k, (p, st) in enumerate(insts):
            ens.load_state(k, st["X"], st["Y"], st["Z"], st.get("VX"), st.get("VY"), st.get("VZ"), n_cells=st["n"])
        if mode == "fused":
            ens.step(steps)
        else:
            for _ in range(steps):
                ens.step(1)
        runs.append(ens)
    for k in range(len(insts)):
        a, b = runs[0].state(k), runs[1].state(k)
        assert a["n"] == b["n"]
        for key in ("X", "Y", "Z", "VX", "VY", "VZ", "pressure", "youngs"):
            assert np.array_equal(a[key].view(np.uint32), b[key].view(np.uint32)), (k, key)
        fa, fb = runs[0].forces(k), runs[1].forces(k)
        for key in fa:
            assert np.array_equal(fa[key].view(np.uint32), fb[key].view(np.uint32)), (k, key)
        assert np.array_equal(runs[0].events(k), runs[1].events(k))
    assert runs[0].stats()["rebuilds"] == runs[1].stats()["rebuilds"]
    if case != "packed":
        assert any(len(runs[0].events(k)) for k in range(len(insts)))
    for ens in runs:
        ens.close()


def test_correct_com_single_steps(mesh):
    """correct_com: all nodes shifted by minus the mean centre of mass after
    every step (and at set-up), the step's grid and centres of mass left
    unshifted, as in the reference."""
    c, vel, L = W.packed_fcc(64, phi=0.5, seed=13)
    c = c + np.float32(3.0)   # off-centre, so the correction moves the nodes
    p = W.base_params(box_len=(L + 6, L + 6, L + 6), growth_rate=0.0, min_pressure=200.0, max_pressure=200.0,
                      div_time_steps=5000, correct_com=1)
    st = W.state(c, velocities=vel)
    sim, orc = make_pair(p, st, mesh, capacity=64)
    _check_init("correct_com init", sim, orc)
    for target in (1, 2, 5):
        cur = sim.stats()["steps"]
        if target - 1 > cur:
            sim.step(target - 1 - cur)
        single_step_check(sim, "correct_com step %d" % target)
    s = sim.state()
    assert abs(float(np.mean(s["X"].reshape(-1, 192)[:, :180]))) < 0.5
    sim.close()
    orc.close()


def test_empty_instance_and_empty_system(mesh):
    """An ensemble instance with no cells steps along with nothing to do and
    leaves the others unchanged (their cell counts and division events equal
    the oracle's); a single simulation with no cells steps, too."""
    insts = []
    for k, (n, gr) in enumerate([(3, 0.002), (8, 0.001)]):
        c = W.random_centres(n, 12.0, W.SplitMix(200 + k))
        p = W.base_params(box_len=(12.0, 12.0, 12.0), growth_rate=gr, rng_ij=k + 5, rng_kl=100 * (k + 5))
        insts.append((p, W.state(c)))
    topo, otopo = topo_for(insts[0][1], mesh)
    empty = np.zeros(0, np.float32)
    params = [insts[0][0], W.base_params(box_len=(12.0, 12.0, 12.0)), insts[1][0]]
    ens = cs.Ensemble(params, topo, [32, 32, 32])
    ens.load_state(0, insts[0][1]["X"], insts[0][1]["Y"], insts[0][1]["Z"], n_cells=insts[0][1]["n"])
    ens.load_state(1, empty, empty, empty, n_cells=0)
    ens.load_state(2, insts[1][1]["X"], insts[1][1]["Y"], insts[1][1]["Z"], n_cells=insts[1][1]["n"])
    ens.step(30)
    assert ens.n_cells(1) == 0 and len(ens.events(1)) == 0
    for k in range(3):
        assert ens.last_error(k) == 0, k
    assert ens.state(1)["n"] == 0
    for k, (p, st) in zip((0, 2), insts):
        o = oracle.System(32, p, otopo)
        o.load(st["X"], st["Y"], st["Z"], n=st["n"])
        o.seed(p["rng_ij"], p["rng_kl"])
        o.init()
        o.step(30)
        assert ens.n_cells(k) == o.n
        assert np.array_equal(ens.events(k), o.events())
        o.close()
    ens.close()
    sim = cs.Simulation(insts[0][0], topo, 8)
    sim.load_state(empty, empty, empty, n_cells=0)
    sim.step(5)
    assert sim.n_cells() == 0 and sim.last_error() == 0
    sim.close()
