"""CUDA path (through the C ABI) against the FP64 oracle on identical inputs:
forces of the initial evaluation and after steps within the 1e-5 parity bar,
contact-pair sets exactly equal, division events exactly equal, grid and box
decisions exactly equal."""
import numpy as np
import pytest

import cellsim3d_b200 as cs
from cellsim3d_b200 import workloads as W

from parity import TOL, force_errors, make_pair, rel_err, sorted_pairs

pytestmark = pytest.mark.gpu


def _report(tag, ec, ed):
    print("%-28s Fc max %.2e glob %.2e p99 %.2e | Fd max %.2e glob %.2e p99 %.2e"
          % ((tag,) + ec + ed))


def _check_forces(tag, sim, orc):
    ec, ed = force_errors(sim, orc)
    _report(tag, ec, ed)
    assert ec[1] < TOL and ed[1] < TOL, (tag, ec, ed)
    assert ec[0] < TOL and ed[0] < TOL, (tag, ec, ed)


def _check_pairs(sim, orc):
    for kind in (0, 1):
        g = sorted_pairs(sim.pairs(kind))
        r = sorted_pairs(orc.recorded_pairs(kind))
        assert g.shape == r.shape and np.array_equal(g, r), ("pair set differs", kind, g.shape, r.shape)


def _check_grid(sim, orc):
    mm, dv = sim.grid()
    assert np.array_equal(mm.view(np.uint32), orc.minmax.view(np.uint32))
    assert tuple(dv) == orc.divs
    cells = sim.cells()
    n = orc.n
    assert np.array_equal(cells["aabb"].view(np.uint32), orc.aabb[:n].view(np.uint32))
    cm = orc.CM[:, :n].T
    assert np.array_equal(cells["cm"].view(np.uint32), cm.view(np.uint32))


def test_config1_initial_forces(mesh):
    p, st, _ = W.config1()
    sim, orc = make_pair(p, st, mesh, capacity=64)
    _check_grid(sim, orc)
    _check_pairs(sim, orc)
    _check_forces("config1 init", sim, orc)


def test_config1_division_at_step1(mesh):
    p, st, _ = W.config1()
    sim, orc = make_pair(p, st, mesh, capacity=64)
    sim.step(1)
    orc.step(1)
    assert sim.n_cells() == orc.n == 16
    assert np.array_equal(sim.events(), orc.events())
    _check_pairs(sim, orc)
    _check_forces("config1 step1", sim, orc)
    s = sim.state()
    n = orc.n
    ex = rel_err([s["X"], s["Y"], s["Z"]], [orc.X, orc.Y, orc.Z], n)
    ev = rel_err([s["VX"], s["VY"], s["VZ"]], [orc.VX, orc.VY, orc.VZ], n)
    print("config1 step1 X", ex, "V", ev)
    assert ex[0] < TOL and ev[1] < TOL
    _check_grid(sim, orc)


@pytest.mark.parametrize("nsteps", [5, 50])
def test_config1_steps(mesh, nsteps):
    p, st, _ = W.config1()
    sim, orc = make_pair(p, st, mesh, capacity=64)
    sim.step(nsteps)
    orc.step(nsteps)
    assert sim.n_cells() == orc.n
    assert np.array_equal(sim.events(), orc.events())
    _check_pairs(sim, orc)
    _check_forces("config1 %d steps" % nsteps, sim, orc)
    s = sim.state()
    ev = rel_err([s["VX"], s["VY"], s["VZ"]], [orc.VX, orc.VY, orc.VZ], orc.n)
    print("config1 %d steps V" % nsteps, ev)
    assert ev[1] < 1e-4


@pytest.mark.parametrize("n_cells", [64, 500])
def test_packed_initial_and_steps(mesh, n_cells):
    c, vel, L = W.packed_fcc(n_cells, phi=0.5, seed=11)
    p = W.base_params(box_len=(L, L, L), growth_rate=0.0, min_pressure=200.0, max_pressure=200.0,
                      div_time_steps=5000)
    st = W.state(c, velocities=vel)
    sim, orc = make_pair(p, st, mesh, capacity=n_cells)
    assert orc.err() == 0
    _check_grid(sim, orc)
    _check_pairs(sim, orc)
    _check_forces("packed %d init" % n_cells, sim, orc)
    for k in (1, 9):
        sim.step(k)
        orc.step(k)
        _check_pairs(sim, orc)
        _check_forces("packed %d +%d" % (n_cells, k), sim, orc)
    assert sim.last_error() == 0


def test_ensemble_instances_match_oracle(mesh):
    import oracle
    from parity import topo_for
    insts = []
    for k, (n, gr) in enumerate([(3, 0.002), (1, 0.004), (8, 0.001)]):
        c = W.random_centres(n, 12.0, W.SplitMix(100 + k))
        p = W.base_params(box_len=(12.0, 12.0, 12.0), growth_rate=gr, division_vol=2.9 - 0.1 * k,
                          rng_ij=k, rng_kl=100 * k)
        insts.append((p, W.state(c)))
    topo, otopo = topo_for(insts[0][1], mesh)
    ens = cs.Ensemble([p for p, _ in insts], topo, [32, 32, 32])
    orcs = []
    for k, (p, st) in enumerate(insts):
        ens.load_state(k, st["X"], st["Y"], st["Z"], n_cells=st["n"])
        o = oracle.System(32, p, otopo)
        o.load(st["X"], st["Y"], st["Z"], n=st["n"])
        o.seed(p["rng_ij"], p["rng_kl"])
        o.init()
        orcs.append(o)
    ens.step(30)
    for k, o in enumerate(orcs):
        o.step(30)
        assert ens.n_cells(k) == o.n
        assert np.array_equal(ens.events(k), o.events())
        f = ens.forces(k)
        ec = rel_err([f["FCX"], f["FCY"], f["FCZ"]], [o.FC[0], o.FC[1], o.FC[2]], o.n)
        print("ensemble inst", k, "n", o.n, "Fc", ec)
        assert ec[1] < TOL


def test_nan_input_raises_error_bit(mesh):
    p, st, _ = W.config1()
    st = dict(st)
    st["X"] = st["X"].copy()
    st["X"][5] = np.nan
    from parity import topo_for
    topo, _ = topo_for(W.config1()[1], mesh)
    sim = cs.Simulation(p, topo, 64)
    sim.load_state(st["X"], st["Y"], st["Z"], n_cells=st["n"])
    rc = sim.step(1, raise_on_error=False)
    assert rc != 0
    assert sim.last_error() & 0x1


def test_capacity_overflow_reports(mesh):
    p, st, _ = W.config1()
    from parity import topo_for
    topo, _ = topo_for(st, mesh)
    sim = cs.Simulation(p, topo, 12)
    sim.load_state(st["X"], st["Y"], st["Z"], n_cells=st["n"])
    rc = sim.step(1, raise_on_error=False)
    assert rc == -69
    assert sim.n_cells() == 12
