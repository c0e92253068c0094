"""Variable bond stiffness (stiffnessParams) and the internal-cells mitotic
count.

CPU: the host's initial soft-cell selection (src/GPUbounce.cu:616-692)
against the oracle's restatement, the inp.json mapping, and the oracle's
schedule (pressure rule src/PressureKernels.cu:4-40, growth-end softening
src/GPUbounce.cu:1340-1429) against plain-Python restatements of the same
rules.  GPU: the CUDA path against the oracle, step by step."""
import json

import numpy as np
import pytest

import cellsim3d_b200 as cs
import oracle
from cellsim3d_b200 import _lib
from cellsim3d_b200 import workloads as W

from parity import make_pair, single_step_check


def _lattice(n_side=3, spacing=2.3, seed=5):
    rng = np.random.default_rng(seed)
    c = np.array([[2 + spacing * i, 2 + spacing * j, 2 + spacing * k]
                  for i in range(n_side) for j in range(n_side) for k in range(n_side)], dtype=np.float32)
    c += rng.uniform(-0.05, 0.05, c.shape).astype(np.float32)
    return W.state(c)


def _config(**kw):
    c = _lib.Config()
    c.youngs_mod = 1000.0
    c.stiff_factor1 = 1.0
    c.soft_stiff_factor = 0.8
    c.use_different_stiffnesses = 1
    c.use_rigid_box = 1
    for k, v in kw.items():
        setattr(c, k, v)
    return c


def _oracle_params(c):
    return W.soft_params(W.base_params(), soft_factor=c.soft_stiff_factor,
                         number_of_softer_cells=c.number_of_softer_cells,
                         fraction_of_softer_cells=c.fraction_of_softer_cells,
                         closeness_to_center=c.closeness_to_center)


@pytest.mark.parametrize("kw", [dict(closeness_to_center=0.5), dict(closeness_to_center=0.8),
                                dict(number_of_softer_cells=5), dict(fraction_of_softer_cells=0.3),
                                dict(number_of_softer_cells=6, use_rigid_box=0),
                                dict(fraction_of_softer_cells=0.45, use_rigid_box=0)])
def test_initial_stiffness_matches_oracle(kw):
    st = _lattice()
    n = st["n"]
    cfg = _config(**kw)
    r_lib = cs.Ranmar(42, 4200)
    E = cs.initial_stiffness(cfg, st["X"], st["Y"], st["Z"], n, r_lib)
    r_orc = oracle.Ranmar(42, 4200)
    E_o = oracle.initial_stiffness(_oracle_params(cfg), cfg.use_rigid_box, st["X"], st["Y"], st["Z"], n, r_orc.st)
    s1, s2 = np.float32(1000.0), np.float32(0.8) * np.float32(1000.0)
    assert np.array_equal(E.view(np.uint32), E_o.view(np.uint32))
    assert set(np.unique(E)) <= {s1, s2}
    soft = int((E == s2).sum())
    assert 0 < soft < n
    if cfg.use_rigid_box and cfg.closeness_to_center == 0:
        k = cfg.number_of_softer_cells or int(round(cfg.fraction_of_softer_cells * n))
        assert list(np.nonzero(E == s2)[0]) == list(range(k))
    # both streams advanced by the same draws
    assert np.array_equal(r_lib.draw(3), r_orc.draw(3))


def test_initial_stiffness_too_many_cells():
    st = _lattice()
    cfg = _config(number_of_softer_cells=28)
    with pytest.raises(cs.CS3DError):
        cs.initial_stiffness(cfg, st["X"], st["Y"], st["Z"], st["n"], cs.Ranmar(1, 100))
    assert oracle.initial_stiffness(_oracle_params(cfg), 1, st["X"], st["Y"], st["Z"], st["n"]) is None


def test_initial_stiffness_off_is_stiffness1():
    st = _lattice()
    cfg = _config(use_different_stiffnesses=0, number_of_softer_cells=5)
    E = cs.initial_stiffness(cfg, st["X"], st["Y"], st["Z"], st["n"])
    assert np.all(E == np.float32(1000.0))


def test_inp_json_stiffness_round_trip(tmp_path):
    p = W.soft_params(W.base_params(div_time_steps=4), phase_count=3, soften_after_growth=1,
                      number_of_softer_cells=5, fraction_of_softer_cells=0.25, choose_random_cell_indices=1,
                      closeness_to_center=0.3, count_internal_radius=0.6)
    with open(tmp_path / "inp.json", "w") as f:
        json.dump(W.inp_json(p, 64, 4, 2), f)
    q = cs.config_to_params(cs.read_json_params(str(tmp_path / "inp.json")))
    assert q.use_different_stiffnesses == 1 and q.soften_after_growth == 1 and q.phase_count == 3
    assert np.float32(q.stiffness2) == np.float32(p["stiffness2"])
    assert q.number_of_softer_cells == 5 and q.choose_random_cell_indices == 1
    assert np.float32(q.fraction_of_softer_cells) == np.float32(0.25)
    assert np.float32(q.closeness_to_center) == np.float32(0.3)
    assert np.float32(q.count_internal_radius) == np.float32(0.6)
    # duringGrowth on: no growth-end softening
    d = W.inp_json(dict(p, soften_after_growth=0), 64, 4, 2)
    with open(tmp_path / "inp2.json", "w") as f:
        json.dump(d, f)
    assert cs.config_to_params(cs.read_json_params(str(tmp_path / "inp2.json"))).soften_after_growth == 0


def test_recalc_r0_is_refused(tmp_path):
    p = W.soft_params(W.base_params())
    d = W.inp_json(p, 64, 4, 2)
    d["stiffnessParams"]["recalc_r0"] = True
    with open(tmp_path / "inp.json", "w") as f:
        json.dump(d, f)
    with pytest.raises(cs.CS3DError):
        cs.config_to_params(cs.read_json_params(str(tmp_path / "inp.json")))


# ---------------------------------------------------------------- oracle semantics
def _schedule_params(**over):
    p = W.soft_params(W.base_params(div_time_steps=2), phase_count=3, soften_after_growth=1,
                      number_of_softer_cells=5)
    p.update(over)
    return p


def _oracle_run(p, st, steps, youngs=None):
    mesh = W.load_mesh()
    r0, th = oracle.r0_theta0(st["X"][:192], st["Y"][:192], st["Z"][:192], mesh["nn"])
    topo = oracle.make_topo(mesh["nn"], mesh["sign"], r0, th, mesh["faces"])
    O = oracle.System(64, p, topo)
    O.load(st["X"], st["Y"], st["Z"], youngs=youngs, n=st["n"])
    O.seed(p["rng_ij"], p["rng_kl"])
    O.init()
    return O


def test_oracle_pressure_rule_and_random_softening():
    """From step phase_count on soft cells have pressure 0; at the end of
    step div_time_steps + 2, distinct RANMAR picks round(u * n) are softened."""
    _, st, _ = W.config1()
    p = _schedule_params(choose_random_cell_indices=1)
    E0 = np.full(8, np.float32(p["stiffness1"]))
    E0[[1, 6]] = np.float32(p["stiffness2"])
    O = _oracle_run(p, st, 0, youngs=E0)
    O.step(3)   # step 1 divides every cell (daughters inherit), steps 2-3
    n = O.n
    soft = O.E[:n] != np.float32(p["stiffness1"])
    assert soft.sum() == 4                                  # cells 1, 6 and their daughters
    assert np.all(O.press[:n][soft] == 0.0)                 # step 3 >= phase_count
    assert np.all(O.press[:n][~soft] > 0.0)
    # replay the growth-end picks from the RANMAR state before step 4
    r = oracle.Ranmar(1, 1)
    r.st = oracle.OrcRanmar.from_buffer_copy(bytes(lib_rng(O)))
    chosen = []
    while len(chosen) < 5:
        ind = int(np.floor(float(np.float32(r.draw(1)[0]) * np.float32(n)) + 0.5))   # roundf
        if ind not in chosen:
            chosen.append(ind)
    expect = soft.copy()
    for ind in chosen:
        if ind < n:
            expect[ind] = True
    O.step(1)   # step 4 = div_time_steps + 2
    assert np.array_equal(O.E[:n] != np.float32(p["stiffness1"]), expect)


def lib_rng(O):
    import ctypes as C
    return C.string_at(oracle.lib().orc_rng(O.h), C.sizeof(oracle.OrcRanmar))


def test_oracle_central_softening_uses_stale_centre():
    """The closeness path measures the largest distance from the previous
    system centre ((1, 1, 1) before any CoM correction) and the candidates
    from the new one, in cell order, up to the count."""
    _, st, _ = W.config1()
    p = _schedule_params(closeness_to_center=0.4, number_of_softer_cells=3)
    O = _oracle_run(p, st, 0)
    O.step(3)
    n = O.n
    O.step(1)
    f32 = np.float32
    # the centres of mass of step 4 are the ones the softening reads
    cm4 = O.CM[:, :n].T.astype(np.float32)
    r2max = max(f32(f32(f32(v[0] * v[0]) + f32(v[1] * v[1])) + f32(v[2] * v[2])) for v in cm4 - np.ones(3, f32))
    s = np.zeros(3, f32)
    for v in cm4:
        s = (s + v).astype(f32)
    s = (s / f32(n)).astype(f32)
    f = f32(f32(1.0) - f32(0.4))
    thr = f32(f32(f * f) * r2max)
    expect, got = [], 0
    for c in range(n):
        v = cm4[c] - s
        r2 = f32(f32(f32(v[0] * v[0]) + f32(v[1] * v[1])) + f32(v[2] * v[2]))
        if got < 3 and r2 <= thr:
            expect.append(c)
            got += 1
    assert list(np.nonzero(O.E[:n] != f32(p["stiffness1"]))[0]) == expect
    assert np.array_equal(O.syscm, s)


# ---------------------------------------------------------------- CUDA path
def _soft_pair(p, st, mesh, youngs):
    st = dict(st, youngs=youngs)
    return make_pair(p, st, mesh, 64)


@pytest.mark.gpu
@pytest.mark.parametrize("path", ["random", "central"])
def test_stiffness_schedule_single_steps(mesh, path):
    """Steps 1-6 of 8 dividing cells with two soft cells: the division
    (daughters inherit), the pressure rule from phase_count = 3 and the
    growth-end softening at step 4, each as one step from the identical state
    (positions, stiffness and pressure exact, forces within the bar)."""
    _, st, _ = W.config1()
    over = dict(choose_random_cell_indices=1) if path == "random" else dict(closeness_to_center=0.4,
                                                                             number_of_softer_cells=3)
    p = _schedule_params(**over)
    E0 = np.full(8, np.float32(p["stiffness1"]))
    E0[[1, 6]] = np.float32(p["stiffness2"])
    sim, orc = _soft_pair(p, st, mesh, E0)
    for k in range(6):
        single_step_check(sim, "stiffness %s step %d" % (path, k + 1))
    s = sim.state()
    n = s["n"]
    assert int((s["youngs"][:n] != np.float32(p["stiffness1"])).sum()) > 4   # softened at step 4
    sim.close()
    orc.close()


@pytest.mark.gpu
def test_stiffness_schedule_multi_step_matches_oracle(mesh):
    """The same schedule in one 12-step launch (graphs, the softening step
    outside them) against the tracking oracle: stiffness, pressure and
    division events exact."""
    _, st, _ = W.config1()
    p = _schedule_params(choose_random_cell_indices=1, number_of_softer_cells=6)
    E0 = np.full(8, np.float32(p["stiffness1"]))
    E0[3] = np.float32(p["stiffness2"])
    sim, orc = _soft_pair(p, st, mesh, E0)
    sim.step(12)
    orc.step(12)
    s = sim.state()
    n = s["n"]
    assert n == orc.n
    assert np.array_equal(sim.events(), orc.events())
    assert np.array_equal(s["youngs"][:n], orc.E[:n])
    assert np.array_equal(s["pressure"][:n].view(np.uint32), orc.press[:n].view(np.uint32))
    sim.close()
    orc.close()


@pytest.mark.gpu
def test_far_counts_match_oracle(mesh):
    """count_only_internal_cells: after the step-1 divisions of 56 cells
    (112 >= 50 cells), num_cells_far's count against the oracle's, and the
    events of the following steps."""
    # a cluster in the middle of a large box: the daughters' centres of mass
    # (still 0) lie far from the system centre
    box = 60.0
    c = W.rsa_centres(56, 14.0, np.random.default_rng(11)) + np.float32(23.0)
    p = W.base_params(box_len=(box, box, box), div_time_steps=10 ** 9, count_internal_radius=0.6,
                      rng_ij=11, rng_kl=1100)
    st = W.state(c)
    sim, orc = make_pair(p, st, mesh, 160, record_pairs=False)
    sim.step(3)
    orc.step(3)
    assert sim.n_cells() == orc.n
    assert np.array_equal(sim.events(), orc.events())
    fg, fo = sim.far_counts(), orc.far_counts()
    print("far counts", fg, fo)
    assert np.array_equal(fg, fo)
    assert len(fo) >= 1 and fo[0, 0] == 1 and fo[0, 1] == 56
    sim.close()
    orc.close()
