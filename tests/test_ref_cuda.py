"""The CUDA path against the reference's own CUDA kernels (compiled unmodified
from the reference sources into oracle/_ref/cs3d_ref by oracle/ref.mk and
driven through the reference's timestep by oracle/ref_harness.cu), on
identical inputs.

The reference computes in FP32, so its forces differ from exact arithmetic
by up to ~1e-5 (per node, relative); the CUDA path is FP64-accurate.  The bar
here: the CUDA path is no farther from the reference than the FP64 oracle is
(within 5%, or 1e-5, whichever is larger), and the division events of the
first 2000 steps of the 8-cell configuration are identical."""
import numpy as np
import pytest

import cellsim3d_b200 as cs
from cellsim3d_b200 import workloads as W
from oracle import ref

from parity import TOL, make_pair, rel_err, topo_for

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not ref.available(), reason="oracle/_ref/cs3d_ref not built (make -f oracle/ref.mk)")]

KEYS = ("FCX", "FCY", "FCZ", "FDX", "FDY", "FDZ")


def _errs(got, r, n):
    ec = rel_err([got[k] for k in KEYS[:3]], [r[k] for k in KEYS[:3]], n)
    ed = rel_err([got[k] for k in KEYS[3:]], [r[k] for k in KEYS[3:]], n)
    return ec, ed


def _packed(n_cells):
    c, vel, L = W.packed_fcc(n_cells, phi=0.5, seed=11)
    p = W.base_params(box_len=(L, L, L), growth_rate=0.0, min_pressure=200.0, max_pressure=200.0,
                      div_time_steps=5000)
    return p, W.state(c, velocities=vel), n_cells


CASES = {"config1": lambda: (lambda p, st, _: (p, st, 64))(*W.config1()),
         "packed64": lambda: _packed(64),
         "packed500": lambda: _packed(500)}


@pytest.mark.parametrize("case", sorted(CASES))
def test_initial_forces_against_reference_kernels(mesh, case):
    p, st, cap = CASES[case]()
    topo, _ = topo_for(st, mesh)
    sim, orc = make_pair(p, st, mesh, capacity=cap, record_pairs=False)
    got = sim.forces()
    exact = dict(zip(KEYS, [orc.FC[0], orc.FC[1], orc.FC[2], orc.FD[0], orc.FD[1], orc.FD[2]]))
    r = ref.run(p, mesh, st, cap, 0, dump_init=True)
    assert r["status"] == 0, r["status_text"]
    n = st["n"]
    (c_max, c_glob, _), (d_max, d_glob, _) = _errs(got, r["init"], n)
    (oc_max, oc_glob, _), (od_max, od_glob, _) = _errs(exact, r["init"], n)
    print("%-10s vs reference kernels: Fc max %.2e glob %.2e (FP64 oracle: %.2e %.2e) | "
          "Fd max %.2e glob %.2e (FP64 oracle: %.2e %.2e)"
          % (case, c_max, c_glob, oc_max, oc_glob, d_max, d_glob, od_max, od_glob))
    for got_e, ora_e in ((c_max, oc_max), (c_glob, oc_glob), (d_max, od_max), (d_glob, od_glob)):
        assert got_e <= max(TOL, 1.05 * ora_e), (case, got_e, ora_e)
    sim.close()
    orc.close()


def test_division_events_against_reference_kernels(mesh):
    """8 cells, pressure ramp, division on: the (step, parent, daughter)
    events of the first 2000 steps."""
    p, st, _ = W.config1()
    topo, _ = topo_for(st, mesh)
    r = ref.run(p, mesh, st, 1024, 2000)
    assert r["status"] == 0, r["status_text"]
    sim = cs.Simulation(p, topo, 1024)
    sim.load_state(st["X"], st["Y"], st["Z"], n_cells=st["n"])
    sim.step(2000)
    ev = np.asarray(sim.events())
    print("2000 steps: reference %d cells / %d events, CUDA path %d cells / %d events"
          % (r["n"], len(r["events"]), sim.n_cells(), len(ev)))
    assert sim.n_cells() == r["n"]
    assert np.array_equal(ev.reshape(-1, 3), r["events"])
    sim.close()


def test_first_step_velocities_against_reference_kernels(mesh):
    """Velocities and forces after one full step (8 cells, all dividing)."""
    p, st, _ = W.config1()
    topo, _ = topo_for(st, mesh)
    r = ref.run(p, mesh, st, 64, 1)
    assert r["status"] == 0, r["status_text"]
    sim = cs.Simulation(p, topo, 64)
    sim.load_state(st["X"], st["Y"], st["Z"], n_cells=st["n"])
    sim.step(1)
    n = sim.n_cells()
    assert n == r["n"] == 16
    s = sim.state()
    ev = rel_err([s["VX"], s["VY"], s["VZ"]], [r["VX"], r["VY"], r["VZ"]], n)
    dx = max(float(np.max(np.abs(s[k][: n * 192] - r[k]))) for k in ("X", "Y", "Z"))
    print("step 1: velocity max %.2e glob %.2e, position max |dx| %.2e" % (ev[0], ev[1], dx))
    assert ev[1] < TOL
    assert dx < 1e-5
    sim.close()


def _soft_config1(**over):
    p, st, _ = W.config1()
    p = W.soft_params(dict(p, div_time_steps=2), phase_count=3, soften_after_growth=1, number_of_softer_cells=5)
    p.update(over)
    E0 = np.full(8, np.float32(p["stiffness1"]))
    E0[[1, 6]] = np.float32(p["stiffness2"])
    return p, dict(st, youngs=E0)


@pytest.mark.parametrize("path", ["random", "central"])
def test_stiffness_schedule_against_reference_kernels(mesh, path):
    """Variable stiffness driven by the reference's own PressureUpdate and
    volumes kernels and its host softening code: 12 steps of 8 dividing cells
    (2 soft), softening at the end of step 4.  Stiffness, pressure and
    division events exact; positions within FP32 noise."""
    over = dict(choose_random_cell_indices=1) if path == "random" else dict(closeness_to_center=0.4,
                                                                             number_of_softer_cells=3)
    p, st = _soft_config1(**over)
    topo, _ = topo_for(st, mesh)
    r = ref.run(p, mesh, st, 64, 12)
    assert r["status"] == 0, r["status_text"]
    sim = cs.Simulation(p, topo, 64)
    sim.load_state(st["X"], st["Y"], st["Z"], youngs=st["youngs"], n_cells=st["n"])
    sim.step(12)
    s = sim.state()
    n = s["n"]
    assert n == r["n"]
    assert np.array_equal(np.asarray(sim.events()).reshape(-1, 3), r["events"])
    assert np.array_equal(s["youngs"][:n], r["youngs"])
    assert np.array_equal(s["pressure"][:n].view(np.uint32), r["pressure"].view(np.uint32))
    assert int((r["youngs"] != np.float32(p["stiffness1"])).sum()) > 4
    dx = max(float(np.max(np.abs(s[k][: n * 192] - r[k]))) for k in ("X", "Y", "Z"))
    print("stiffness %s: %d soft of %d, position max |dx| %.2e" % (path, int((r["youngs"] != p["stiffness1"]).sum()),
                                                                 n, dx))
    assert dx < 1e-4
    sim.close()


def test_correct_com_against_reference_kernels(mesh):
    """CoM correction by the reference's CorrectCoMMotion kernel and host
    calc_sys_CM, at set-up and after every step (8 cells dividing at step 1).
    No rigid box: the correction centres the system on the origin, outside a
    box that starts there.  The node positions agree to FP32 noise after one
    step and after 20, and the CUDA path is no farther from the reference
    than the FP64 oracle is."""
    p, st, _ = W.config1()
    p = dict(p, correct_com=1, use_rigid_box=0)
    topo, _ = topo_for(st, mesh)

    def dist(a, b, n):
        # the 180 nodes of every cell: the padding slots carry no state (with the
        # correction the reference's follow its stale XP copies)
        return max(float(np.max(np.abs(a[k][: n * 192].reshape(n, 192)[:, :180] -
                                       b[k][: n * 192].reshape(n, 192)[:, :180]))) for k in ("X", "Y", "Z"))

    for steps in (1, 20):
        r = ref.run(p, mesh, st, 64, steps)
        assert r["status"] == 0, r["status_text"]
        sim, orc = make_pair(p, st, mesh, 64, record_pairs=False)
        sim.step(steps)
        orc.step(steps)
        s = sim.state()
        n = s["n"]
        assert n == r["n"] == orc.n
        assert np.array_equal(np.asarray(sim.events()).reshape(-1, 3), r["events"])
        o = {"X": orc.X, "Y": orc.Y, "Z": orc.Z}
        d_ours, d_orc, d_pair = dist(s, r, n), dist(o, r, n), dist(s, o, n)
        centre = np.array([r[k][: n * 192].reshape(n, 192)[:, :180].mean() for k in ("X", "Y", "Z")])
        print("correct_com %2d steps: |dx| CUDA-reference %.2e, oracle-reference %.2e, CUDA-oracle %.2e, "
              "reference centre %s" % (steps, d_ours, d_orc, d_pair, centre))
        assert np.all(np.abs(centre) < 1e-2)      # the system is centred on the origin
        assert d_ours < 2e-5
        assert d_ours <= max(1e-5, 1.5 * d_orc)
        sim.close()
        orc.close()


def test_far_counts_against_reference_kernels(mesh):
    """The internal-cells mitotic count (num_cells_far) after the step-1
    divisions of 56 clustered cells, against the reference's host code."""
    box = 60.0
    c = W.rsa_centres(56, 14.0, np.random.default_rng(11)) + np.float32(23.0)
    p = W.base_params(box_len=(box, box, box), div_time_steps=10 ** 9, count_internal_radius=0.6,
                      rng_ij=11, rng_kl=1100)
    st = W.state(c)
    topo, _ = topo_for(st, mesh)
    r = ref.run(p, mesh, st, 160, 3)
    assert r["status"] == 0, r["status_text"]
    sim = cs.Simulation(p, topo, 160)
    sim.load_state(st["X"], st["Y"], st["Z"], n_cells=st["n"])
    sim.step(3)
    assert sim.n_cells() == r["n"]
    assert np.array_equal(np.asarray(sim.events()).reshape(-1, 3), r["events"])
    assert np.array_equal(sim.far_counts(), r["far"])
    assert len(r["far"]) and r["far"][0].tolist() == [1, 56]
    sim.close()


def test_langevin_statistics_against_reference_kernels(mesh):
    """The Langevin force is Philox4x32-10 here and curand XORWOW (MT19937
    seeds) in the reference, so parity is statistical: 27 non-dividing cells,
    200 steps with rand_scale_factor 1.  The last step's random forces of both
    are samples of the same normal law (two-sample KS test, mean and standard
    deviation), and the node velocities they drive have the same spread."""
    from scipy import stats
    c = np.array([[3 + 2.3 * i, 3 + 2.3 * j, 3 + 2.3 * k] for i in range(3) for j in range(3) for k in range(3)],
                 dtype=np.float32)
    p = W.base_params(box_len=(12.0, 12.0, 12.0), growth_rate=0.0, min_pressure=100.0, max_pressure=100.0,
                      add_rands=1, rand_scale_factor=1.0, rand_seed=17)
    st = W.state(c)
    topo, _ = topo_for(st, mesh)
    r = ref.run(p, mesh, st, 64, 200)
    assert r["status"] == 0, r["status_text"]
    sim = cs.Simulation(p, topo, 64)
    sim.load_state(st["X"], st["Y"], st["Z"], n_cells=st["n"])
    sim.step(200)
    n = st["n"]
    mask = np.zeros((n, 192), bool)
    mask[:, :180] = True
    mask = mask.reshape(-1)
    fr = sim.random_force()
    ours = np.concatenate([fr[k][: n * 192][mask] for k in ("FRX", "FRY", "FRZ")])
    theirs = np.concatenate([r[k][mask] for k in ("FRX", "FRY", "FRZ")])
    ks = stats.ks_2samp(ours, theirs)
    s = sim.state()
    v_ours = np.concatenate([s[k][: n * 192][mask] for k in ("VX", "VY", "VZ")])
    v_ref = np.concatenate([r[k][mask] for k in ("VX", "VY", "VZ")])
    print("random force: ours mean %.4f sd %.4f, reference mean %.4f sd %.4f, KS p %.3f; "
          "velocity sd ours %.4e reference %.4e"
          % (ours.mean(), ours.std(), theirs.mean(), theirs.std(), ks.pvalue, v_ours.std(), v_ref.std()))
    assert ks.pvalue > 1e-3
    for a in (ours, theirs):
        assert abs(a.mean()) < 0.05 and abs(a.std() - 1.0) < 0.03
    assert abs(v_ours.std() / v_ref.std() - 1.0) < 0.15
    sim.close()


def fma32(a, b, c):
    """Elementwise fmaf(a, b, c) of float32 arrays: a*b + c rounded once.  In
    float64 a*b is exact and the sum is rounded twice only where it falls on
    a float32 rounding tie, which the exact fractions recompute."""
    from fractions import Fraction
    a, b, c = (np.asarray(v, np.float32) for v in (a, b, c))
    s = a.astype(np.float64) * b + c
    r = s.astype(np.float32)
    # ties of the float32 rounding of s: recompute exactly
    lo = np.nextafter(r, np.float32(-np.inf)).astype(np.float64)
    hi = np.nextafter(r, np.float32(np.inf)).astype(np.float64)
    tie = (s == 0.5 * (lo + r.astype(np.float64))) | (s == 0.5 * (hi + r.astype(np.float64)))
    for k in np.flatnonzero(tie):
        r[k] = np.float32(float(Fraction(float(a[k])) * Fraction(float(b[k])) + Fraction(float(c[k]))))
    return r


def _reference_accepted(st, n, g, ra):
    """(cell, node, accepted cell) of every node from the reference's own grid
    (bin lists, bounding boxes, extents read back after its makeNNlist), with
    the reference's float expressions for the node's bin and the box filter
    (src/propagate.cu:360-392), in float32 operation by operation."""
    f32 = np.float32
    DL = f32(2.9)
    X = np.stack([st[k][: n * 192].reshape(n, 192)[:, :180] for k in ("X", "Y", "Z")], -1).astype(f32)
    divs = g["divs"]
    idx = []
    for d in range(3):
        s = ((X[..., d] - f32(g["minx"][2 * d])) / DL).astype(f32)
        s = np.trunc(s).astype(np.int64)
        idx.append(np.clip(s, 0, divs[d] - 1))
    b = idx[2] * divs[0] * divs[1] + idx[1] * divs[0] + idx[0]
    bb = g["bb"]
    ra2 = f32(f32(ra) * f32(ra))
    # every (node, cell of the node's bin) pair, vectorised
    bflat = b.reshape(-1)
    cnt = g["counts"][bflat]
    node = np.repeat(np.arange(n * 180), cnt)
    start = np.repeat(np.cumsum(cnt) - cnt, cnt)
    slot = np.arange(len(node)) - start
    cell = g["lists"][bflat[node], slot]
    a = node // 180
    keep = cell != a
    node, cell, a = node[keep], cell[keep], a[keep]
    Xn = X.reshape(-1, 3)[node]
    dd = []
    for d in range(3):
        x = Xn[:, d]
        u = (x - bb[cell, 2 * d + 1]).astype(f32)
        w = (bb[cell, 2 * d] - x).astype(f32)
        dd.append(((u > 0).astype(f32) * u + (w > 0).astype(f32) * w).astype(f32))
    # the reference's build evaluates dx*dx + dy*dy + dz*dz contracted:
    # fma(dz, dz, fma(dx, dx, dy*dy)) (fma32: the exact value rounded once)
    r2 = fma32(dd[2], dd[2], fma32(dd[0], dd[0], (dd[1] * dd[1]).astype(f32)))
    ok = ~(r2 > ra2)
    return list(zip(a[ok].tolist(), (node[ok] % 180).tolist(), cell[ok].tolist()))


@pytest.mark.parametrize("case", ["config1", "packed500"])
def test_candidate_stage_against_the_reference_grid(mesh, case):
    """The reference's own grid after its first makeNNlist
    (src/propagatebound.cu:10-263: bounding boxes, extents, bin lists, read
    back from its device buffers) against the oracle's and the CUDA path's:
    boxes, extents and divisions bit for bit, every bin the same set of cells
    (the reference fills bins in atomic order), and the per-node accepted
    cells derived from the reference's bins (src/propagate.cu:356-404) equal
    to the oracle's.  The CUDA path's contact pairs at this step equal the
    oracle's (pair-set parity), so they come from the reference's
    candidates."""
    import oracle
    from parity import pair_keys
    p, st, cap = CASES[case]()
    n = st["n"]
    r = ref.run(p, mesh, st, cap, 0, dump_grid=True)
    assert r["status"] == 0 and r["max_bin"] <= 32, r["status_text"]
    g = r["grid"]
    sim, O = make_pair(p, st, mesh, capacity=cap)
    assert np.array_equal(g["minx"].view(np.uint32), O.minmax.view(np.uint32))
    assert tuple(g["divs"]) == tuple(O.divs)
    assert np.array_equal(g["bb"].view(np.uint32), O.aabb[:n].view(np.uint32))
    mm, dv = sim.grid()
    assert np.array_equal(mm.view(np.uint32), g["minx"].view(np.uint32)) and tuple(dv) == tuple(g["divs"])
    assert np.array_equal(sim.cells()["aabb"].view(np.uint32), g["bb"].view(np.uint32))
    bins = O.bins()
    assert len(bins) == len(g["counts"])
    for b_, cells in enumerate(bins):
        assert sorted(g["lists"][b_, : g["counts"][b_]].tolist()) == cells.tolist(), b_
    acc_ref = sorted(_reference_accepted(st, n, g, p["attraction_range"]))
    acc_orc = sorted(map(tuple, O.accepted().tolist()))
    print("%s: %d bins, %d (node, accepted cell) entries from the reference's grid" % (case, len(bins), len(acc_ref)))
    assert acc_ref == acc_orc
    for kind in (0, 1):
        assert np.array_equal(pair_keys(sim.pairs(kind)), pair_keys(O.recorded_pairs(kind)))
    sim.close()
    O.close()


def test_boundary_pair_decided_as_the_reference_build(mesh):
    """The reference's own kernels, the CUDA path and the oracle on two cells
    whose one node pair lies at the dissipative cut-off in the uncontracted
    float expression and above it in the contracted one
    (tests/golden/fma_boundary_case.npz, made by make_fma_case.py).  The
    reference's build leaves the pair out (node i feels no friction), and so
    do the CUDA path and the oracle."""
    import os
    import oracle
    c = np.load(os.path.join(os.path.dirname(__file__), "golden", "fma_boundary_case.npz"))
    i, j = int(c["i"]), int(c["j"])
    st = {k: c[k] for k in ("X", "Y", "Z", "VX", "VY", "VZ")}
    st["n"] = 2
    p = W.base_params(box_len=(30.0, 30.0, 30.0))
    r = ref.run(p, mesh, st, 2, 0, dump_init=True)
    assert r["status"] == 0, r["status_text"]
    fd_ref = [float(r["init"][k][i]) for k in ("FDX", "FDY", "FDZ")]
    sim, orc = make_pair(p, st, mesh, capacity=2)
    f = sim.forces()
    fd_gpu = [float(f[k][i]) for k in ("FDX", "FDY", "FDZ")]
    fd_orc = [float(orc.FD[q][i]) for q in range(3)]
    print("boundary pair: reference Fd %s, CUDA path %s, oracle %s" % (fd_ref, fd_gpu, fd_orc))
    assert fd_ref == [0.0, 0.0, 0.0]
    assert fd_gpu == [0.0, 0.0, 0.0] and fd_orc == [0.0, 0.0, 0.0]
    pairs = {tuple(x) for x in sim.pairs(1).tolist()}
    assert (0, i, 1, j) not in pairs and (1, j, 0, i) not in pairs
    # the pair lists of both cut-offs agree with the oracle's
    from parity import pair_keys
    for kind in (0, 1):
        assert np.array_equal(pair_keys(sim.pairs(kind)), pair_keys(orc.recorded_pairs(kind)))
    sim.close()
    orc.close()
