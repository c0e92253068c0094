"""Shared helpers of the parity tests.

The parity bar is checked on identical inputs: a single step of the CUDA
path (through the C ABI) and of the FP64 oracle from the same float state,
taken from the CUDA path itself.  Error metrics: per node
|F - F_ref| / max(|F_ref|, 1e-3 * median|F_ref|) and globally
||dF||_2 / ||F_ref||_2."""
import numpy as np

import cellsim3d_b200 as cs
import oracle

TOL = 1e-5   # relative force / velocity tolerance of the parity bar


def topo_for(st, mesh):
    """The library's tables (cs3d_topology_build) and the oracle's, each
    computed independently from cell 0 of the state (the oracle's by its own
    restatement of src/GPUbounce.cu:1890-1908 and :909-935); they must agree
    bit for bit."""
    m = cs.mesh_from_arrays(mesh)
    topo = cs.build_topology(m, st["X"][:192], st["Y"][:192], st["Z"][:192])
    r0, th = oracle.r0_theta0(st["X"][:192], st["Y"][:192], st["Z"][:192], mesh["nn"])
    assert np.array_equal(np.frombuffer(topo.r0, np.float32).view(np.uint32), r0.view(np.uint32)), "R0 tables differ"
    assert np.array_equal(np.frombuffer(topo.theta0, np.float32).view(np.uint32), th.view(np.uint32)), \
        "theta0 tables differ"
    otopo = oracle.make_topo(mesh["nn"], mesh["sign"], r0, th, mesh["faces"])
    return topo, otopo


def make_pair(p, st, mesh, capacity, record_pairs=True, pair_capacity=1 << 22):
    """A Simulation and a tracking oracle started from the same initial state."""
    topo, otopo = topo_for(st, mesh)
    sim = cs.Simulation(p, topo, capacity)
    if record_pairs:
        sim.set_option(cs.OPT_PAIR_CAPACITY, pair_capacity)
        sim.set_option(cs.OPT_RECORD_PAIRS, 1)
    sim.load_state(st["X"], st["Y"], st["Z"], st.get("VX"), st.get("VY"), st.get("VZ"),
                   st.get("pressure"), st.get("youngs"), n_cells=st["n"])
    orc = oracle.System(capacity, p, otopo)
    orc.load(st["X"], st["Y"], st["Z"], st.get("VX"), st.get("VY"), st.get("VZ"),
             pressure=st.get("pressure"), youngs=st.get("youngs"), n=st["n"])
    orc.seed(p["rng_ij"], p["rng_kl"])
    orc.set_record(record_pairs)
    orc.init()
    sim.otopo = otopo
    sim.params = p
    sim.capacity = capacity
    return sim, orc


def node_mask(n, exclude_cells=()):
    m = np.zeros((n, 192), bool)
    m[:, :180] = True
    for c in exclude_cells:
        if c < n:
            m[c] = False
    return m.reshape(-1)


def rel_err(got, ref, n, exclude_cells=()):
    """(max per-node floor-relative error, global relative error, p99)."""
    msk = node_mask(n, exclude_cells)
    g = np.stack([np.asarray(a)[: n * 192] for a in got], -1)[msk].astype(np.float64)
    r = np.stack([np.asarray(a)[: n * 192] for a in ref], -1)[msk].astype(np.float64)
    if len(r) == 0:
        return 0.0, 0.0, 0.0
    nr = np.linalg.norm(r, axis=1)
    floor = max(1e-3 * float(np.median(nr)), 1e-30)
    e = np.linalg.norm(g - r, axis=1) / np.maximum(nr, floor)
    glob = np.linalg.norm(g - r) / max(np.linalg.norm(r), 1e-30)
    return float(e.max()), float(glob), float(np.percentile(e, 99))


def force_errors(sim, orc, exclude_cells=()):
    n = sim.n_cells()
    f = sim.forces()
    FC, FD = orc.FC, orc.FD
    ec = rel_err([f["FCX"], f["FCY"], f["FCZ"]], [FC[0], FC[1], FC[2]], n, exclude_cells)
    ed = rel_err([f["FDX"], f["FDY"], f["FDZ"]], [FD[0], FD[1], FD[2]], n, exclude_cells)
    return ec, ed


def sorted_pairs(a):
    a = np.asarray(a, dtype=np.int64)
    if len(a) == 0:
        return a.reshape(0, 4)
    key = ((a[:, 0] * 256 + a[:, 1]) * (1 << 24) + a[:, 2]) * 256 + a[:, 3]
    return a[np.argsort(key, kind="stable")]


def pair_keys(a):
    """The pair set (cell_a, node_i, cell_b, node_j) as sorted unique int64
    keys: equal key arrays mean equal sets (cells < 2^24, nodes < 256)."""
    a = np.asarray(a)
    if len(a) == 0:
        return np.zeros(0, np.int64)
    key = ((a[:, 0].astype(np.int64) * 256 + a[:, 1]) * (1 << 24) + a[:, 2]) * 256 + a[:, 3]
    key.sort()
    return key


def snapshot(sim, inst=0):
    st = sim.state(inst)
    st.update(sim.forces(inst))
    st.update(sim.random_force(inst))
    cells = sim.cells(inst)
    st["cm"] = cells["cm"]
    st["aabb"] = cells["aabb"]
    st["minmax"] = sim.grid(inst)[0]
    st["rng"] = sim.get_rng(inst)
    st["step"] = sim.stats()["steps"]
    return st


def oracle_from(snap, p, otopo, capacity, record=True):
    """An oracle holding the CUDA path's state after a step (float inputs)."""
    O = oracle.System(capacity, p, otopo)
    n = snap["n"]
    O.load(snap["X"], snap["Y"], snap["Z"], snap["VX"], snap["VY"], snap["VZ"],
           pressure=snap["pressure"], youngs=snap["youngs"], n=n)
    O.load_forces(snap["FCX"], snap["FCY"], snap["FCZ"], snap["FDX"], snap["FDY"], snap["FDZ"])
    k = n * 192
    O.FR[0][:k], O.FR[1][:k], O.FR[2][:k] = snap["FRX"][:k], snap["FRY"][:k], snap["FRZ"][:k]
    O.load_cm(snap["cm"])
    O.set_rng_from(snap["rng"].state)
    O.set_step(snap["step"])
    if "aabb" in snap:
        O.load_grid(snap["aabb"], snap["minmax"])   # the stale grid is part of the state
    else:
        O.compute_grid()
    O.set_record(record)
    return O


def single_step_check(sim, tag="", tol=TOL, check_pairs=True):
    """Step the CUDA path once and the oracle once from the identical state;
    returns a dict of the measured errors after asserting the parity bar."""
    return ensemble_step_check(sim, [sim.params], [sim.capacity], sim.otopo, [tag], tol, check_pairs)[0]


def ensemble_step_check(ens, params, caps, otopo, tags, tol=TOL, check_pairs=True):
    """One step of every instance of `ens` and of one oracle per instance
    started from the instance's state (positions, velocities, forces, stale
    grid, centres of mass, RANMAR state: everything the step reads).  Per
    instance: cell count, the step's division events, both contact-pair sets,
    positions, pressures and stiffnesses exactly; the conservative force, the
    dissipative force and the velocities within `tol`."""
    n_inst = len(params)
    before = [snapshot(ens, k) for k in range(n_inst)]
    Os = [oracle_from(before[k], params[k], otopo, caps[k], record=check_pairs) for k in range(n_inst)]
    ens.step(1)
    out = []
    for k in range(n_inst):
        p, cap, tag, O = params[k], caps[k], tags[k], Os[k]
        O.step(1)
        after = snapshot(ens, k)
        n = after["n"]
        res = {"tag": tag, "n": n}
        # discrete results: cell count, division events of this step, pair sets
        assert n == O.n, (tag, n, O.n)
        ev_g = ens.events(k)
        ev_g = ev_g[ev_g[:, 0] == after["step"]] if len(ev_g) else ev_g
        ev_o = O.events()
        assert np.array_equal(ev_g, ev_o), (tag, "division events", ev_g, ev_o)
        res["events"] = len(ev_o)
        divided = set(ev_g[:, 1].tolist()) | set(ev_g[:, 2].tolist()) if len(ev_g) else set()
        if check_pairs:
            npairs = []
            for kind in (0, 1):
                g = pair_keys(ens.pairs(kind, k))
                r = pair_keys(O.recorded_pairs(kind))
                assert g.shape == r.shape and np.array_equal(g, r), (tag, "pair set", kind, g.shape, r.shape)
                npairs.append(len(g))
            res["pairs"] = tuple(npairs)
        # positions after the drift and the division geometry: bit-exact
        kk = n * 192
        for a, b in (("X", O.X), ("Y", O.Y), ("Z", O.Z)):
            assert np.array_equal(after[a][:kk].view(np.uint32), b[:kk].view(np.uint32)), (tag, "positions", a)
        # per-cell pressure and bond stiffness: exact
        assert np.array_equal(after["pressure"][:n].view(np.uint32), O.press[:n].view(np.uint32)), (tag, "pressure")
        assert np.array_equal(after["youngs"][:n].view(np.uint32), O.E[:n].view(np.uint32)), (tag, "stiffness")
        cm_o = O.CM[:, :n].T
        # conservative force (identical inputs)
        ec = rel_err([after["FCX"], after["FCY"], after["FCZ"]], [O.FC[0], O.FC[1], O.FC[2]], n)
        # velocities after the step
        evv = rel_err([after["VX"], after["VY"], after["VZ"]], [O.VX, O.VY, O.VZ], n)
        # dissipative force on identical inputs: the CUDA path's own v3 and x,
        # stale grid of the previous step.  The positions are those of the
        # force evaluation: the positions after the step, except for the cells
        # that divided this step, whose nodes the division moved after the
        # evaluation (their neighbours' friction saw the old ones), and except
        # with correct_com, which shifts every node after the evaluation; both
        # are rebuilt from the state before the step by the integrator's float
        # arithmetic.  The two cells of each division are left out of the
        # comparison.
        O2 = oracle_from(before[k], p, otopo, cap, record=False)
        O2.X[:kk], O2.Y[:kk], O2.Z[:kk] = after["X"][:kk], after["Y"][:kk], after["Z"][:kk]
        n_before = before[k]["n"]
        parents = [c for c in divided if c < n_before]
        if p.get("correct_com") or parents:
            xs = drift_positions(before[k], p)
            kb = n_before * 192
            if p.get("correct_com"):
                O2.X[:kb], O2.Y[:kb], O2.Z[:kb] = xs[0][:kb], xs[1][:kb], xs[2][:kb]
            else:
                for c in parents:
                    sl = slice(c * 192, (c + 1) * 192)
                    O2.X[sl], O2.Y[sl], O2.Z[sl] = xs[0][sl], xs[1][sl], xs[2][sl]
        O2.VX[:kk], O2.VY[:kk], O2.VZ[:kk] = after["VX"][:kk], after["VY"][:kk], after["VZ"][:kk]
        O2._n[0] = n
        O2.dis_force()
        fd_ref = O2.FD
        ed = rel_err([after["FDX"], after["FDY"], after["FDZ"]], [fd_ref[0], fd_ref[1], fd_ref[2]], n,
                     exclude_cells=sorted(divided))
        res.update(fc=ec, fd=ed, v=evv,
                   cm_exact=bool(np.array_equal(after["cm"].view(np.uint32), cm_o.view(np.uint32))))
        print("%-26s n=%6d Fc max %.2e glob %.2e | Fd max %.2e glob %.2e | V max %.2e glob %.2e | pairs %s"
              % (tag, n, ec[0], ec[1], ed[0], ed[1], evv[0], evv[1], res.get("pairs")))
        assert ec[0] < tol and ec[1] < tol, (tag, "Fc", ec)
        assert ed[0] < tol and ed[1] < tol, (tag, "Fd", ed)
        assert evv[0] < tol and evv[1] < tol, (tag, "V", evv)
        O.close()
        O2.close()
        out.append(res)
    return out


def drift_positions(snap, p):
    """Positions after the first half kick and drift of a step from the state
    `snap` (Integrate + ForwardTime: float sums, the kick scaled in double,
    x + v dt rounded once)."""
    f32, f64 = np.float32, np.float64
    dt = f32(p["time_interval"])
    m = f64(p["particle_mass"])
    rdt = np.sqrt(dt, dtype=np.float32)
    out = []
    for a, fc, fd, fr, v in (("X", "FCX", "FDX", "FRX", "VX"), ("Y", "FCY", "FDY", "FRY", "VY"),
                             ("Z", "FCZ", "FDZ", "FRZ", "VZ")):
        s = (dt * snap[fc].astype(f32)).astype(f32) + (dt * snap[fd].astype(f32)).astype(f32)
        if p.get("add_rands"):
            s = s + (rdt * snap[fr].astype(f32)).astype(f32)
        v1 = (snap[v].astype(f64) + 0.5 * s.astype(f64) / m).astype(f32)
        out.append((snap[a].astype(f64) + v1.astype(f64) * f64(dt)).astype(f32))
    return out


def write_mesh_files(d, mesh):
    """The reference's mesh files (C180, C180NN, C180C, C180_pentahexa) from
    the fixture, in the reference's text formats."""
    import os
    with open(os.path.join(d, "C180"), "w") as f:
        for p in mesh["xyz"]:
            f.write("%.9g  %.9g  %.9g\n" % tuple(float(v) for v in p))
    with open(os.path.join(d, "C180NN"), "w") as f:
        for i in range(180):
            f.write(" %d,  %d,  %d,  %d\n" % (mesh["nn"][0, i] + 1, mesh["nn"][1, i] + 1, mesh["nn"][2, i] + 1,
                                            mesh["sign"][i]))
    with open(os.path.join(d, "C180C"), "w") as f:
        for a, b in mesh["bonds"]:
            f.write(" %d,  %d\n" % (a + 1, b + 1))
    with open(os.path.join(d, "C180_pentahexa"), "w") as f:
        for k in range(92):
            m = 5 if k < 12 else 6
            f.write("  ".join(str(v) for v in mesh["faces"][k, :m]) + "\n")
