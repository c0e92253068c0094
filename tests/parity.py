"""Shared helpers of the parity tests: set up one workload in the CUDA path
(through the C ABI) and in the oracle from identical float32 inputs, and the
error metrics of the parity bar (per node: |F - F_ref| / max(|F_ref|,
1e-3 * median|F_ref|); global: ||dF||_2 / ||F_ref||_2)."""
import numpy as np

import cellsim3d_b200 as cs
import oracle
from cellsim3d_b200 import workloads as W

TOL = 1e-5   # relative force / velocity tolerance of the parity bar


def topo_for(st, mesh):
    m = cs.mesh_from_arrays(mesh)
    topo = cs.build_topology(m, st["X"][:192], st["Y"][:192], st["Z"][:192])
    r0 = np.frombuffer(topo.r0, np.float32)
    th = np.frombuffer(topo.theta0, np.float32)
    otopo = oracle.make_topo(mesh["nn"], mesh["sign"], r0, th, mesh["faces"])
    return topo, otopo


def make_pair(p, st, mesh, capacity, record_pairs=True, pair_capacity=1 << 22):
    topo, otopo = topo_for(st, mesh)
    sim = cs.Simulation(p, topo, capacity)
    if record_pairs:
        sim.set_option(cs.OPT_PAIR_CAPACITY, pair_capacity)
        sim.set_option(cs.OPT_RECORD_PAIRS, 1)
    sim.load_state(st["X"], st["Y"], st["Z"], st.get("VX"), st.get("VY"), st.get("VZ"),
                   st.get("pressure"), None, n_cells=st["n"])
    orc = oracle.System(capacity, p, otopo)
    orc.load(st["X"], st["Y"], st["Z"], st.get("VX"), st.get("VY"), st.get("VZ"),
             pressure=st.get("pressure"), n=st["n"])
    orc.seed(p["rng_ij"], p["rng_kl"])
    orc.set_record(record_pairs)
    orc.init()
    return sim, orc


def node_mask(n):
    m = np.zeros((n, 192), bool)
    m[:, :180] = True
    return m.reshape(-1)


def rel_err(got, ref, n):
    """(max per-node floor-relative error, global relative error)."""
    msk = node_mask(n)
    g = np.stack([a[: n * 192] for a in got], -1)[msk].astype(np.float64)
    r = np.stack([a[: n * 192] for a in ref], -1)[msk].astype(np.float64)
    nr = np.linalg.norm(r, axis=1)
    floor = max(1e-3 * float(np.median(nr)), 1e-30)
    e = np.linalg.norm(g - r, axis=1) / np.maximum(nr, floor)
    glob = np.linalg.norm(g - r) / max(np.linalg.norm(r), 1e-30)
    return float(e.max()), float(glob), float(np.percentile(e, 99))


def force_errors(sim, orc):
    n = sim.n_cells()
    f = sim.forces()
    FC, FD = orc.FC, orc.FD
    ec = rel_err([f["FCX"], f["FCY"], f["FCZ"]], [FC[0], FC[1], FC[2]], n)
    ed = rel_err([f["FDX"], f["FDY"], f["FDZ"]], [FD[0], FD[1], FD[2]], n)
    return ec, ed


def sorted_pairs(a):
    a = np.asarray(a, dtype=np.int64)
    if len(a) == 0:
        return a.reshape(0, 4)
    key = ((a[:, 0] * 256 + a[:, 1]) * (1 << 24) + a[:, 2]) * 256 + a[:, 3]
    return a[np.argsort(key, kind="stable")]
