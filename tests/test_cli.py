"""The drop-in executable (`cs3d N inp.json gpu`, the reference's `CellDiv`)
end to end: it reads inp.json and the mesh files from the working directory,
runs the steps on the GPU and writes the binary trajectory that
scripts/celldiv.py reads.  Its frames must equal a library run of the same
parameters (read back from the same inp.json) bit for bit."""
import json
import os
import subprocess

import numpy as np
import pytest

import cellsim3d_b200 as cs
from cellsim3d_b200 import traj
from cellsim3d_b200 import workloads as W

from parity import write_mesh_files

CLI = os.path.join(os.path.dirname(cs.__file__), "cs3d")


def test_cli_rejects_bad_arguments():
    """No GPU needed: usage text and a missing inp.json."""
    if not os.path.exists(CLI):
        pytest.skip("cs3d driver not built")
    r = subprocess.run([CLI], capture_output=True, text=True, timeout=60)
    assert "Usage" in r.stdout
    r = subprocess.run([CLI, "8", "/nonexistent/inp.json", "0"], capture_output=True, text=True, timeout=60)
    assert r.returncode != 0 and "cannot open" in r.stderr


@pytest.mark.gpu
def test_cli_trajectory_matches_library(tmp_path, mesh):
    p, st, _ = W.config1()
    p = dict(p, write_cont_force=1)
    steps, every = 300, 100
    write_mesh_files(str(tmp_path), mesh)
    with open(tmp_path / "inp.json", "w") as f:
        json.dump(W.inp_json(p, 256, steps, every, "traj.bin", seed=42), f, indent=1)
    n = st["n"]
    init = dict(st, pressure=np.full(n, p["min_pressure"], np.float32),
                youngs=np.full(n, p["stiffness1"], np.float32))
    W.write_init_file(str(tmp_path / "init.bin"), init)
    env = dict(os.environ, CS3D_INIT_FILE=str(tmp_path / "init.bin"))
    r = subprocess.run([CLI, str(n), "inp.json", "0"], cwd=tmp_path, env=env, capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    hdr, frames = traj.read_traj(str(tmp_path / "traj.bin"))
    assert [f["step"] for f in frames] == [0, 100, 200, 300]
    # the first header word ends as the final cell count, src/GPUbounce.cu:1508-1511
    assert hdr["max_cells"] == frames[-1]["X"].shape[0]

    prm = cs.config_to_params(cs.read_json_params(str(tmp_path / "inp.json")))
    topo = cs.build_topology(cs.read_fullerene_nn(str(tmp_path)), st["X"][:192], st["Y"][:192], st["Z"][:192])
    sim = cs.Simulation(prm, topo, 256)
    sim.load_state(st["X"], st["Y"], st["Z"], n_cells=n)
    # the force file (write_cont_force, writeForces src/GPUbounce.cu:2567-2597):
    # a header, then one row per node at step 0 and at every frame
    lines = open(tmp_path / "forces.csv").read().splitlines()
    assert lines[0] == "step,num_cells,cell_ind,node_ind,glob_node_ind,FX,FY,FZ,F,VX,VY,VZ,V,X,Y,Z,P,Vol"
    rows = {}
    for ln in lines[1:]:
        rows.setdefault(int(ln.split(",", 1)[0]), []).append(ln)
    assert sorted(rows) == [0, 100, 200, 300]

    def expect_rows(step, s, fc, vol, X=None):
        m = s["n"]
        X = X if X is not None else (s["X"], s["Y"], s["Z"])
        out = []
        for c in range(m):
            for k in range(180):
                g = c * 192 + k
                F = [np.float32(fc[q][g]) for q in ("FCX", "FCY", "FCZ")]
                V = [np.float32(s[q][g]) for q in ("VX", "VY", "VZ")]
                mag = lambda a: np.sqrt(np.float32(np.float32(a[0] * a[0] + a[1] * a[1]) + a[2] * a[2]), dtype=np.float32)
                vals = F + [mag(F)] + V + [mag(V)] + [np.float32(X[q][g]) for q in range(3)] + [s["pressure"][c], vol[c]]
                out.append("%d,%d,%d,%d,%d," % (step, m, c, k, g) + ",".join("%.8f" % float(v) for v in vals))
        return out

    s0 = sim.state()
    assert rows[0] == expect_rows(0, s0, sim.forces(), sim.cells()["volume"], (st["X"], st["Y"], st["Z"]))
    for f in frames[1:]:
        sim.step(every)
        s = sim.state()
        m = s["n"]
        assert f["X"].shape[0] == m
        for key in ("X", "Y", "Z"):
            assert np.array_equal(f[key].reshape(-1).view(np.uint32), s[key][: m * 192].view(np.uint32)), (f["step"], key)
        assert rows[f["step"]] == expect_rows(f["step"], s, sim.forces(), sim.cells()["volume"]), f["step"]
    print("cs3d driver: %d frames, %d cells at step %d" % (len(frames), frames[-1]["X"].shape[0], steps))
    sim.close()


@pytest.mark.gpu
def test_cli_variable_stiffness_and_internal_count(tmp_path, mesh):
    """The driver with variable stiffness and the internal-cells mitotic
    count: 56 clustered cells divide at step 1 (their daughters all lie far
    from the system centre), the central cells start soft, RANMAR picks are
    softened at the end of step 202; the binary frames carry the stiffness class of
    every cell, and the mitotic-index file leaves the far daughters out."""
    box = 60.0
    c = W.rsa_centres(56, 14.0, np.random.default_rng(11)) + np.float32(23.0)
    p = W.soft_params(W.base_params(box_len=(box, box, box), count_internal_radius=0.6), phase_count=100,
                      soften_after_growth=1, number_of_softer_cells=10, closeness_to_center=0.5,
                      choose_random_cell_indices=1)
    steps, non_div, every = 200, 100, 100
    st = W.state(c)
    n = st["n"]
    write_mesh_files(str(tmp_path), mesh)
    with open(tmp_path / "inp.json", "w") as f:
        json.dump(W.inp_json(p, 256, steps, every, "traj.bin", seed=42, non_div_steps=non_div), f, indent=1)
    cfg = cs.read_json_params(str(tmp_path / "inp.json"))
    prm = cs.config_to_params(cfg)
    E0 = cs.initial_stiffness(cfg, st["X"], st["Y"], st["Z"], n)
    assert 0 < int((E0 != np.float32(prm.stiffness1)).sum()) < n
    init = dict(st, pressure=np.full(n, p["min_pressure"], np.float32), youngs=E0)
    W.write_init_file(str(tmp_path / "init.bin"), init)
    env = dict(os.environ, CS3D_INIT_FILE=str(tmp_path / "init.bin"))
    r = subprocess.run([CLI, str(n), "inp.json", "0"], cwd=tmp_path, env=env, capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    hdr, frames = traj.read_traj(str(tmp_path / "traj.bin"))
    assert hdr["variable_stiffness"] == 1
    assert [f["step"] for f in frames] == [0, 100, 200, 300]

    topo = cs.build_topology(cs.read_fullerene_nn(str(tmp_path)), st["X"][:192], st["Y"][:192], st["Z"][:192])
    sim = cs.Simulation(prm, topo, 256)
    sim.load_state(st["X"], st["Y"], st["Z"], youngs=E0, n_cells=n)
    soft_counts = []
    for f in frames:
        if f["step"]:
            sim.step(every)
        s = sim.state()
        m = s["n"]
        assert f["X"].shape[0] == m
        assert np.array_equal(f["X"].reshape(-1).view(np.uint32), s["X"][: m * 192].view(np.uint32)), f["step"]
        types = (s["youngs"][:m] != np.float32(prm.stiffness1)).astype(np.int32)
        assert np.array_equal(f["types"], types), f["step"]
        soft_counts.append(int(types.sum()))
    assert soft_counts[-1] > soft_counts[-2]          # softened at the end of step 202

    # mitotic index of internal cells (src/GPUbounce.cu:1288-1302, :1515-1547)
    ev, far = sim.events(), sim.far_counts()
    assert len(far) and far[0].tolist() == [1, 56]
    born = np.zeros(steps + 1, int)
    for e in ev:
        born[e[0]] += 1
    counted = born.copy()
    for s_, k in far:
        counted[s_] -= k
    cci = max(1, min(1000, steps))
    buckets = [0.0] * (steps // cci + 1)
    cells = n
    for s_ in range(1, steps + 1):
        cells += born[s_]
        if s_ % cci == 0:
            nc = counted[s_ - cci + 1: s_ + 1].sum()
            tot = cells - nc
            buckets[(s_ - 1) // cci] = float(np.float32(nc) / np.float32(tot)) if nc and tot else 0.0
    got = [float(v) for v in open(tmp_path / "mit-index.dat").read().split()]
    assert got == pytest.approx(buckets, abs=1e-6)
    sim.close()
