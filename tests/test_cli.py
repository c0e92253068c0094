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
    for f in frames[1:]:
        sim.step(every)
        s = sim.state()
        m = s["n"]
        assert f["X"].shape[0] == m
        for key in ("X", "Y", "Z"):
            assert np.array_equal(f[key].reshape(-1).view(np.uint32), s[key][: m * 192].view(np.uint32)), (f["step"], key)
    print("cs3d driver: %d frames, %d cells at step %d" % (len(frames), frames[-1]["X"].shape[0], steps))
    sim.close()
