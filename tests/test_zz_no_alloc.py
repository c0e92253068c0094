"""cs3d_forces_static: the force evaluation for callers that cannot allocate
GPU memory (a host that owns the device's memory through its own pool, a
real-time loop that must not call cudaMalloc/cudaFree, a plugin host that
forbids allocation in callbacks).  It takes device pointers the caller owns
and keeps its scratch in a static device array of the library.

Checked through the C ABI against the existing entry point (cs3d_load_state
followed by cs3d_get_forces) on the same inputs, on two calls in a row, with
the tolerance of the parity tests.  This file is collected last on purpose.
"""
import ctypes as C

import numpy as np
import pytest

import cellsim3d_b200 as cs
from cellsim3d_b200 import _lib
from cellsim3d_b200 import workloads as W

from parity import TOL, rel_err

pytestmark = pytest.mark.gpu


def _states():
    p1, st1, _ = W.config1()
    c, vel, L = W.packed_fcc(27, phi=0.5, seed=5)
    p2 = W.base_params(box_len=(L, L, L), growth_rate=0.0, min_pressure=200.0, max_pressure=200.0)
    return [(p1, st1), (p2, W.state(c, velocities=vel))]


def _reference_forces(p, st, topo):
    sim = cs.Simulation(p, topo, st["n"])
    sim.load_state(st["X"], st["Y"], st["Z"], st.get("VX"), st.get("VY"), st.get("VZ"), n_cells=st["n"])
    f = sim.forces()
    sim.close()
    return f


def _static_forces(p, st, topo, torch):
    n = st["n"]
    dev = torch.device("cuda", 0)
    ins = {k: torch.from_numpy(np.ascontiguousarray(st[k][: n * 192])).to(dev)
           for k in ("X", "Y", "Z", "VX", "VY", "VZ") if k in st}
    outs = {k: torch.full((n * 192,), float("nan"), dtype=torch.float32, device=dev)
            for k in ("FCX", "FCY", "FCZ", "FDX", "FDY", "FDZ")}
    torch.cuda.synchronize()
    ptr = lambda k: C.c_void_p(ins[k].data_ptr()) if k in ins else None
    rc = _lib.lib().cs3d_forces_static(C.byref(cs.make_params(p)), C.byref(topo), n,
                                       ptr("X"), ptr("Y"), ptr("Z"), ptr("VX"), ptr("VY"), ptr("VZ"), None, None,
                                       *[C.c_void_p(outs[k].data_ptr()) for k in ("FCX", "FCY", "FCZ", "FDX", "FDY", "FDZ")],
                                       None)
    assert rc == 0, cs.CS3DError("cs3d_forces_static", rc)
    torch.cuda.synchronize()
    return {k: v.cpu().numpy() for k, v in outs.items()}


def test_static_forces_match_existing_entry_point(mesh):
    import torch
    m = cs.mesh_from_arrays(mesh)
    for p, st in _states():
        topo = cs.build_topology(m, st["X"][:192], st["Y"][:192], st["Z"][:192])
        ref = _reference_forces(p, st, topo)
        n = st["n"]
        free_after_first = None
        for call in range(2):
            got = _static_forces(p, st, topo, torch)
            if call == 0:
                free_after_first = torch.cuda.mem_get_info()[0]
            ec = rel_err([got["FCX"], got["FCY"], got["FCZ"]], [ref["FCX"], ref["FCY"], ref["FCZ"]], n)
            ed = rel_err([got["FDX"], got["FDY"], got["FDZ"]], [ref["FDX"], ref["FDY"], ref["FDZ"]], n)
            assert ec[0] < TOL and ed[0] < TOL, (n, call, ec, ed)
            pad = np.zeros((n, 192), bool)
            pad[:, 180:] = True
            assert np.all(got["FCX"].reshape(n, 192)[pad.reshape(n, 192)] == 0)
        # the second call allocated nothing the device reports
        assert torch.cuda.mem_get_info()[0] == free_after_first


def test_static_forces_reject_oversized_system(mesh):
    p, st, _ = W.config1()
    topo = cs.build_topology(cs.mesh_from_arrays(mesh), st["X"][:192], st["Y"][:192], st["Z"][:192])
    rc = _lib.lib().cs3d_forces_static(C.byref(cs.make_params(p)), C.byref(topo), 65, *([C.c_void_p(16)] * 3),
                                       None, None, None, None, None, *([C.c_void_p(16)] * 6), None)
    assert rc == _lib.E_ARG
