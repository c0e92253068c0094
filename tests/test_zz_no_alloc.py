"""cs3d_forces_static: the force evaluation for callers that cannot allocate
GPU memory (a host that owns the device's memory through its own pool, a
real-time loop that must not call cudaMalloc/cudaFree, a plugin host that
forbids allocation in callbacks).  It takes device pointers the caller owns
and keeps its scratch in a static device array of the library.

Checked through the C ABI against the FP64 oracle's initial forces and
against the existing entry point (cs3d_load_state followed by
cs3d_get_forces) on the same inputs, on two calls in a row, with the
tolerance of the parity tests.  This file is collected last on purpose.
"""
import ctypes as C

import numpy as np
import pytest

import cellsim3d_b200 as cs
from cellsim3d_b200 import _lib
from cellsim3d_b200 import workloads as W

import oracle
from parity import TOL, rel_err, topo_for

pytestmark = pytest.mark.gpu


def _states():
    p1, st1, _ = W.config1()
    c, vel, L = W.packed_fcc(27, phi=0.5, seed=5)
    p2 = W.base_params(box_len=(L, L, L), growth_rate=0.0, min_pressure=200.0, max_pressure=200.0)
    # centre-of-mass correction with the rigid box on: the shift moves the
    # cells against the box walls, so the wall forces depend on it
    p3 = dict(p1, correct_com=1, use_rigid_box=1)
    return [(p1, st1), (p2, W.state(c, velocities=vel)), (p3, st1)]


def _reference_forces(p, st, topo):
    sim = cs.Simulation(p, topo, st["n"])
    sim.load_state(st["X"], st["Y"], st["Z"], st.get("VX"), st.get("VY"), st.get("VZ"), n_cells=st["n"])
    f = sim.forces()
    sim.close()
    return f


def _oracle_forces(p, st, mesh):
    """The oracle's initial forces (src/GPUbounce.cu:978-1004) on the same
    state, with the oracle's own R0/theta0 tables (equal to the library's,
    which topo_for asserts)."""
    _, otopo = topo_for(st, mesh)
    n = st["n"]
    o = oracle.System(n, p, otopo)
    o.load(st["X"], st["Y"], st["Z"], st.get("VX"), st.get("VY"), st.get("VZ"), n=n)
    o.seed(p["rng_ij"], p["rng_kl"])
    o.init()
    f = {"FCX": o.FC[0].copy(), "FCY": o.FC[1].copy(), "FCZ": o.FC[2].copy(),
         "FDX": o.FD[0].copy(), "FDY": o.FD[1].copy(), "FDZ": o.FD[2].copy()}
    o.close()
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
    """Two calls in a row per state, each against the FP64 oracle and
    against the existing entry point (cs3d_load_state + cs3d_get_forces)
    within the parity tolerance."""
    import torch
    m = cs.mesh_from_arrays(mesh)
    for p, st in _states():
        topo = cs.build_topology(m, st["X"][:192], st["Y"][:192], st["Z"][:192])
        ref = _reference_forces(p, st, topo)
        orc = _oracle_forces(p, st, mesh)
        n = st["n"]
        for call in range(2):
            got = _static_forces(p, st, topo, torch)
            for tag, want in (("oracle", orc), ("entry point", ref)):
                ec = rel_err([got["FCX"], got["FCY"], got["FCZ"]], [want["FCX"], want["FCY"], want["FCZ"]], n)
                ed = rel_err([got["FDX"], got["FDY"], got["FDZ"]], [want["FDX"], want["FDY"], want["FDZ"]], n)
                assert ec[0] < TOL and ed[0] < TOL, (tag, n, call, p.get("correct_com"), ec, ed)
            # padding slots 180..191 are zero in all six outputs
            for k in ("FCX", "FCY", "FCZ", "FDX", "FDY", "FDZ"):
                assert np.all(got[k].reshape(n, 192)[:, 180:] == 0), (k, call)


def test_static_forces_allocate_nothing(mesh):
    """Free device memory stays the same across calls.  Only calls after the
    first one of this test are compared: with CUDA's lazy module loading, the
    library's module image (the static scratch array included) is placed on
    the device at the first use of any of its kernels or symbols, which in a
    fresh process is this test's first call."""
    import torch
    p, st, _ = W.config1()
    topo = cs.build_topology(cs.mesh_from_arrays(mesh), st["X"][:192], st["Y"][:192], st["Z"][:192])
    # the caller's device buffers, allocated before any measurement
    n = st["n"]
    dev = torch.device("cuda", 0)
    ins = [torch.from_numpy(np.ascontiguousarray(st[k][: n * 192])).to(dev) for k in ("X", "Y", "Z")]
    outs = [torch.zeros(n * 192, dtype=torch.float32, device=dev) for _ in range(6)]
    torch.cuda.synchronize()
    free0 = None
    for call in range(3):
        rc = _lib.lib().cs3d_forces_static(C.byref(cs.make_params(p)), C.byref(topo), n,
                                           *[C.c_void_p(t.data_ptr()) for t in ins], None, None, None, None, None,
                                           *[C.c_void_p(t.data_ptr()) for t in outs], None)
        assert rc == 0
        torch.cuda.synchronize()
        if free0 is None:
            free0 = torch.cuda.mem_get_info()[0]
        assert torch.cuda.mem_get_info()[0] == free0, call


def test_static_forces_reject_oversized_system(mesh):
    p, st, _ = W.config1()
    topo = cs.build_topology(cs.mesh_from_arrays(mesh), st["X"][:192], st["Y"][:192], st["Z"][:192])
    rc = _lib.lib().cs3d_forces_static(C.byref(cs.make_params(p)), C.byref(topo), 65, *([C.c_void_p(16)] * 3),
                                       None, None, None, None, None, *([C.c_void_p(16)] * 6), None)
    assert rc == _lib.E_ARG
