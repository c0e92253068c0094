"""The equilibrium bond lengths R0 and angles theta0, computed three ways from
the same cell-0 positions, must agree bit for bit:

* the library's cs3d_topology_build (cellsim3d_b200/csrc/cs3d_host.cpp);
* the oracle's restatement (oracle/cs3d_oracle.c, orc_r0_theta0);
* the reference's own host code (src/GPUbounce.cu:1890-1908 for R0, :909-935
  for theta0, with the float3 helpers of inc/VectorFunctions.hpp), compiled
  from the reference sources into oracle/_ref/cs3d_ref and run in its
  `--tables` mode, which makes no CUDA call.

Placements: every benchmark configuration's cell 0, the unscaled native mesh,
and meshes translated far from the origin (where the float subtractions of
the differences round differently)."""
import numpy as np
import pytest

import cellsim3d_b200 as cs
import oracle
from cellsim3d_b200 import workloads as W


def _placements(mesh):
    out = {}
    p, st, _ = W.config1()
    out["config1"] = (p, st)
    p, st, _ = W.config2()
    out["config2"] = (p, st)
    c, vel, L = W.packed_fcc(64, phi=0.5, seed=123)
    out["packed"] = (W.base_params(box_len=(L, L, L)), W.state(c, velocities=vel))
    p5, st5 = W.config5(n_inst=2)[1]
    out["het64 instance"] = (p5, st5)
    native = W.centred(mesh["xyz"])
    for name, shift in (("native", (0.0, 0.0, 0.0)), ("native far", (47.3, -81.9, 1234.5)),
                        ("scaled far", (93.1, 0.7, 61.25))):
        xyz = native if name.startswith("native") else W.centred(W.scaled_xyz(mesh))
        X, Y, Z = W.place(xyz, [shift])
        out[name] = (W.base_params(box_len=(100.0, 100.0, 100.0)), {"X": X, "Y": Y, "Z": Z, "n": 1})
    return out


def _bits(a):
    return np.ascontiguousarray(a, dtype=np.float32).view(np.uint32)


@pytest.fixture(scope="module")
def placements(mesh):
    return _placements(mesh)


def test_library_tables_equal_oracle_tables(mesh, placements):
    for name, (p, st) in placements.items():
        t = cs.build_topology(cs.mesh_from_arrays(mesh), st["X"][:192], st["Y"][:192], st["Z"][:192])
        r0, th = oracle.r0_theta0(st["X"][:192], st["Y"][:192], st["Z"][:192], mesh["nn"])
        assert np.array_equal(_bits(np.frombuffer(t.r0, np.float32)), _bits(r0)), name
        assert np.array_equal(_bits(np.frombuffer(t.theta0, np.float32)), _bits(th)), name
        # the angles are of a C180 vertex: two hexagon-hexagon and one
        # pentagon-hexagon angle near 2 rad, all inside (0, pi)
        assert np.all((th[:540] > 1.5) & (th[:540] < 2.5)), name
        assert np.all(r0.reshape(3, 192)[:, :180] > 0), name


def test_reference_host_tables_equal_library_tables(mesh, placements):
    from oracle import ref
    if not ref.available():
        pytest.skip("oracle/_ref/cs3d_ref not built (needs the reference sources)")
    for name, (p, st) in placements.items():
        r0_ref, th_ref = ref.tables(p, mesh, st)
        t = cs.build_topology(cs.mesh_from_arrays(mesh), st["X"][:192], st["Y"][:192], st["Z"][:192])
        assert np.array_equal(_bits(r0_ref), _bits(np.frombuffer(t.r0, np.float32))), name
        assert np.array_equal(_bits(th_ref), _bits(np.frombuffer(t.theta0, np.float32))), name


def test_tables_detect_a_one_ulp_change(mesh):
    """The comparison is sharp: moving one node of cell 0 by one ulp changes
    at least one table entry in the oracle's restatement."""
    p, st, _ = W.config1()
    X = st["X"][:192].copy()
    r0a, tha = oracle.r0_theta0(X, st["Y"][:192], st["Z"][:192], mesh["nn"])
    X[5] = np.nextafter(X[5], np.float32(np.inf), dtype=np.float32)
    r0b, thb = oracle.r0_theta0(X, st["Y"][:192], st["Z"][:192], mesh["nn"])
    assert not (np.array_equal(_bits(r0a), _bits(r0b)) and np.array_equal(_bits(tha), _bits(thb)))
