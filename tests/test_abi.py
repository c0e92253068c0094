"""The C-ABI library loads without a GPU and exports every entry point that
include/cs3d.h declares; host-only entry points work on the CPU."""
import ctypes as C
import os
import re

import pytest

import cellsim3d_b200 as cs
from cellsim3d_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared():
    txt = open(os.path.join(ROOT, "include", "cs3d.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(cs3d_[a-z0-9_]+)\s*\(", txt)))


def test_every_declared_symbol_is_exported():
    L = C.CDLL(_lib.LIB_PATH)
    names = declared()
    assert len(names) >= 30
    for n in names:
        assert hasattr(L, n), n
    assert sorted(_lib.EXPORTS) == names


def test_strerror_and_version():
    assert cs.version() >= 10000
    assert _lib.lib().cs3d_strerror(-69) == b"population exceeded the allocated capacity"


def test_create_without_gpu_fails_cleanly(mesh):
    import torch
    if torch.cuda.is_available():
        pytest.skip("GPU present")
    from cellsim3d_b200 import workloads as W
    p, st, _ = W.config1()
    topo = cs.build_topology(cs.mesh_from_arrays(mesh), st["X"][:192], st["Y"][:192], st["Z"][:192])
    with pytest.raises(cs.CS3DError):
        cs.Simulation(p, topo, 64)
