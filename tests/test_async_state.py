"""Asynchronous frame read-back (cs3d_get_state_async / cs3d_wait_state):
the copy of a frame overlaps the next steps and lands bit-identical to the
synchronous read of the same step, through both staging slots and their
reuse; the drop-in driver writes its trajectory this way (tests/test_cli.py
checks that trajectory against a library run)."""
import numpy as np
import pytest

import cellsim3d_b200 as cs
from cellsim3d_b200 import workloads as W

from parity import topo_for

pytestmark = pytest.mark.gpu

KEYS = ("X", "Y", "Z", "VX", "VY", "VZ")


def _pinned(cap):
    import torch
    out = {k: torch.empty(cap * 192, dtype=torch.float32).pin_memory().numpy() for k in KEYS}
    out["pressure"] = torch.empty(cap, dtype=torch.float32).pin_memory().numpy()
    out["youngs"] = torch.empty(cap, dtype=torch.float32).pin_memory().numpy()
    for a in out.values():
        a[:] = np.nan
    return out


def test_async_frames_equal_synchronous_reads(mesh):
    p, st, _ = W.config1()
    topo, _ = topo_for(st, mesh)
    cap = 256
    sim = cs.Simulation(p, topo, cap)
    sim.load_state(st["X"], st["Y"], st["Z"], n_cells=st["n"])
    bufs = [_pinned(cap), _pinned(cap)]
    for frame in range(5):
        slot = frame % 2
        sim.step(7)
        ref = sim.state()
        n = sim.state_async(0, slot, bufs[slot])
        assert n == ref["n"]
        sim.step(3)            # overlaps the copy
        sim.wait_state(slot)
        for k in KEYS:
            assert np.array_equal(bufs[slot][k][: n * 192].view(np.uint32), ref[k][: n * 192].view(np.uint32)), \
                (frame, k)
        for k in ("pressure", "youngs"):
            assert np.array_equal(bufs[slot][k][:n].view(np.uint32), ref[k][:n].view(np.uint32)), (frame, k)
    # a partial request: positions only, other buffers untouched
    part = _pinned(cap)
    n = sim.state_async(0, 0, {k: part[k] for k in ("X", "Y", "Z")})
    sim.wait_state(0)
    ref = sim.state()
    assert np.array_equal(part["X"][: n * 192].view(np.uint32), ref["X"][: n * 192].view(np.uint32))
    assert np.all(np.isnan(part["VX"]))
    # waiting on a slot with nothing pending returns at once
    sim.wait_state(1)
    sim.wait_state(1)
    sim.close()


def test_async_argument_checks(mesh):
    p, st, _ = W.config1()
    topo, _ = topo_for(st, mesh)
    sim = cs.Simulation(p, topo, 64)
    sim.load_state(st["X"], st["Y"], st["Z"], n_cells=st["n"])
    with pytest.raises(cs.CS3DError):
        sim.state_async(0, 2, {})
    with pytest.raises(cs.CS3DError):
        sim.wait_state(-1)
    sim.close()
