"""cellsim3d_b200 -- B200-native CellSim3D timestep.

Python mirror of the reference's host-side interface over the C ABI of
libcs3d.so (include/cs3d.h).  Names follow the reference where it has one:

  read_json_params   src/GPUbounce.cu:1914-2247  (inp.json with comments)
  read_fullerene_nn  src/GPUbounce.cu:1814-1911  (mesh files)
  initialize_C180s   src/GPUbounce.cu:1598-1774  (initial placement)
  Ranmar             src/marsaglia.h, src/RandomVector.h
  Simulation         the step loop of src/GPUbounce.cu:1055-1506 on the GPU
  Ensemble           many independent simulations stepped together

Arrays are float32 numpy arrays in the reference's layout: per-node arrays of
length n_cells*192 indexed cell*192 + node (slots 180..191 padding), per-cell
arrays of length n_cells.  The GPU path has no CPU fallback: if libcs3d.so is
missing every call raises.
"""
import ctypes as C

import numpy as np

from . import _lib
from ._lib import (CS3DError, Config, Mesh, Params, Rng, Topology, ERRBITS, SLOTS, NODES,
                   OPT_RECORD_PAIRS, OPT_SKIN, OPT_PAIR_CAPACITY, OPT_REBUILD, OPT_HALO_STATS)

__all__ = ["read_json_params", "config_to_params", "make_params", "read_fullerene_nn", "mesh_from_arrays",
           "build_topology", "Ranmar", "seed_map", "initialize_C180s", "Simulation", "Ensemble",
           "CS3DError", "Config", "Params", "Mesh", "Topology", "SLOTS", "NODES", "version"]


def _fp(a):
    return a.ctypes.data_as(C.POINTER(C.c_float)) if a is not None else None


def _ip(a):
    return a.ctypes.data_as(C.POINTER(C.c_int32)) if a is not None else None


def _f32(a, n=None):
    if a is None:
        return None
    a = np.ascontiguousarray(a, dtype=np.float32).reshape(-1)
    if n is not None and a.size < n:
        raise ValueError("array of %d elements, need %d" % (a.size, n))
    return a


def version():
    return _lib.lib().cs3d_version()


def read_json_params(path):
    """Parse inp.json (comments allowed) with the reference's validation."""
    cfg = Config()
    err = C.create_string_buffer(512)
    st = _lib.lib().cs3d_config_read_json(str(path).encode(), C.byref(cfg), err, 512)
    if st != 0:
        raise CS3DError("read_json_params: " + err.value.decode(errors="replace"), st)
    return cfg


def config_to_params(cfg):
    p = Params()
    _lib.check(_lib.lib().cs3d_config_to_params(C.byref(cfg), C.byref(p)), "config_to_params")
    return p


def make_params(d):
    """Params from a dict with the cs3d_params field names (see workloads.base_params)."""
    p = Params()
    for name, _t in Params._fields_:
        if name == "box_len":
            for k in range(3):
                p.box_len[k] = float(d["box_len"][k])
        elif name in d:
            setattr(p, name, d[name])
    return p


def read_fullerene_nn(directory="."):
    """Read C180, C180NN, C180C and C180_pentahexa from a directory."""
    m = Mesh()
    _lib.check(_lib.lib().cs3d_mesh_read(str(directory).encode(), C.byref(m)), "read_fullerene_nn")
    return m


def mesh_from_arrays(d):
    """Mesh from the arrays of workloads.load_mesh()."""
    m = Mesh()
    C.memmove(m.xyz, np.ascontiguousarray(d["xyz"], dtype=np.float32).ctypes.data, 540 * 4)
    C.memmove(m.nn, np.ascontiguousarray(d["nn"], dtype=np.int32).ctypes.data, 576 * 4)
    C.memmove(m.sign, np.ascontiguousarray(d["sign"], dtype=np.int32).ctypes.data, 180 * 4)
    C.memmove(m.bonds, np.ascontiguousarray(d["bonds"], dtype=np.int32).ctypes.data, 540 * 4)
    C.memmove(m.faces, np.ascontiguousarray(d["faces"], dtype=np.int32).ctypes.data, 644 * 4)
    return m


def build_topology(mesh, X, Y, Z):
    """Bond lengths and angles from cell 0's initial positions (host float)."""
    X, Y, Z = _f32(X, 192), _f32(Y, 192), _f32(Z, 192)
    t = Topology()
    _lib.check(_lib.lib().cs3d_topology_build(C.byref(mesh), _fp(X), _fp(Y), _fp(Z), C.byref(t)),
               "build_topology")
    return t


def seed_map(seed):
    ij, kl = C.c_int32(), C.c_int32()
    _lib.lib().cs3d_seed_map(int(seed), C.byref(ij), C.byref(kl))
    return ij.value, kl.value


class Ranmar:
    """RANMAR generator (rmarin / ranmar) and the Marsaglia sphere point."""

    def __init__(self, ij, kl):
        self.state = Rng()
        _lib.check(_lib.lib().cs3d_rng_init(C.byref(self.state), int(ij), int(kl)), "rmarin")

    def draw(self, n):
        out = np.zeros(n, dtype=np.float32)
        _lib.check(_lib.lib().cs3d_rng_draw(C.byref(self.state), _fp(out), n), "ranmar")
        return out

    def random_vector(self):
        out = np.zeros(3, dtype=np.float32)
        _lib.check(_lib.lib().cs3d_rng_random_vector(C.byref(self.state), _fp(out)), "GetRandomVector")
        return out


def initialize_C180s(cfg, mesh, n_cells, rng=None):
    """Initial placement as the reference (lattice or RANMAR random insertion)."""
    X = np.zeros(n_cells * 192, dtype=np.float32)
    Y = np.zeros_like(X)
    Z = np.zeros_like(X)
    st = _lib.lib().cs3d_init_positions(C.byref(cfg), C.byref(mesh), int(n_cells),
                                        C.byref(rng.state) if rng is not None else None, _fp(X), _fp(Y), _fp(Z))
    _lib.check(st, "initialize_C180s")
    return X, Y, Z


def initial_stiffness(cfg, X, Y, Z, n_cells, rng=None):
    """Bond stiffness of the initial cells (src/GPUbounce.cu:616-692): stiffness1,
    or stiffness2 for the softer cells the config selects."""
    out = np.zeros(max(n_cells, 1), dtype=np.float32)
    X, Y, Z = _f32(X), _f32(Y), _f32(Z)
    st = _lib.lib().cs3d_initial_stiffness(C.byref(cfg), int(n_cells), _fp(X), _fp(Y), _fp(Z),
                                           C.byref(rng.state) if rng is not None else None, _fp(out))
    _lib.check(st, "initial_stiffness")
    return out[:n_cells]


class Ensemble:
    """Independent simulations stepped together on one GPU.

    params: list of Params (or dicts), topo: Topology, capacities: list of int.
    """

    def __init__(self, params, topo, capacities, device=0, stream=None):
        L = _lib.lib()
        n = len(params)
        arr = (Params * n)()
        for k, p in enumerate(params):
            arr[k] = p if isinstance(p, Params) else make_params(p)
        caps = np.ascontiguousarray(capacities, dtype=np.int32)
        self._topo = topo
        self.h = C.c_void_p()
        st = L.cs3d_create_ensemble(n, arr, C.byref(topo), _ip(caps), int(device),
                                    C.c_void_p(stream) if stream else None, C.byref(self.h))
        _lib.check(st, "cs3d_create_ensemble")
        self.n_inst = n
        self._n0 = [0] * n
        self.capacities = caps.copy()

    # -- lifetime
    def close(self):
        if getattr(self, "h", None) and self.h.value:
            _lib.lib().cs3d_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # -- state in
    def load_state(self, inst, X, Y, Z, VX=None, VY=None, VZ=None, pressure=None, youngs=None, n_cells=None):
        n = int(n_cells if n_cells is not None else len(X) // 192)
        k = n * 192
        X, Y, Z = _f32(X, k), _f32(Y, k), _f32(Z, k)
        VX, VY, VZ = _f32(VX, k), _f32(VY, k), _f32(VZ, k)
        pressure, youngs = _f32(pressure, n), _f32(youngs, n)
        st = _lib.lib().cs3d_load_state(self.h, inst, n, _fp(X), _fp(Y), _fp(Z), _fp(VX), _fp(VY), _fp(VZ),
                                        _fp(pressure), _fp(youngs))
        _lib.check(st, "cs3d_load_state")
        self._n0[inst] = n

    def set_rng(self, inst, rng):
        _lib.check(_lib.lib().cs3d_set_rng(self.h, inst, C.byref(rng.state)), "cs3d_set_rng")

    def get_rng(self, inst=0):
        r = Ranmar.__new__(Ranmar)
        r.state = Rng()
        _lib.check(_lib.lib().cs3d_get_rng(self.h, inst, C.byref(r.state)), "cs3d_get_rng")
        return r

    def set_option(self, option, value):
        _lib.check(_lib.lib().cs3d_set_option(self.h, option, int(value)), "cs3d_set_option")

    def set_skin_schedule(self, min_cells=(), skins=()):
        """Neighbour-list skin by population range (cs3d_set_skin_schedule):
        an instance with at least min_cells[k] cells steps with skins[k];
        empty sequences clear the schedule.  Changes the time, not the
        results."""
        mc = np.ascontiguousarray(min_cells, dtype=np.int32)
        sk = np.ascontiguousarray(skins, dtype=np.float32)
        if mc.shape != sk.shape or mc.ndim != 1:
            raise ValueError("min_cells and skins must be 1-D sequences of one length")
        _lib.check(_lib.lib().cs3d_set_skin_schedule(self.h, int(mc.size), _ip(mc), _fp(sk)),
                   "cs3d_set_skin_schedule")

    # -- stepping
    def step(self, n=1, raise_on_error=True):
        st = _lib.lib().cs3d_step(self.h, int(n))
        if st != 0 and raise_on_error:
            raise CS3DError("cs3d_step", st, self.last_error(-1))
        return st

    def profile_step(self, n_steps=3):
        """Average device time (ms) of each launch of a step, by kernel name."""
        ms = (C.c_float * 64)()
        names = C.create_string_buffer(2048)
        nk = C.c_int32()
        st = _lib.lib().cs3d_profile_step(self.h, int(n_steps), ms, names, 2048, 64, C.byref(nk))
        if st != 0:
            raise CS3DError("cs3d_profile_step", st, self.last_error(-1))
        return list(zip(names.value.decode().split(","), [ms[k] for k in range(nk.value)]))

    def last_step_ms(self):
        v = C.c_float()
        _lib.lib().cs3d_last_step_ms(self.h, C.byref(v))
        return v.value

    # -- state out
    def n_cells(self, inst=0):
        n = C.c_int32()
        _lib.check(_lib.lib().cs3d_get_state(self.h, inst, C.byref(n), *([None] * 8)), "cs3d_get_state")
        return n.value

    def state(self, inst=0, out=None):
        """Positions, velocities (192-stride SoA), pressures and stiffnesses.
        out: optional dict of preallocated float32 arrays (e.g. pinned host
        memory) with room for the current cells, filled in place."""
        n = self.n_cells(inst)
        k = n * 192
        if out is not None:
            a = dict(out)
            for key in ("X", "Y", "Z", "VX", "VY", "VZ"):
                if a[key].dtype != np.float32 or not a[key].flags.c_contiguous or a[key].size < k:
                    raise ValueError("out[%s]: contiguous float32 with room for %d values needed" % (key, k))
            for key in ("pressure", "youngs"):
                if key not in a or a[key].size < n:
                    a[key] = np.zeros(n, dtype=np.float32)
        else:
            a = {key: np.zeros(k, dtype=np.float32) for key in ("X", "Y", "Z", "VX", "VY", "VZ")}
            a["pressure"] = np.zeros(n, dtype=np.float32)
            a["youngs"] = np.zeros(n, dtype=np.float32)
        nn = C.c_int32()
        st = _lib.lib().cs3d_get_state(self.h, inst, C.byref(nn), _fp(a["X"]), _fp(a["Y"]), _fp(a["Z"]),
                                       _fp(a["VX"]), _fp(a["VY"]), _fp(a["VZ"]), _fp(a["pressure"]),
                                       _fp(a["youngs"]))
        _lib.check(st, "cs3d_get_state")
        a["n"] = n
        return a

    def state_async(self, inst, slot, out):
        """Start reading instance inst back into `out` (a dict of float32
        arrays X, Y, Z, VX, VY, VZ with room for the capacity and pressure,
        youngs per cell; any key may be missing) without waiting: the copy
        overlaps the next steps.  Returns the cell count; the arrays are valid
        after wait_state(slot).  Page-locked arrays (torch pin_memory, or
        cs3d_host_alloc) make the copy asynchronous."""
        n = C.c_int32()
        get = lambda k: _fp(out[k]) if k in out else None
        st = _lib.lib().cs3d_get_state_async(self.h, inst, int(slot), C.byref(n), get("X"), get("Y"), get("Z"),
                                             get("VX"), get("VY"), get("VZ"), get("pressure"), get("youngs"))
        _lib.check(st, "cs3d_get_state_async")
        return n.value

    def wait_state(self, slot):
        _lib.check(_lib.lib().cs3d_wait_state(self.h, int(slot)), "cs3d_wait_state")

    def forces(self, inst=0):
        n = self.n_cells(inst)
        k = n * 192
        a = {key: np.zeros(k, dtype=np.float32) for key in ("FCX", "FCY", "FCZ", "FDX", "FDY", "FDZ")}
        st = _lib.lib().cs3d_get_forces(self.h, inst, *[_fp(a[q]) for q in ("FCX", "FCY", "FCZ", "FDX", "FDY", "FDZ")])
        _lib.check(st, "cs3d_get_forces")
        return a

    def random_force(self, inst=0):
        """Langevin random force of the last step (192-stride SoA)."""
        n = self.n_cells(inst)
        a = {key: np.zeros(n * 192, dtype=np.float32) for key in ("FRX", "FRY", "FRZ")}
        _lib.check(_lib.lib().cs3d_get_random_force(self.h, inst, _fp(a["FRX"]), _fp(a["FRY"]), _fp(a["FRZ"])),
                   "cs3d_get_random_force")
        return a

    def cells(self, inst=0):
        n = self.n_cells(inst)
        cm = np.zeros(3 * n, dtype=np.float32)
        vol = np.zeros(n, dtype=np.float32)
        area = np.zeros(n, dtype=np.float32)
        bb = np.zeros(6 * n, dtype=np.float32)
        _lib.check(_lib.lib().cs3d_get_cells(self.h, inst, _fp(cm), _fp(vol), _fp(area), _fp(bb)), "cs3d_get_cells")
        return {"cm": cm.reshape(n, 3), "volume": vol, "area": area, "aabb": bb.reshape(n, 6)}

    def grid(self, inst=0):
        mm = np.zeros(6, dtype=np.float32)
        dv = np.zeros(3, dtype=np.int32)
        _lib.check(_lib.lib().cs3d_get_grid(self.h, inst, _fp(mm), _ip(dv)), "cs3d_get_grid")
        return mm, dv

    def pairs(self, kind, inst=0):
        cnt = C.c_longlong()
        L = _lib.lib()
        _lib.check(L.cs3d_get_pairs(self.h, inst, kind, None, 0, C.byref(cnt)), "cs3d_get_pairs")
        out = np.zeros((max(cnt.value, 1), 4), dtype=np.int32)
        _lib.check(L.cs3d_get_pairs(self.h, inst, kind, _ip(out), cnt.value, C.byref(cnt)), "cs3d_get_pairs")
        return out[:cnt.value]

    def events(self, inst=0):
        cnt = C.c_int32()
        L = _lib.lib()
        _lib.check(L.cs3d_get_events(self.h, inst, None, 0, C.byref(cnt)), "cs3d_get_events")
        out = np.zeros((max(cnt.value, 1), 3), dtype=np.int32)
        _lib.check(L.cs3d_get_events(self.h, inst, _ip(out), cnt.value, C.byref(cnt)), "cs3d_get_events")
        return out[:cnt.value]

    def far_counts(self, inst=0):
        """(step, cells) of the division steps whose far cells the internal-cells
        mitotic count left out."""
        cnt = C.c_int32()
        L = _lib.lib()
        _lib.check(L.cs3d_get_far_counts(self.h, inst, None, 0, C.byref(cnt)), "cs3d_get_far_counts")
        out = np.zeros((max(cnt.value, 1), 2), dtype=np.int32)
        _lib.check(L.cs3d_get_far_counts(self.h, inst, _ip(out), cnt.value, C.byref(cnt)), "cs3d_get_far_counts")
        return out[:cnt.value]

    def volume_histogram(self, inst=0, lo=0.0, hi=6.0, nbins=60, volumes=False):
        """Counts of the cells' volumes at the current positions, computed on the
        device: [below lo, nbins equal bins of [lo, hi), at or above hi]; with
        volumes=True also every cell's volume."""
        counts = np.zeros(nbins + 2, dtype=np.int64)
        n = self.n_cells(inst)
        vols = np.zeros(max(n, 1), dtype=np.float32) if volumes else None
        _lib.check(_lib.lib().cs3d_volume_histogram(self.h, inst, float(lo), float(hi), int(nbins),
                                                     counts.ctypes.data_as(C.POINTER(C.c_int64)),
                                                     _fp(vols) if volumes else None), "cs3d_volume_histogram")
        return (counts, vols[:n]) if volumes else counts

    def population(self, inst=0, steps=None, n0=None):
        """Cell count after every step 0..steps, from the division events
        (the curve scripts/pop.py draws from a trajectory)."""
        ev = self.events(inst)
        steps = int(self.stats()["steps"]) if steps is None else int(steps)
        n0 = self._n0[inst] if n0 is None else int(n0)
        born = np.bincount(ev[:, 0], minlength=steps + 1)[: steps + 1] if len(ev) else np.zeros(steps + 1, int)
        return n0 + np.cumsum(born)

    def last_error(self, inst=0):
        b = C.c_uint32()
        _lib.check(_lib.lib().cs3d_last_error(self.h, inst, C.byref(b)), "cs3d_last_error")
        return b.value

    def stats(self):
        s = (C.c_longlong * 8)()
        _lib.check(_lib.lib().cs3d_get_stats(self.h, s, 8), "cs3d_get_stats")
        return {"steps": s[0], "rebuilds": s[1], "max_entries": s[2], "max_cand": s[3], "launches_per_step": s[4],
                "max_halo": s[5], "lists_built": s[6], "rebuilds_div_rule": s[7]}


class Simulation(Ensemble):
    """One simulation (an ensemble of one instance)."""

    def __init__(self, params, topo, capacity, device=0, stream=None):
        super().__init__([params], topo, [capacity], device=device, stream=stream)

    def load_state(self, X, Y, Z, VX=None, VY=None, VZ=None, pressure=None, youngs=None, n_cells=None):
        super().load_state(0, X, Y, Z, VX, VY, VZ, pressure, youngs, n_cells)

    def set_rng(self, rng):
        super().set_rng(0, rng)
