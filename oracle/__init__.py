"""TEST INFRASTRUCTURE ONLY: ctypes wrapper of the FP64 CPU oracle.

The oracle (oracle/cs3d_oracle.c) restates CellSim3D's per-timestep loop on
the CPU (FP64 force values, float state and float decisions).  It is the
checker for the CUDA path; only tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline leg may import it.  Nothing in cellsim3d_b200 uses it.
"""
import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = os.path.join(_HERE, "liboracle.so")
_lib = None


class OrcParams(C.Structure):
    _fields_ = [(n, C.c_float) for n in (
        "mass", "rep_range", "att_range", "rep_strength", "att_strength", "youngs_mod",
        "stiffness1", "gamma_int", "gamma_ext", "gamma_o", "div_vol", "dt", "max_p", "min_p",
        "growth_rate", "thresh_dist")] + [("box", C.c_float * 3)] + [(n, C.c_int) for n in (
        "check_sphericity", "constrain_angles", "use_rigid_box", "daught_same_stiffness",
        "div_time_steps", "pad_", "add_rands")] + [("rand_scale", C.c_float), ("rand_seed", C.c_uint),
                                                   ("correct_com", C.c_int)] + [
        ("diff_stiff", C.c_int), ("stiffness2", C.c_float), ("phase_count", C.c_int),
        ("soften_after_growth", C.c_int), ("soft_n", C.c_int), ("soft_frac", C.c_float), ("soft_rand", C.c_int),
        ("closeness", C.c_float), ("far_r", C.c_float)]


class OrcTopo(C.Structure):
    _fields_ = [("nn", C.c_int * 576), ("sign", C.c_int * 180), ("r0", C.c_float * 576),
                ("theta0", C.c_float * 576), ("faces", C.c_int * 644)]


class OrcRanmar(C.Structure):
    _fields_ = [("u", C.c_float * 98), ("c", C.c_float), ("cd", C.c_float), ("cm", C.c_float),
                ("i97", C.c_int), ("j97", C.c_int), ("ok", C.c_int)]


def build():
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB):
            build()
        L = C.CDLL(_LIB)
        P = C.c_void_p
        L.orc_create.restype = P
        L.orc_create.argtypes = [C.c_int, C.POINTER(OrcParams), C.POINTER(OrcTopo)]
        L.orc_destroy.argtypes = [P]
        L.orc_ptr_f.restype = C.POINTER(C.c_float)
        L.orc_ptr_f.argtypes = [P, C.c_int]
        L.orc_ptr_d.restype = C.POINTER(C.c_double)
        L.orc_ptr_d.argtypes = [P, C.c_int]
        L.orc_ptr_i.restype = C.POINTER(C.c_int)
        L.orc_ptr_i.argtypes = [P, C.c_int]
        L.orc_err.restype = C.c_uint
        L.orc_err.argtypes = [P]
        L.orc_rng.restype = C.POINTER(OrcRanmar)
        L.orc_rng.argtypes = [P]
        for fn in ("orc_init", "orc_center_of_mass", "orc_build_grid", "orc_con_force",
                   "orc_dis_force", "orc_volumes", "orc_step", "orc_rebuild_bins"):
            getattr(L, fn).argtypes = [P]
        L.orc_run.argtypes = [P, C.c_int]
        L.orc_pairs.restype = C.c_long
        L.orc_pairs.argtypes = [P, C.c_int, C.POINTER(C.c_int), C.c_long]
        L.orc_set_record.argtypes = [P, C.c_int]
        L.orc_recorded_pairs.restype = C.c_long
        L.orc_recorded_pairs.argtypes = [P, C.c_int, C.POINTER(C.c_int), C.c_long]
        L.orc_accepted.restype = C.c_long
        L.orc_accepted.argtypes = [P, C.POINTER(C.c_int), C.c_long]
        L.orc_max_local_nn.restype = C.c_int
        L.orc_max_local_nn.argtypes = [P]
        L.orc_forces_subset.argtypes = [P, C.POINTER(C.c_int), C.c_int]
        L.orc_rmarin.restype = C.c_int
        L.orc_rmarin.argtypes = [C.POINTER(OrcRanmar), C.c_int, C.c_int]
        L.orc_ranmar_draw.argtypes = [C.POINTER(OrcRanmar), C.POINTER(C.c_float), C.c_int]
        L.orc_random_vector.argtypes = [C.POINTER(OrcRanmar), C.POINTER(C.c_float)]
        L.orc_seed_map.argtypes = [C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int)]
        L.orc_random_force.argtypes = [C.POINTER(OrcParams), C.c_int, C.c_int, C.POINTER(C.c_float)]
        L.orc_initial_stiffness.restype = C.c_int
        L.orc_initial_stiffness.argtypes = [C.POINTER(OrcParams), C.c_int, C.c_int] + [C.POINTER(C.c_float)] * 3 + [
            C.POINTER(OrcRanmar), C.POINTER(C.c_float)]
        L.orc_r0_theta0.argtypes = [C.POINTER(C.c_float)] * 3 + [C.POINTER(C.c_int),
                                                                 C.POINTER(C.c_float), C.POINTER(C.c_float)]
        L.orc_divide_cell.restype = C.c_int
        L.orc_divide_cell.argtypes = [P, C.c_int, C.POINTER(C.c_float)]
        L.orc_sizeof_params.restype = C.c_int
        L.orc_sizeof_topo.restype = C.c_int
        assert L.orc_sizeof_params() == C.sizeof(OrcParams)
        assert L.orc_sizeof_topo() == C.sizeof(OrcTopo)
        _lib = L
    return _lib


def _fp(a):
    return a.ctypes.data_as(C.POINTER(C.c_float))


def _ip(a):
    return a.ctypes.data_as(C.POINTER(C.c_int))


class Ranmar:
    """RANMAR (src/marsaglia.h:54-144), float, bit-exact."""

    def __init__(self, ij, kl):
        self.st = OrcRanmar()
        if lib().orc_rmarin(C.byref(self.st), ij, kl) != 0:
            raise ValueError("seed out of range")

    def draw(self, n):
        out = np.zeros(n, dtype=np.float32)
        lib().orc_ranmar_draw(C.byref(self.st), _fp(out), n)
        return out

    def random_vector(self):
        out = np.zeros(3, dtype=np.float32)
        lib().orc_random_vector(C.byref(self.st), _fp(out))
        return out


def seed_map(seed):
    ij, kl = C.c_int(), C.c_int()
    lib().orc_seed_map(seed, C.byref(ij), C.byref(kl))
    return ij.value, kl.value


def r0_theta0(X, Y, Z, nn):
    X = np.ascontiguousarray(X, dtype=np.float32)
    Y = np.ascontiguousarray(Y, dtype=np.float32)
    Z = np.ascontiguousarray(Z, dtype=np.float32)
    nn = np.ascontiguousarray(nn, dtype=np.int32).reshape(-1)
    r0 = np.zeros(576, dtype=np.float32)
    th = np.zeros(576, dtype=np.float32)
    lib().orc_r0_theta0(_fp(X), _fp(Y), _fp(Z), _ip(nn), _fp(r0), _fp(th))
    return r0, th


def make_params(p):
    """OrcParams from a dict of cs3d_params-like fields."""
    o = OrcParams()
    o.mass = p["particle_mass"]
    o.rep_range = p["repulsion_range"]
    o.att_range = p["attraction_range"]
    o.rep_strength = p["repulsion_strength"]
    o.att_strength = p["attraction_strength"]
    o.youngs_mod = p["youngs_mod"]
    o.stiffness1 = p["stiffness1"]
    o.gamma_int = p["internal_damping"]
    o.gamma_ext = p["viscotic_damping"]
    o.gamma_o = p["gamma_visc"]
    o.div_vol = p["division_vol"]
    o.dt = p["time_interval"]
    o.max_p = p["max_pressure"]
    o.min_p = p["min_pressure"]
    o.growth_rate = p["growth_rate"]
    o.thresh_dist = p["thresh_dist"]
    for k in range(3):
        o.box[k] = p["box_len"][k]
    o.check_sphericity = int(p["check_sphericity"])
    o.constrain_angles = int(p["constrain_angles"])
    o.use_rigid_box = int(p["use_rigid_box"])
    o.daught_same_stiffness = int(p["daught_same_stiffness"])
    o.div_time_steps = int(p["div_time_steps"])
    o.add_rands = int(p.get("add_rands", 0))
    o.rand_scale = float(p.get("rand_scale_factor", 0.0))
    o.rand_seed = int(p.get("rand_seed", 0)) & 0xffffffff
    o.correct_com = int(p.get("correct_com", 0))
    o.diff_stiff = int(p.get("use_different_stiffnesses", 0))
    o.stiffness2 = float(p.get("stiffness2", 0.0))
    o.phase_count = int(p.get("phase_count", 0))
    o.soften_after_growth = int(p.get("soften_after_growth", 0))
    o.soft_n = int(p.get("number_of_softer_cells", 0))
    o.soft_frac = float(p.get("fraction_of_softer_cells", 0.0))
    o.soft_rand = int(p.get("choose_random_cell_indices", 0))
    o.closeness = float(p.get("closeness_to_center", 0.0))
    o.far_r = float(p.get("count_internal_radius", 0.0))
    return o


def initial_stiffness(params, rigid, X, Y, Z, n, rng=None):
    """The oracle's initial bond stiffness of n cells (None when more softer
    cells than cells are asked for)."""
    P = make_params(params) if isinstance(params, dict) else params
    E = np.zeros(max(n, 1), dtype=np.float32)
    X = np.ascontiguousarray(X, dtype=np.float32)
    Y = np.ascontiguousarray(Y, dtype=np.float32)
    Z = np.ascontiguousarray(Z, dtype=np.float32)
    r = rng if rng is not None else OrcRanmar()
    rc = lib().orc_initial_stiffness(C.byref(P), int(rigid), int(n), _fp(X), _fp(Y), _fp(Z), C.byref(r), _fp(E))
    return None if rc else E[:n]


def random_force(params, node, step):
    """The oracle's Langevin random force of one node and step (3 floats)."""
    P = make_params(params) if isinstance(params, dict) else params
    out = np.zeros(3, dtype=np.float32)
    lib().orc_random_force(C.byref(P), int(node), int(step), _fp(out))
    return out


def make_topo(nn, sign, r0, theta0, faces):
    t = OrcTopo()
    C.memmove(t.nn, np.ascontiguousarray(nn, dtype=np.int32).ctypes.data, 576 * 4)
    C.memmove(t.sign, np.ascontiguousarray(sign, dtype=np.int32).ctypes.data, 180 * 4)
    C.memmove(t.r0, np.ascontiguousarray(r0, dtype=np.float32).ctypes.data, 576 * 4)
    C.memmove(t.theta0, np.ascontiguousarray(theta0, dtype=np.float32).ctypes.data, 576 * 4)
    C.memmove(t.faces, np.ascontiguousarray(faces, dtype=np.int32).ctypes.data, 644 * 4)
    return t


class System:
    """One simulation in the oracle.  Arrays are numpy views of oracle memory."""

    def __init__(self, capacity, params, topo):
        self._p = make_params(params) if isinstance(params, dict) else params
        self._t = topo
        self.h = lib().orc_create(capacity, C.byref(self._p), C.byref(self._t))
        if not self.h:
            raise MemoryError("oracle allocation failed")
        self.cap = capacity
        L = lib()
        nn = capacity * 192

        def fv(w, n):
            return np.ctypeslib.as_array(L.orc_ptr_f(self.h, w), shape=(n,))

        self.X, self.Y, self.Z = fv(0, nn), fv(1, nn), fv(2, nn)
        self.VX, self.VY, self.VZ = fv(3, nn), fv(4, nn), fv(5, nn)
        self.CM = fv(6, 3 * capacity).reshape(3, capacity)
        self.press, self.E = fv(7, capacity), fv(8, capacity)
        self.vol, self.area = fv(9, capacity), fv(10, capacity)
        self.aabb = fv(11, 6 * capacity).reshape(capacity, 6)
        self.minmax = fv(12, 6)
        self.FR = fv(13, 3 * nn).reshape(3, nn)
        self.FC = np.ctypeslib.as_array(L.orc_ptr_d(self.h, 0), shape=(3, nn))
        self.FD = np.ctypeslib.as_array(L.orc_ptr_d(self.h, 1), shape=(3, nn))
        self._n = np.ctypeslib.as_array(L.orc_ptr_i(self.h, 0), shape=(1,))
        self._step = np.ctypeslib.as_array(L.orc_ptr_i(self.h, 1), shape=(1,))
        self._div = np.ctypeslib.as_array(L.orc_ptr_i(self.h, 2), shape=(3,))
        self._nev = np.ctypeslib.as_array(L.orc_ptr_i(self.h, 3), shape=(1,))
        self._ev = L.orc_ptr_i(self.h, 4)
        self._nfar = np.ctypeslib.as_array(L.orc_ptr_i(self.h, 9), shape=(1,))
        self._far = L.orc_ptr_i(self.h, 10)
        self.syscm = fv(14, 3)

    def close(self):
        if self.h:
            lib().orc_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def n(self):
        return int(self._n[0])

    @property
    def step_count(self):
        return int(self._step[0])

    @property
    def divs(self):
        return tuple(int(v) for v in self._div)

    def load(self, X, Y, Z, VX=None, VY=None, VZ=None, pressure=None, youngs=None, n=None):
        n = n if n is not None else len(X) // 192
        k = n * 192
        self.X[:] = 0; self.Y[:] = 0; self.Z[:] = 0
        self.VX[:] = 0; self.VY[:] = 0; self.VZ[:] = 0
        self.X[:k] = X[:k]; self.Y[:k] = Y[:k]; self.Z[:k] = Z[:k]
        if VX is not None:
            self.VX[:k] = VX[:k]; self.VY[:k] = VY[:k]; self.VZ[:k] = VZ[:k]
        self.press[:] = 0
        self.press[:n] = pressure[:n] if pressure is not None else self._p.min_p
        self.E[:] = 0
        self.E[:n] = youngs[:n] if youngs is not None else self._p.stiffness1
        self.CM[:] = 0
        self.FC[:] = 0
        self.FD[:] = 0
        self._n[0] = n

    def set_step(self, step):
        self._step[0] = int(step)

    def load_forces(self, FCX, FCY, FCZ, FDX, FDY, FDZ):
        """Forces of the previous evaluation (float arrays from the CUDA path)."""
        n = len(FCX)
        for q, a in enumerate((FCX, FCY, FCZ)):
            self.FC[q, :n] = a
        for q, a in enumerate((FDX, FDY, FDZ)):
            self.FD[q, :n] = a

    def load_cm(self, cm):
        """Per-cell centres of mass (n, 3) as the stale values of the next step."""
        n = len(cm)
        self.CM[:, :n] = np.asarray(cm, dtype=np.float32).T

    def seed(self, ij, kl):
        if lib().orc_rmarin(lib().orc_rng(self.h), ij, kl) != 0:
            raise ValueError("seed out of range")

    def set_rng(self, st):
        C.memmove(lib().orc_rng(self.h), C.byref(st), C.sizeof(OrcRanmar))

    def init(self):
        lib().orc_init(self.h)

    def step(self, n=1):
        lib().orc_run(self.h, n)

    def err(self):
        return int(lib().orc_err(self.h))

    def events(self):
        ne = int(self._nev[0])
        return np.ctypeslib.as_array(self._ev, shape=(3 * max(ne, 1),))[:3 * ne].reshape(ne, 3).copy()

    def far_counts(self):
        """(step, cells) of num_cells_far at the division steps where it left cells out."""
        nf = int(self._nfar[0])
        return np.ctypeslib.as_array(self._far, shape=(2 * max(nf, 1),))[:2 * nf].reshape(nf, 2).copy()

    def pairs(self, kind):
        cnt = lib().orc_pairs(self.h, kind, None, 0)
        out = np.zeros((max(cnt, 1), 4), dtype=np.int32)
        lib().orc_pairs(self.h, kind, _ip(out), cnt)
        return out[:cnt]

    def set_record(self, on=True):
        lib().orc_set_record(self.h, int(on))

    def recorded_pairs(self, kind):
        """Pairs used by the last force evaluation (set_record(True) first)."""
        cnt = lib().orc_recorded_pairs(self.h, kind, None, 0)
        out = np.zeros((max(cnt, 1), 4), dtype=np.int32)
        lib().orc_recorded_pairs(self.h, kind, _ip(out), cnt)
        return out[:cnt]

    def bins(self):
        """The oracle's current grid bins (makeNNlist, src/propagatebound.cu:209-263):
        a list of int arrays, the cells of each bin in ascending order."""
        L = lib()
        nb = L.orc_ptr_i(self.h, 13)[0]
        start = np.ctypeslib.as_array(L.orc_ptr_i(self.h, 11), shape=(nb + 1,)).copy()
        total = int(start[nb])
        cells = np.ctypeslib.as_array(L.orc_ptr_i(self.h, 12), shape=(max(total, 1),))[:total].copy()
        return [cells[start[b]:start[b + 1]] for b in range(nb)]

    def accepted(self):
        """(cell, node, accepted cell) triples of every node with the current
        stale grid (src/propagate.cu:356-404)."""
        cnt = lib().orc_accepted(self.h, None, 0)
        out = np.zeros((max(cnt, 1), 3), dtype=np.int32)
        lib().orc_accepted(self.h, _ip(out), cnt)
        return out[:cnt]

    def max_local_nn(self):
        return int(lib().orc_max_local_nn(self.h))

    def forces_subset(self, cells):
        cells = np.ascontiguousarray(cells, dtype=np.int32)
        lib().orc_forces_subset(self.h, _ip(cells), len(cells))

    def compute_grid(self):
        lib().orc_build_grid(self.h)

    def load_grid(self, aabb, minmax):
        """Boxes (n, 6) and grid extents (6) of a handed-over state; bins rebuilt."""
        n = self.n
        self.aabb[:n] = np.asarray(aabb, dtype=np.float32).reshape(n, 6)
        self.minmax[:] = np.asarray(minmax, dtype=np.float32).reshape(6)
        lib().orc_rebuild_bins(self.h)

    def compute_cm(self):
        lib().orc_center_of_mass(self.h)

    def compute_volumes(self):
        """Centres of mass and volumes (src/volume.cu:5-163) of the current positions."""
        lib().orc_center_of_mass(self.h)
        lib().orc_volumes(self.h)
        return self.vol[: self.n].copy()


def _attach_force_methods():
    def con_force(self):
        """Conservative force at the current state with the current grid."""
        lib().orc_con_force(self.h)

    def dis_force(self):
        """Dissipative force at the current state with the current grid."""
        lib().orc_dis_force(self.h)

    def set_rng_from(self, rng_struct):
        """RANMAR state from a cs3d_rng-layout ctypes structure."""
        C.memmove(lib().orc_rng(self.h), C.byref(rng_struct), C.sizeof(OrcRanmar))

    System.con_force = con_force
    System.dis_force = dis_force
    System.set_rng_from = set_rng_from


_attach_force_methods()
