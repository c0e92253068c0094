"""Runner of oracle/_ref/cs3d_ref: the reference CellSim3D CUDA kernels,
compiled unmodified from the reference sources by oracle/ref.mk and driven
through the reference's timestep by oracle/ref_harness.cu.

TEST AND BASELINE INFRASTRUCTURE ONLY: the parity tests use it to pin the
restatement against the reference's own arithmetic, and the benchmark uses it
to time the reference on the same GPU.  Nothing in the product imports it.

Nothing here loads libcs3d.so or imports cellsim3d_b200: the parameter
struct and the mesh tables are packed by the ctypes structures below (the
layouts of cs3d_params and cs3d_topology in include/cs3d.h; the harness checks
both sizes), and the equilibrium bond lengths and angles are computed by the
harness itself from cell 0 of the input positions, as the reference's set-up
does (src/GPUbounce.cu:1890-1908, :909-935).

File formats (little-endian):
  input   "CS3DREF2", int32 sizeof(cs3d_params), sizeof(cs3d_topology),
          cs3d_params, cs3d_topology (include/cs3d.h; its r0 and theta0 are
          zero here and are replaced by the harness's own),
          int32 n, capacity, steps, flags (bit 0: dump the initial forces),
          warmup (steps before the timed region),
          float32 X, Y, Z, VX, VY, VZ [n*192], pressure [n], youngs [n]
  output  "CS3DREFO", int32 status, steps_done, n, n_events, max_bin, max_nn,
          float32 total_ms, guard_ms (timed region), int32 events [n_events*3] (step, parent,
          daughter), float32 X, Y, Z, VX, VY, VZ, FCX..FCZ, FDX..FDZ [n*192],
          pressure [n], stiffness [n], CM x, y, z [n], int32 n_init, n_first, float32 initial
          FCX..FCZ, FDX..FDZ [n_init*192] when requested, float32 FRX..FRZ [n*192]
          (random force of the last step), int32 n_far, (step, cells) [n_far] of
          the internal-cells count, int32 n_mark, (int32 step, int32 cells, float32 ms)
          [n_mark]: colony mode (flags bit 1), the device time (guards excluded) at the
          first step with at least 10, 100, 1000 and 4096 cells; the run ends at 4096;
          int32 n_grid, then when n_grid > 0 (flags bit 2) the reference's grid after
          its first makeNNlist: float32 Minx[6], int32 Xdiv, Ydiv, Zdiv, nbins,
          counts [nbins], lists [32*nbins], float32 bounding boxes [6*n_grid].
"""
import os
import struct
import subprocess
import tempfile

import ctypes as C

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
BIN = os.path.join(HERE, "_ref", "cs3d_ref")
_DEPS = [os.path.join(HERE, "ref_harness.cu"), os.path.join(HERE, "..", "include", "cs3d.h")]

STATUS = {0: "ok", 1: "a grid bin held more than 32 cells (clamped)",
          2: "more than 10 cells passed the box filter for a node (bin cut)",
          3: "NaN position", 4: "division past capacity", 5: "grid larger than the reference's buffers",
          6: "more distinct softer cells requested than exist"}


_f, _i = C.c_float, C.c_int32


class RefParams(C.Structure):
    """cs3d_params (include/cs3d.h), field for field."""
    _fields_ = [(n, _f) for n in (
        "particle_mass", "repulsion_range", "attraction_range", "repulsion_strength",
        "attraction_strength", "youngs_mod", "stiffness1", "internal_damping", "viscotic_damping",
        "gamma_visc", "division_vol", "time_interval", "max_pressure", "min_pressure",
        "growth_rate", "thresh_dist")] + [("box_len", _f * 3)] + [(n, _i) for n in (
        "check_sphericity", "constrain_angles", "use_rigid_box", "daught_same_stiffness",
        "div_time_steps", "rng_ij", "rng_kl", "add_rands")] + [
        ("rand_scale_factor", _f), ("rand_seed", _i), ("correct_com", _i),
        ("use_different_stiffnesses", _i), ("stiffness2", _f), ("phase_count", _i),
        ("soften_after_growth", _i), ("number_of_softer_cells", _i), ("fraction_of_softer_cells", _f),
        ("choose_random_cell_indices", _i), ("closeness_to_center", _f), ("count_internal_radius", _f)]


class RefTopology(C.Structure):
    """cs3d_topology (include/cs3d.h)."""
    _fields_ = [("nn", _i * 576), ("sign", _i * 180), ("r0", _f * 576), ("theta0", _f * 576),
                ("faces", _i * 644)]


def pack_params(p):
    """RefParams from a dict of cs3d_params field names (missing fields 0)."""
    out = RefParams()
    for name, _t in RefParams._fields_:
        if name == "box_len":
            for k in range(3):
                out.box_len[k] = float(p["box_len"][k])
        elif name in p:
            setattr(out, name, p[name])
    return out


def pack_mesh(mesh):
    """RefTopology holding the mesh connectivity (neighbours, signs, faces)."""
    t = RefTopology()
    C.memmove(t.nn, np.ascontiguousarray(mesh["nn"], dtype=np.int32).ctypes.data, 576 * 4)
    C.memmove(t.sign, np.ascontiguousarray(mesh["sign"], dtype=np.int32).ctypes.data, 180 * 4)
    C.memmove(t.faces, np.ascontiguousarray(mesh["faces"], dtype=np.int32).ctypes.data, 644 * 4)
    return t


def available():
    """The harness is built and not older than its sources (a stale build
    would read a different parameter layout; it rejects such input)."""
    if not os.path.exists(BIN):
        return False
    t = os.path.getmtime(BIN)
    return all(not os.path.exists(dep) or os.path.getmtime(dep) <= t for dep in _DEPS)


def build(ref_root):
    """Compile oracle/_ref/cs3d_ref with oracle/ref.mk from the reference
    sources under `ref_root` (the CellSim3D checkout)."""
    subprocess.run(["make", "-s", "-f", os.path.join(HERE, "ref.mk"), "REF=" + ref_root, "-j8"], check=True)


def _f32(a, n):
    a = np.ascontiguousarray(np.asarray(a, dtype=np.float32).ravel()[:n])
    if a.size != n:
        raise ValueError("array of %d values, %d needed" % (a.size, n))
    return a


def _write_input(path, params, topo, state, capacity, steps, flags, warmup):
    n = int(state["n"])
    k = n * 192
    zeros = np.zeros(k, np.float32)
    press = state.get("pressure")
    if press is None:
        press = np.full(n, params.min_pressure, np.float32)
    youngs = state.get("youngs")
    if youngs is None:
        youngs = np.full(n, params.stiffness1, np.float32)
    with open(path, "wb") as f:
        f.write(b"CS3DREF2")
        f.write(struct.pack("<2i", C.sizeof(params), C.sizeof(topo)))
        f.write(bytes(params))
        f.write(bytes(topo))
        f.write(struct.pack("<5i", n, int(capacity), int(steps), int(flags), int(warmup)))
        for key in ("X", "Y", "Z", "VX", "VY", "VZ"):
            a = state.get(key)
            f.write((_f32(a, k) if a is not None else zeros).tobytes())
        f.write(_f32(press, n).tobytes())
        f.write(_f32(youngs, n).tobytes())


def tables(params, mesh, state, timeout=120):
    """The reference's equilibrium bond lengths and angles (float32 r0[576],
    theta0[576] in the cs3d_topology layout), computed by the harness from
    cell 0 of `state` with the reference's own host arithmetic.  Makes no CUDA
    call, so it runs without a GPU."""
    if not available():
        raise FileNotFoundError(BIN + " not built (make -f oracle/ref.mk)")
    P = params if isinstance(params, RefParams) else pack_params(params)
    with tempfile.TemporaryDirectory() as tmp:
        fin, fout = os.path.join(tmp, "in.bin"), os.path.join(tmp, "out.bin")
        _write_input(fin, P, pack_mesh(mesh), state, max(int(state["n"]), 1), 0, 0, 0)
        p = subprocess.run([BIN, "--tables", fin, fout], capture_output=True, text=True, timeout=timeout)
        if p.returncode != 0:
            raise RuntimeError("cs3d_ref --tables failed (%d): %s" % (p.returncode, p.stderr[-2000:]))
        with open(fout, "rb") as f:
            buf = f.read()
    if buf[:8] != b"CS3DREFT" or len(buf) != 8 + 2 * 576 * 4:
        raise RuntimeError("cs3d_ref --tables: bad output")
    return (np.frombuffer(buf, np.float32, 576, 8).copy(), np.frombuffer(buf, np.float32, 576, 8 + 576 * 4).copy())


def run(params, mesh, state, capacity, steps, dump_init=False, warmup=0, timeout=3600, workdir=None,
        decades=False, dump_grid=False):
    """Run the reference for `steps` steps from `state`.

    params: dict of cs3d_params field names (or a RefParams); mesh: dict with
    the mesh connectivity arrays nn (3, 192), sign (180) and faces (92, 7);
    state: dict with X, Y, Z (and optionally VX, VY, VZ, pressure, youngs)
    and n.  The harness computes R0 and theta0 from cell 0 of the state.
    Returns a dict of the output file."""
    if not available():
        raise FileNotFoundError(BIN + " not built (make -f oracle/ref.mk)")
    params = params if isinstance(params, RefParams) else pack_params(params)
    topo = pack_mesh(mesh)
    n = int(state["n"])
    with tempfile.TemporaryDirectory(dir=workdir) as tmp:
        fin, fout = os.path.join(tmp, "in.bin"), os.path.join(tmp, "out.bin")
        _write_input(fin, params, topo, state, capacity, steps,
                     (1 if dump_init else 0) | (2 if decades else 0) | (4 if dump_grid else 0), warmup)
        # modules loaded before the first launch, so that no kernel's first
        # launch carries its loading time
        env = dict(os.environ, CUDA_MODULE_LOADING="EAGER")
        p = subprocess.run([BIN, fin, fout], capture_output=True, text=True, timeout=timeout, env=env)
        if p.returncode != 0:
            raise RuntimeError("cs3d_ref failed (%d): %s" % (p.returncode, p.stderr[-2000:]))
        with open(fout, "rb") as f:
            buf = f.read()
    if buf[:8] != b"CS3DREFO":
        raise RuntimeError("cs3d_ref: bad output")
    off = 8
    status, done, nf, nev, max_bin, max_nn = struct.unpack_from("<6i", buf, off)
    off += 24
    total_ms, guard_ms = struct.unpack_from("<2f", buf, off)
    off += 8
    ev = np.frombuffer(buf, np.int32, 3 * nev, off).reshape(nev, 3).copy()
    off += 12 * nev
    out = {"status": status, "status_text": STATUS.get(status, "?"), "steps": done, "n": nf,
           "max_bin": max_bin, "max_local_nn": max_nn, "total_ms": total_ms, "guard_ms": guard_ms,
           "events": ev}
    kf = nf * 192
    for key in ("X", "Y", "Z", "VX", "VY", "VZ", "FCX", "FCY", "FCZ", "FDX", "FDY", "FDZ"):
        out[key] = np.frombuffer(buf, np.float32, kf, off).copy()
        off += 4 * kf
    out["pressure"] = np.frombuffer(buf, np.float32, nf, off).copy()
    off += 4 * nf
    out["youngs"] = np.frombuffer(buf, np.float32, nf, off).copy()
    off += 4 * nf
    out["cm"] = np.frombuffer(buf, np.float32, 3 * nf, off).reshape(3, nf).T.copy()
    off += 12 * nf
    n_init, n_first = struct.unpack_from("<2i", buf, off)
    off += 8
    if n_first:
        first = np.frombuffer(buf, np.float32, n_first, off).reshape(6, n_init * 192)
        out["init"] = {key: first[q].copy() for q, key in enumerate(("FCX", "FCY", "FCZ", "FDX", "FDY", "FDZ"))}
        off += 4 * n_first
    for key in ("FRX", "FRY", "FRZ"):
        out[key] = np.frombuffer(buf, np.float32, kf, off).copy()
        off += 4 * kf
    (nfar,) = struct.unpack_from("<i", buf, off)
    off += 4
    out["far"] = np.frombuffer(buf, np.int32, 2 * nfar, off).reshape(nfar, 2).copy()
    off += 8 * nfar
    (nmark,) = struct.unpack_from("<i", buf, off)
    off += 4
    out["marks"] = [struct.unpack_from("<2if", buf, off + 12 * q) for q in range(nmark)]
    off += 12 * nmark
    (ngrid,) = struct.unpack_from("<i", buf, off)
    off += 4
    if ngrid:
        minx = np.frombuffer(buf, np.float32, 6, off).copy()
        off += 24
        xdiv, ydiv, zdiv, nbins = struct.unpack_from("<4i", buf, off)
        off += 16
        counts = np.frombuffer(buf, np.int32, nbins, off).copy()
        off += 4 * nbins
        lists = np.frombuffer(buf, np.int32, 32 * nbins, off).reshape(nbins, 32).copy()
        off += 128 * nbins
        bb = np.frombuffer(buf, np.float32, 6 * ngrid, off).reshape(ngrid, 6).copy()
        out["grid"] = {"minx": minx, "divs": (xdiv, ydiv, zdiv), "counts": counts, "lists": lists, "bb": bb}
    return out
