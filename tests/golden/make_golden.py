"""Generate the committed golden fixtures from the reference checkout.

Run once in a container that has the reference mounted:

    python tests/golden/make_golden.py /path/to/CellSim3D

Writes, next to this script:
  c180_mesh.npz   -- the C180 mesh exactly as the reference's loaders read it
                     (C180 coordinates as float32 via fscanf("%f"), C180NN
                     neighbours and signs, C180C bonds, C180_pentahexa faces);
                     src/GPUbounce.cu:1616-1627 and :1814-1888.
  ranmar_kat.json -- RANMAR known-answer test from the comment in
                     src/marsaglia.h:66-72 (seeds 1802/9373, values after 20000
                     draws times 4096*4096).
  traj_small.bin  -- a two-frame binary trajectory written by this library's
  traj_small.json    writer, and the frames that scripts/celldiv.py reads back
                     from it (step, frame, cell count, coordinates checksum).
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def _strtof(tok):
    """Decimal -> float exactly as fscanf("%f") (glibc strtof), no double rounding."""
    import ctypes
    libc = ctypes.CDLL(None)
    libc.strtof.restype = ctypes.c_float
    libc.strtof.argtypes = [ctypes.c_char_p, ctypes.c_void_p]
    return np.float32(libc.strtof(tok.encode(), None))


def read_mesh(root):
    xyz = []
    with open(os.path.join(root, "C180")) as f:
        for line in f:
            if line.strip():
                xyz.append([_strtof(t) for t in line.split()[:3]])
    xyz = np.array(xyz[:180], dtype=np.float32)
    nn = np.zeros((3, 192), dtype=np.int32)
    sign = np.zeros(180, dtype=np.int32)
    with open(os.path.join(root, "C180NN")) as f:
        rows = [r for r in f.read().replace(",", " ").split("\n") if r.strip()]
    for i in range(180):
        a, b, c, s = [int(t) for t in rows[i].split()[:4]]
        nn[:, i] = (a - 1, b - 1, c - 1)
        sign[i] = s
    with open(os.path.join(root, "C180C")) as f:
        rows = [r for r in f.read().replace(",", " ").split("\n") if r.strip()]
    bonds = np.array([[int(t) - 1 for t in r.split()[:2]] for r in rows[:270]], dtype=np.int32)
    faces = np.zeros((92, 7), dtype=np.int32)
    with open(os.path.join(root, "C180_pentahexa")) as f:
        rows = [r for r in f.read().split("\n") if r.strip()]
    for i in range(12):
        v = [int(t) for t in rows[i].split()[:5]]
        faces[i] = v + [v[0], v[0]]
    for i in range(80):
        v = [int(t) for t in rows[12 + i].split()[:6]]
        faces[12 + i] = v + [v[0]]
    return xyz, nn, sign, bonds, faces


def main(root, with_traj=True):
    xyz, nn, sign, bonds, faces = read_mesh(root)
    np.savez(os.path.join(HERE, "c180_mesh.npz"), xyz=xyz, nn=nn, sign=sign, bonds=bonds, faces=faces)
    kat = {"ij": 1802, "kl": 9373, "skip": 20000,
           "expect_x4096sq": [6533892.0, 14220222.0, 7275067.0, 6172232.0, 8354498.0, 10633180.0],
           "source": "src/marsaglia.h:66-72"}
    with open(os.path.join(HERE, "ranmar_kat.json"), "w") as f:
        json.dump(kat, f, indent=1)
    if not with_traj:
        return
    # trajectory round trip through the reference's own reader
    sys.path.insert(0, os.path.join(root, "scripts"))
    sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
    import celldiv  # reference reader, scripts/celldiv.py
    from cellsim3d_b200 import traj
    rng = np.random.default_rng(5)
    path = os.path.join(HERE, "traj_small.bin")
    frames = []
    with traj.TrajWriter(path, max_cells=16, variable_stiffness=False, max_frames=2) as w:
        for k, (step, n) in enumerate([(0, 2), (10, 3)]):
            X = rng.standard_normal((n, 192)).astype(np.float32)
            Y = rng.standard_normal((n, 192)).astype(np.float32)
            Z = rng.standard_normal((n, 192)).astype(np.float32)
            w.write_frame(step, k + 1, X, Y, Z)
            frames.append((step, k + 1, n))
        w.set_final_cells(3)
    th = celldiv.TrajHandle(path) if hasattr(celldiv, "TrajHandle") else celldiv.TrajHandleBinary(path)
    out = {"maxNCells": int(th.maxNCells), "variableStiffness": int(th.variableStiffness),
           "maxFrames": int(th.maxFrames), "frames": []}
    for k in range(2):
        fr = th.ReadFrame()
        arr = np.array(fr, dtype=np.float64)
        out["frames"].append({"step": int(th.step), "frame": int(th.currFrameNum),
                              "n": len(fr), "sum": float(arr.sum()),
                              "first": [float(v) for v in arr[0, 0]]})
    th.close()
    with open(os.path.join(HERE, "traj_small.json"), "w") as f:
        json.dump(out, f, indent=1)
    print("golden fixtures written to", HERE)


if __name__ == "__main__":
    args = [a for a in sys.argv[1:] if not a.startswith("--")]
    root = args[0] if args else os.environ.get("CELLSIM3D_REF") or os.path.join(
        os.path.dirname(os.path.dirname(os.path.dirname(HERE))), "reference")
    main(root, with_traj="--no-traj" not in sys.argv)
