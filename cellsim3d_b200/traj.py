"""Binary trajectory files (the format scripts/celldiv.py reads).

TrajWriter drives the native writer of libcs3d.so (header
src/GPUbounce.cu:1007-1018, frames :2446-2477, final cell count :1508-1511);
read_traj is a small reader of the same format for tests and tools.
"""
import ctypes as C

import numpy as np

from . import _lib


class TrajWriter:
    def __init__(self, path, max_cells, variable_stiffness=False, max_frames=0):
        self.h = C.c_void_p()
        st = _lib.lib().cs3d_traj_open(str(path).encode(), int(max_cells), int(bool(variable_stiffness)),
                                       int(max_frames), C.byref(self.h))
        _lib.check(st, "cs3d_traj_open")
        self.final = -1

    def write_frame(self, step, frame, X, Y, Z, types=None):
        X = np.ascontiguousarray(X, dtype=np.float32).reshape(-1)
        Y = np.ascontiguousarray(Y, dtype=np.float32).reshape(-1)
        Z = np.ascontiguousarray(Z, dtype=np.float32).reshape(-1)
        n = X.size // 192
        t = np.ascontiguousarray(types, dtype=np.int32) if types is not None else None
        fp = C.POINTER(C.c_float)
        st = _lib.lib().cs3d_traj_write_frame(self.h, int(step), int(frame), n, X.ctypes.data_as(fp),
                                              Y.ctypes.data_as(fp), Z.ctypes.data_as(fp),
                                              t.ctypes.data_as(C.POINTER(C.c_int32)) if t is not None else None)
        _lib.check(st, "cs3d_traj_write_frame")

    def set_final_cells(self, n):
        self.final = int(n)

    def close(self):
        if self.h.value:
            _lib.check(_lib.lib().cs3d_traj_close(self.h, self.final), "cs3d_traj_close")
            self.h = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


def read_traj(path):
    """Header dict and a list of frames (step, frame, X, Y, Z as (n,192) arrays, types)."""
    raw = np.fromfile(path, dtype=np.uint8)
    off = 0

    def ints(k):
        nonlocal off
        v = np.frombuffer(raw[off:off + 4 * k].tobytes(), dtype=np.int32)
        off += 4 * k
        return v

    def floats(k):
        nonlocal off
        v = np.frombuffer(raw[off:off + 4 * k].tobytes(), dtype=np.float32)
        off += 4 * k
        return v

    max_cells, var, max_frames = ints(3)
    frames = []
    while off < raw.size:
        step, frame, n = ints(3)
        X = np.zeros((n, 192), np.float32)
        Y = np.zeros_like(X)
        Z = np.zeros_like(X)
        types = np.zeros(n, np.int32)
        for c in range(n):
            ints(1)
            X[c] = floats(192)
            Y[c] = floats(192)
            Z[c] = floats(192)
            if var:
                types[c] = ints(1)[0]
        frames.append({"step": int(step), "frame": int(frame), "X": X, "Y": Y, "Z": Z, "types": types})
    return {"max_cells": int(max_cells), "variable_stiffness": int(var), "max_frames": int(max_frames)}, frames
