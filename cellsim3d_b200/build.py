"""Build libcs3d.so (sm_100a) and the cs3d command-line driver in-tree.

    python -m cellsim3d_b200.build          # library + driver
"""
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libcs3d.so")
CLI = os.path.join(HERE, "cs3d")

NVCC = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-ffp-contract=off",
                  "-I" + os.path.join(ROOT, "include")]
CXXFLAGS = ["-O2", "-fPIC", "-std=c++17", "-ffp-contract=off", "-fno-fast-math", "-Wall",
            "-I" + os.path.join(ROOT, "include")]


def _run(cmd, verbose):
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)


def _stale(target, sources):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(s) > t for s in sources)


def build(verbose=False, force=False, extra_nvflags=()):
    os.makedirs(BUILD, exist_ok=True)
    hdrs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    hdrs.append(os.path.join(ROOT, "include", "cs3d.h"))
    host_o = os.path.join(BUILD, "cs3d_host.o")
    api_o = os.path.join(BUILD, "cs3d_api.o")
    host_src = os.path.join(CSRC, "cs3d_host.cpp")
    api_src = os.path.join(CSRC, "cs3d_api.cu")
    if force or _stale(host_o, [host_src] + hdrs):
        _run(["g++"] + CXXFLAGS + ["-c", host_src, "-o", host_o], verbose)
    if force or extra_nvflags or _stale(api_o, [api_src] + hdrs):
        _run([NVCC] + NVFLAGS + list(extra_nvflags) + ["-c", api_src, "-o", api_o], verbose)
    if force or _stale(LIB, [host_o, api_o]):
        _run([NVCC] + ARCH + ["-shared", "-cudart", "static", "-o", LIB, host_o, api_o], verbose)
    main_src = os.path.join(CSRC, "cs3d_main.cpp")
    if force or _stale(CLI, [main_src, LIB] + hdrs):
        _run(["g++"] + CXXFLAGS + ["-pthread", main_src, "-o", CLI, "-L" + HERE, "-lcs3d",
                                   "-Wl,-rpath,$ORIGIN"], verbose)
    return LIB


if __name__ == "__main__":
    build(verbose=True, force="--force" in sys.argv)
