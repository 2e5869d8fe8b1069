"""Build the engine's shared library with nvcc for sm_100a (in-tree, so the .so
travels with the sources).  `python -m storm_b200.build` rebuilds it."""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libstorm_cuda.so")
SOURCES = ["storm_kernels.cu", "storm_runtime.cu", "storm_noalloc.cu", "storm_server.cpp", "storm_mesh.cpp"]
HEADERS = ["storm_device.cuh", "storm_internal.h"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
# --fmad=false: plain expressions round like the reference's build (no contraction)
FLAGS = ["-O3", "-lineinfo", "--fmad=false", "-std=c++17", "-Xcompiler", "-fPIC,-O2", "-shared", "-lpthread"]


def _stale():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in SOURCES + HEADERS] + [os.path.join(ROOT, "include", "storm_cuda.h")]
    return any(os.path.getmtime(d) > t for d in deps)


def build(force=False, verbose=False):
    if not force and not _stale():
        return LIB
    cmd = ["nvcc"] + ARCH + FLAGS + ["-I" + os.path.join(ROOT, "include"), "-I" + CSRC] + \
          [os.path.join(CSRC, f) for f in SOURCES] + ["-o", LIB]
    if verbose:
        print(" ".join(cmd))
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("nvcc failed:\n" + r.stdout + r.stderr)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
