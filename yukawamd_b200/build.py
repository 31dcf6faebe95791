"""Build the engine's shared library for sm_100a.

    python -m yukawamd_b200.build          # -> yukawamd_b200/libyukawa_b200.so

The library links the CUDA runtime statically, so loading it needs only the
NVIDIA driver when a GPU is used (and nothing at all for symbol inspection on
a machine without one).  nvcc cross-compiles sm_100a without a GPU.
"""
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libyukawa_b200.so")

SOURCES = ["yk_engine.cu", "yk_batch.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-shared",
         "-cudart", "static", "--expt-relaxed-constexpr",
         "-Xcompiler", "-fvisibility=hidden"]


def nvcc():
    path = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(path):
        raise RuntimeError("nvcc not found")
    return path


def sources():
    return [os.path.join(CSRC, s) for s in SOURCES]


def deps():
    out = [os.path.join(ROOT, "include", "yukawa_engine.h")]
    for f in os.listdir(CSRC):
        if f.endswith((".cu", ".cuh", ".h")):
            out.append(os.path.join(CSRC, f))
    return out


def up_to_date():
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    return all(os.path.getmtime(d) <= t for d in deps())


def build(force=False, verbose=False, ptxas_info=False):
    if not force and up_to_date():
        return LIB
    cmd = [nvcc()] + ARCH + FLAGS + ["-I", os.path.join(ROOT, "include")]
    if ptxas_info:
        cmd += ["-Xptxas", "-v"]
    cmd += sources() + ["-o", LIB + ".tmp"]
    if verbose:
        print(" ".join(cmd), flush=True)
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        sys.stderr.write(res.stdout + res.stderr)
        raise RuntimeError("nvcc failed building %s" % LIB)
    if ptxas_info or verbose:
        sys.stderr.write(res.stderr)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True, ptxas_info="--ptxas" in sys.argv)
    print(LIB)
