"""Builds libinching_b200.so (all CUDA sources under csrc/) for sm_100a, in tree.

    python -m inching_b200.build        # or inching_b200.build.build()

nvcc cross-compiles without a GPU.  The shared library is written next to this
file so it travels with the source tree.
"""
from __future__ import annotations

import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libinching_b200.so")


def _cuda_home() -> str:
    """Toolkit root: $CUDA_HOME / $CUDA_PATH, else the directory above the nvcc on PATH."""
    for var in ("CUDA_HOME", "CUDA_PATH"):
        if os.environ.get(var):
            return os.environ[var]
    import shutil
    nv = shutil.which("nvcc")
    if nv:
        return os.path.dirname(os.path.dirname(os.path.realpath(nv)))
    raise RuntimeError("no CUDA toolkit: set CUDA_HOME or put nvcc on PATH")


CUDA_HOME = _cuda_home()
NVCC = os.environ.get("NVCC", os.path.join(CUDA_HOME, "bin", "nvcc"))

NVCC_FLAGS = [
    "-O3", "-std=c++17", "-lineinfo",
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
    "-Xptxas", "-warn-spills",
]


def sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")))


def _stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = sources() + glob.glob(os.path.join(CSRC, "*.cuh")) + \
        glob.glob(os.path.join(HERE, "..", "include", "*.h"))
    return any(os.path.getmtime(p) > t for p in deps)


def build(force: bool = False, verbose: bool = False) -> str:
    """Compile every .cu in csrc/ into one shared library (parallel per file)."""
    if not force and not _stale():
        return LIB
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    procs = []
    objs = []
    for src in sources():
        obj = os.path.join(objdir, os.path.basename(src)[:-3] + ".o")
        objs.append(obj)
        cmd = [NVCC, *NVCC_FLAGS, "-c", src, "-o", obj]
        if verbose:
            print(" ".join(cmd))
        procs.append((src, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT)))
    failed = []
    for src, p in procs:
        out = p.communicate()[0].decode()
        if p.returncode != 0:
            failed.append((src, out))
        elif verbose and out.strip():
            print(out)
    if failed:
        msg = "\n".join(f"--- {s}\n{o}" for s, o in failed)
        raise RuntimeError(f"nvcc failed:\n{msg}")
    tmp = LIB + ".tmp"
    # cuBLAS for the tall-skinny GEMMs of the block-solver entry points; the rpath
    # finds the toolkit's copy when no other libcublas.so.12 is loaded already
    cmd = [NVCC, "-shared", "-gencode", "arch=compute_100a,code=sm_100a", *objs, "-lcublas",
           "-Xlinker", "-rpath=" + os.path.join(CUDA_HOME, "lib64"), "-o", tmp]
    r = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT)
    if r.returncode != 0:
        raise RuntimeError("link failed:\n" + r.stdout.decode())
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
