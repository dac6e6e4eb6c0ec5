"""Build the engine's CUDA library in-tree for sm_100a.

``build_library()`` compiles every ``csrc/*.cu`` (and the host-only
``csrc/*.cpp``) with nvcc into
``liboxav1_b200.so`` next to this file (objects in ``_build/``), rebuilding only
what changed.  The library is the product: the Python host layer loads it with
ctypes and has no fallback when it is missing.
"""
import os
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
REPO = PKG.parent
CSRC = PKG / "csrc"
BUILD = PKG / "_build"
LIB = PKG / "liboxav1_b200.so"
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
         "-I" + str(REPO / "include"), "-I" + str(CSRC)]


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("command failed: " + " ".join(cmd))
    return r.stdout + r.stderr


def build_library(force: bool = False, verbose: bool = False) -> Path:
    BUILD.mkdir(exist_ok=True)
    headers = list(CSRC.glob("*.cuh")) + list(CSRC.glob("*.h")) + list((REPO / "include").glob("*.h"))
    hdr_mtime = max(p.stat().st_mtime for p in headers)
    objs = []
    for cu in sorted(list(CSRC.glob("*.cu")) + list(CSRC.glob("*.cpp"))):
        obj = BUILD / (cu.stem + ".o")
        objs.append(obj)
        if force or not obj.exists() or obj.stat().st_mtime < max(cu.stat().st_mtime, hdr_mtime):
            out = _run([NVCC, *ARCH, *FLAGS, "-Xptxas", "-v" if verbose else "-O3", "-c", str(cu), "-o", str(obj)])
            if verbose:
                sys.stderr.write(out)
    if force or not LIB.exists() or LIB.stat().st_mtime < max(o.stat().st_mtime for o in objs):
        _run([NVCC, *ARCH, "-shared", "-o", str(LIB), *map(str, objs), "-lcudart"])
    return LIB


if __name__ == "__main__":
    print(build_library(force="--force" in sys.argv, verbose="-v" in sys.argv))
