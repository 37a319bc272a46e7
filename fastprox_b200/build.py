"""Builds libfastprox_b200.so in-tree: the sm_100a kernels (nvcc) and the
C-ABI host code (g++, C++17), linked with the static CUDA runtime so the
library needs nothing at run time beyond the driver.

    python -m fastprox_b200.build        # rebuild if any source changed
"""

from __future__ import annotations

import os
import pathlib
import shutil
import subprocess
import sys

HERE = pathlib.Path(__file__).resolve().parent
CSRC = HERE / "csrc"
LIB = HERE / "libfastprox_b200.so"
BUILD = HERE.parent / "_build"
CUDA = pathlib.Path(os.environ.get("CUDA_HOME", "/usr/local/cuda"))
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
              "--expt-relaxed-constexpr"] + ARCH
CXX_FLAGS = ["-std=c++17", "-O2", "-fPIC", "-fvisibility=hidden", "-Wall", "-Wextra", f"-I{CUDA / 'include'}"]

CU_SOURCES = sorted(CSRC.glob("*.cu"))
CPP_SOURCES = sorted(CSRC.glob("*.cpp"))
HEADERS = sorted(list(CSRC.glob("*.h")) + list(CSRC.glob("*.cuh")) + list((HERE.parent / "include").glob("*.h")))


def _stale() -> bool:
    if not LIB.exists():
        return True
    t = LIB.stat().st_mtime
    return any(p.stat().st_mtime > t for p in CU_SOURCES + CPP_SOURCES + HEADERS)


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(" ".join(map(str, cmd)) + "\n" + r.stdout + r.stderr)
        raise RuntimeError(f"build step failed: {cmd[0]} {cmd[-1]}")
    return r


def build(force: bool = False, verbose: bool = False) -> pathlib.Path:
    """Compiles every kernel for sm_100a and links the shared library."""
    if not force and not _stale():
        return LIB
    nvcc = shutil.which("nvcc") or str(CUDA / "bin" / "nvcc")
    BUILD.mkdir(exist_ok=True)
    objs = []
    procs = []
    for src in CU_SOURCES:
        obj = BUILD / (src.stem + ".o")
        cmd = [nvcc, *NVCC_FLAGS, "-c", str(src), "-o", str(obj)]
        procs.append((cmd, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True)))
        objs.append(obj)
    for src in CPP_SOURCES:
        obj = BUILD / (src.stem + ".o")
        cmd = ["g++", *CXX_FLAGS, "-c", str(src), "-o", str(obj)]
        procs.append((cmd, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True)))
        objs.append(obj)
    failed = False
    for cmd, p in procs:
        out, err = p.communicate()
        if p.returncode != 0:
            failed = True
            sys.stderr.write(" ".join(cmd) + "\n" + out + err)
        elif verbose and (out or err):
            sys.stderr.write(out + err)
    if failed:
        raise RuntimeError("compilation failed")
    tmp = LIB.with_suffix(".so.tmp")
    _run([nvcc, "-shared", *ARCH, "-cudart", "static", "-o", str(tmp), *map(str, objs),
          "-Xlinker", "--no-undefined", "-lpthread", "-ldl", "-lrt"])
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
    print(LIB)
