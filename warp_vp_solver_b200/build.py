"""Build the in-tree CUDA library ``libvpb200.so`` for sm_100a.

Usage: ``python -m warp_vp_solver_b200.build [-v]``. The library is placed next to this file so
that it travels with the source tree. Nothing is installed into site-packages.
"""

from __future__ import annotations

import os
import shutil
import subprocess
import sys

PKG_DIR = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(PKG_DIR, "csrc")
LIB_NAME = "libvpb200.so"
LIB_PATH = os.path.join(PKG_DIR, LIB_NAME)
INCLUDE_DIR = os.path.join(os.path.dirname(PKG_DIR), "include")

SOURCES = ["vp_capi.cu", "vp_kernels.cu", "vp_ops.cu", "vp_resident.cu", "vp_mlp.cu"]
HEADERS = ["vp_internal.h", "vp_device.cuh"]

ARCH_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = [
    "-O3", "-lineinfo", "-std=c++17",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-ffp-contract=off", "-Xcompiler", "-O2",
    "-shared", "-cudart", "shared",
]


def nvcc_path() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found; set NVCC or add the CUDA toolkit to PATH")


def _stale() -> bool:
    if not os.path.exists(LIB_PATH):
        return True
    lib_t = os.path.getmtime(LIB_PATH)
    deps = [os.path.join(CSRC, f) for f in SOURCES + HEADERS]
    deps.append(os.path.join(INCLUDE_DIR, "vp_b200.h"))
    return any(os.path.getmtime(d) > lib_t for d in deps if os.path.exists(d))


def build(force: bool = False, verbose: bool = False, ptxas_info: bool = False) -> str:
    if not force and not ptxas_info and not _stale():
        return LIB_PATH
    cmd = [nvcc_path(), *ARCH_FLAGS, *NVCC_FLAGS, f"-I{INCLUDE_DIR}"]
    if ptxas_info:
        cmd += ["-Xptxas", "-v"]
    cmd += [os.path.join(CSRC, s) for s in SOURCES]
    tmp = LIB_PATH + ".tmp"
    cmd += ["-o", tmp]
    if verbose:
        print(" ".join(cmd), flush=True)
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"nvcc failed ({res.returncode}):\n{res.stdout}\n{res.stderr}")
    if verbose or ptxas_info:
        sys.stdout.write(res.stdout + res.stderr)
    os.replace(tmp, LIB_PATH)
    return LIB_PATH


if __name__ == "__main__":
    build(force=True, verbose="-v" in sys.argv, ptxas_info="--ptxas" in sys.argv)
    print(LIB_PATH)
