"""Build the in-tree CUDA library ``libvpb200.so`` for sm_100a.

Usage: ``python -m warp_vp_solver_b200.build [-v] [--ptxas] [--force]``. Each source is compiled to an
object under ``_build/`` in parallel (one nvcc process per file, rebuilt only when the file or a
header changed), then linked into the library next to this file so that it travels with the
source tree. Nothing is installed into site-packages.
"""

from __future__ import annotations

import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

PKG_DIR = os.path.dirname(os.path.abspath(__file__))
ROOT_DIR = os.path.dirname(PKG_DIR)
CSRC = os.path.join(PKG_DIR, "csrc")
LIB_NAME = "libvpb200.so"
LIB_PATH = os.path.join(PKG_DIR, LIB_NAME)
INCLUDE_DIR = os.path.join(ROOT_DIR, "include")
OBJ_DIR = os.path.join(ROOT_DIR, "_build")

SOURCES = ["vp_capi.cu", "vp_kernels.cu", "vp_ops.cu", "vp_resident.cu", "vp_mlp.cu", "vp_persist.cu", "vp_strip.cu"]
HEADERS = ["vp_internal.h", "vp_device.cuh", "vp_pst.cuh"]

ARCH_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMPILE_FLAGS = [
    "-O3", "-lineinfo", "-std=c++17",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-ffp-contract=off", "-Xcompiler", "-O2",
]
LINK_FLAGS = ["-shared", "-cudart", "shared"]


def nvcc_path() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found; set NVCC or add the CUDA toolkit to PATH")


def _sources():
    return [s for s in SOURCES if os.path.exists(os.path.join(CSRC, s))]


def _headers():
    hs = [os.path.join(CSRC, h) for h in HEADERS]
    hs.append(os.path.join(INCLUDE_DIR, "vp_b200.h"))
    return [h for h in hs if os.path.exists(h)]


def _obj(src: str) -> str:
    return os.path.join(OBJ_DIR, os.path.splitext(src)[0] + ".o")


def _obj_stale(src: str) -> bool:
    o = _obj(src)
    if not os.path.exists(o):
        return True
    t = os.path.getmtime(o)
    return any(os.path.getmtime(d) > t for d in [os.path.join(CSRC, src), *_headers()])


def _stale() -> bool:
    if not os.path.exists(LIB_PATH):
        return True
    lib_t = os.path.getmtime(LIB_PATH)
    deps = [os.path.join(CSRC, s) for s in _sources()] + _headers()
    return any(os.path.getmtime(d) > lib_t for d in deps)


def _compile(src: str, ptxas_info: bool):
    cmd = [nvcc_path(), *ARCH_FLAGS, *COMPILE_FLAGS, f"-I{INCLUDE_DIR}", "-c",
           os.path.join(CSRC, src), "-o", _obj(src) + ".tmp"]
    if ptxas_info:
        cmd[1:1] = ["-Xptxas", "-v"]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode == 0:
        os.replace(_obj(src) + ".tmp", _obj(src))
    return src, cmd, res


def build(force: bool = False, verbose: bool = False, ptxas_info: bool = False) -> str:
    if not force and not ptxas_info and not _stale():
        return LIB_PATH
    os.makedirs(OBJ_DIR, exist_ok=True)
    srcs = _sources()
    todo = [s for s in srcs if force or ptxas_info or _obj_stale(s)]
    with ThreadPoolExecutor(max_workers=max(1, min(len(todo), os.cpu_count() or 1))) as ex:
        results = list(ex.map(lambda s: _compile(s, ptxas_info), todo))
    for src, cmd, res in results:
        if verbose:
            print(" ".join(cmd), flush=True)
        if res.returncode != 0:
            raise RuntimeError(f"nvcc failed on {src} ({res.returncode}):\n{res.stdout}\n{res.stderr}")
        if verbose or ptxas_info:
            sys.stdout.write(res.stdout + res.stderr)
    tmp = LIB_PATH + ".tmp"
    cmd = [nvcc_path(), *ARCH_FLAGS, *LINK_FLAGS, *[_obj(s) for s in srcs], "-o", tmp]
    if verbose:
        print(" ".join(cmd), flush=True)
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"nvcc link failed ({res.returncode}):\n{res.stdout}\n{res.stderr}")
    os.replace(tmp, LIB_PATH)
    return LIB_PATH


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv, ptxas_info="--ptxas" in sys.argv)
    print(LIB_PATH)
