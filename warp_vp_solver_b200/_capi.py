"""ctypes bindings to ``libvpb200.so`` (the C ABI declared in ``include/vp_b200.h``).

The library is loaded from this package directory. There is no CPU fallback: if the library
is missing or no CUDA device is present, the calls that need it raise.
"""

from __future__ import annotations

import ctypes
import os
import threading

import numpy as np

VP_OK = 0
VP_ERR_ARG = 1
VP_ERR_CUDA = 2
VP_ERR_TIMEOUT = 3
VP_ERR_UNSUPPORTED = 4
VP_F32 = 0
VP_F64 = 1
VP_SCHEME_STRANG = 0
VP_SCHEME_MERGED = 1
VP_STATUS_NONFINITE_INPUT = 1
VP_STATUS_WAIT_TIMEOUT = 2
ABI_VERSION = 7   # VP_ABI_VERSION of the header these bindings follow

LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "libvpb200.so")

_lib = None
_lock = threading.Lock()

c_int = ctypes.c_int
c_i32 = ctypes.c_int32
c_i64 = ctypes.c_int64
c_dbl = ctypes.c_double
c_size = ctypes.c_size_t
c_vp = ctypes.c_void_p


class MeshDesc(ctypes.Structure):
    _fields_ = [
        ("nx", c_i32),
        ("nv", c_i32),
        ("xs", ctypes.POINTER(c_dbl)),
        ("vs", ctypes.POINTER(c_dbl)),
        ("dx", c_dbl),
        ("dv", c_dbl),
        ("period_x", c_dbl),
        ("period_v", c_dbl),
    ]


class LaunchConfig(ctypes.Structure):
    _fields_ = [
        ("rows_per_cta", c_i32),
        ("threads", c_i32),
        ("n_chunks", c_i32),
        ("chunk_cols", c_i32),
        ("tail_inline", c_i32),
        ("tail_threads", c_i32),
        ("fused_smem_bytes", c_i64),
        ("tail_smem_bytes", c_i64),
        ("cluster_size", c_i32),
        ("cluster_threads", c_i32),
        ("cluster_smem_bytes", c_i64),
        ("stage_rows", c_i32),
        ("stage_threads", c_i32),
        ("stage_span", c_i32),
        ("stage_smem_bytes", c_i64),
        ("persist_rows", c_i32),
        ("persist_ctas", c_i32),
        ("persist_smem_bytes", c_i64),
        ("strip_rows", c_i32),
        ("strip_ctas", c_i32),
        ("strip_smem_bytes", c_i64),
        ("strip_cols", c_i32),
        ("strip_adj_cols", c_i32),
    ]


class BatchConfig(ctypes.Structure):
    _fields_ = [
        ("rows_per_tile", c_i32),
        ("chunk_cols", c_i32),
        ("threads", c_i32),
        ("ctas_per_sm", c_i32),
        ("n_tiles", c_i32),
        ("grid_fwd", c_i32),
        ("grid_bwd", c_i32),
        ("strip", c_i32),
        ("strip_ctas", c_i32),
    ]


# name -> (restype, argtypes)
SIGNATURES = {
    "vp_abi_version": (c_int, []),
    "vp_get_last_error": (c_int, [ctypes.c_char_p, c_size]),
    "vp_launch_count": (c_i64, []),
    "vp_reset_launch_count": (None, []),
    "vp_plan_create": (c_int, [ctypes.POINTER(MeshDesc), c_dbl, ctypes.POINTER(c_dbl), c_int,
                               ctypes.POINTER(c_vp)]),
    "vp_plan_create_from_row": (c_int, [ctypes.POINTER(MeshDesc), c_dbl, ctypes.POINTER(c_dbl), c_int,
                                        ctypes.POINTER(c_vp)]),
    "vp_plan_destroy": (c_int, [c_vp]),
    "vp_plan_get_config": (c_int, [c_vp, ctypes.POINTER(LaunchConfig)]),
    "vp_plan_set_scheme": (c_int, [c_vp, c_i32]),
    "vp_plan_get_scheme": (c_int, [c_vp, ctypes.POINTER(c_i32)]),
    "vp_plan_set_config": (c_int, [c_vp, ctypes.POINTER(LaunchConfig)]),
    "vp_num_steps": (c_int, [c_vp, c_dbl, ctypes.POINTER(c_i32)]),
    "vp_workspace_bytes": (c_int, [c_vp, c_i32, c_i32, ctypes.POINTER(c_size)]),
    "vp_tape_bytes": (c_int, [c_vp, c_i32, c_i32, ctypes.POINTER(c_size)]),
    "vp_resolve_checkpoint_every": (c_int, [c_vp, c_i32, c_i32, ctypes.POINTER(c_i32)]),
    "vp_forward": (c_int, [c_vp, c_vp, c_vp, c_i32, c_vp, c_vp, c_vp, c_vp, c_vp, c_i32, c_vp,
                           c_size, c_vp]),
    "vp_backward": (c_int, [c_vp, c_vp, c_i32, c_vp, c_i32, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp,
                            c_vp, c_size, c_vp]),
    "vp_slab_create": (c_int, [c_vp, c_i32, c_i32, ctypes.POINTER(c_vp)]),
    "vp_slab_destroy": (c_int, [c_vp]),
    "vp_slab_geometry": (c_int, [c_vp, ctypes.POINTER(c_i32), ctypes.POINTER(c_i32), ctypes.POINTER(c_size)]),
    "vp_slab_forward_start": (c_int, [c_vp, c_vp, c_vp, c_vp, c_vp]),
    "vp_slab_field": (c_int, [c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp]),
    "vp_slab_forward_step": (c_int, [c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp]),
    "vp_slab_backward_start": (c_int, [c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp]),
    "vp_slab_backward_field": (c_int, [c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp]),
    "vp_slab_backward_step": (c_int, [c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp]),
    "vp_slab_backward_finish": (c_int, [c_vp, c_vp, c_vp, c_vp, c_vp, c_vp]),
    "vp_forward_noalloc": (c_int, [c_vp, c_vp, c_vp, c_i32, c_vp, c_vp, c_vp, c_vp, c_vp]),
    "vp_forward_stream_history": (c_int, [c_vp, c_vp, c_vp, c_i32, c_vp, c_vp, c_vp, c_i32, c_vp, c_vp,
                                          c_vp, c_i32, c_vp, c_size, c_vp, c_vp]),
    "vp_batch_create": (c_int, [c_i32, ctypes.POINTER(MeshDesc), ctypes.POINTER(c_dbl),
                                ctypes.POINTER(ctypes.POINTER(c_dbl)), c_int, ctypes.POINTER(c_vp)]),
    "vp_batch_destroy": (c_int, [c_vp]),
    "vp_batch_get_config": (c_int, [c_vp, ctypes.POINTER(BatchConfig)]),
    "vp_batch_set_config": (c_int, [c_vp, ctypes.POINTER(BatchConfig)]),
    "vp_batch_offsets": (c_int, [c_vp, ctypes.POINTER(c_i64), ctypes.POINTER(c_i64),
                                 ctypes.POINTER(c_i64), ctypes.POINTER(c_i64)]),
    "vp_batch_workspace_bytes": (c_int, [c_vp, c_i32, ctypes.POINTER(c_size)]),
    "vp_batch_tape_bytes": (c_int, [c_vp, c_i32, ctypes.POINTER(c_size)]),
    "vp_batch_forward": (c_int, [c_vp, c_vp, c_vp, c_i32, c_vp, c_vp, c_vp, c_vp, c_vp, c_size,
                                 c_vp]),
    "vp_batch_backward": (c_int, [c_vp, c_vp, c_i32, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp,
                                  c_size, c_vp]),
    "vp_mlp_create": (c_int, [c_i32, ctypes.POINTER(c_i32), c_i32, ctypes.POINTER(c_vp)]),
    "vp_mlp_destroy": (c_int, [c_vp]),
    "vp_mlp_param_count": (c_int, [c_vp, ctypes.POINTER(c_i64)]),
    "vp_mlp_set_params": (c_int, [c_vp, c_vp, c_vp]),
    "vp_mlp_get_params": (c_int, [c_vp, c_vp, c_vp, c_vp]),
    "vp_mlp_forward": (c_int, [c_vp, c_vp, c_i64, c_vp, c_i32, c_vp, c_i64, c_vp]),
    "vp_mlp_backward": (c_int, [c_vp, c_vp, c_i64, c_i32, c_i32, c_vp, c_i64, c_vp]),
    "vp_mlp_mse_backward": (c_int, [c_vp, c_vp, c_i64, c_vp, c_i32, c_vp, c_vp]),
    "vp_mlp_adam": (c_int, [c_vp, ctypes.c_float, ctypes.c_float, ctypes.c_float, ctypes.c_float, c_vp]),
    "vp_mlp_status": (c_int, [c_vp, ctypes.POINTER(ctypes.c_uint32)]),
    "vp_mlp_clear_status": (c_int, [c_vp]),
    "vp_mlp_set_wait_limit": (c_int, [c_vp, ctypes.c_uint64]),
    "vp_plan_status": (c_int, [c_vp, ctypes.POINTER(ctypes.c_uint32)]),
    "vp_plan_clear_status": (c_int, [c_vp]),
    "vp_plan_set_wait_limit": (c_int, [c_vp, ctypes.c_uint64]),
    "vp_mlp_search": (c_int, [c_vp, c_vp, c_i32, ctypes.c_float, ctypes.c_float, ctypes.c_float,
                              ctypes.c_float, ctypes.c_float, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp]),
    "vp_gemm_bf16": (c_int, [c_vp, c_i64, c_vp, c_i64, c_i32, c_i32, c_i32, c_vp, c_i32, c_vp, c_i64,
                             c_vp, c_i64, c_vp, c_i64, c_vp, c_i64, c_vp, c_vp]),
    "vp_kl_divergence": (c_int, [c_vp, c_vp, c_dbl, c_vp, c_vp, c_vp]),
    "vp_compute_rho": (c_int, [c_vp, c_vp, c_vp, c_vp]),
    "vp_poisson": (c_int, [c_vp, c_vp, c_vp, c_int, c_vp]),
    "vp_electric_energy": (c_int, [c_vp, c_vp, c_vp, c_vp]),
    "vp_semilag_x": (c_int, [c_vp, c_vp, c_vp, c_dbl, c_int, c_vp]),
    "vp_semilag_v": (c_int, [c_vp, c_vp, c_vp, c_vp, c_dbl, c_int, c_vp, c_vp, c_vp]),
}


class VPError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(msg)
        self.code = code


def load():
    """Load the library (once) and declare the C signatures."""
    global _lib
    with _lock:
        if _lib is None:
            if not os.path.exists(LIB_PATH):
                raise RuntimeError(
                    f"{LIB_PATH} is missing: build it with `python -m warp_vp_solver_b200.build` "
                    "(there is no CPU fallback)")
            lib = ctypes.CDLL(LIB_PATH)
            for name, (res, args) in SIGNATURES.items():
                fn = getattr(lib, name)
                fn.restype = res
                fn.argtypes = args
            if lib.vp_abi_version() != ABI_VERSION:
                raise RuntimeError(f"{LIB_PATH} has ABI version {lib.vp_abi_version()}, the bindings "
                                   f"expect {ABI_VERSION}: rebuild with `python -m warp_vp_solver_b200.build`")
            _lib = lib
    return _lib


def last_error() -> str:
    buf = ctypes.create_string_buffer(512)
    load().vp_get_last_error(buf, len(buf))
    return buf.value.decode(errors="replace")


def check(rc: int) -> None:
    if rc == VP_OK:
        return
    msg = last_error()
    if rc == VP_ERR_ARG:
        raise ValueError(msg)
    if rc == VP_ERR_UNSUPPORTED:
        raise NotImplementedError(msg)
    raise VPError(rc, msg)


def ptr(t) -> int | None:
    """Device pointer of a torch tensor (or None)."""
    return None if t is None else int(t.data_ptr())


def dbl_ptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(c_dbl))
