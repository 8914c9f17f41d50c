"""Serial Python interpreter for the subset of NVIDIA Warp that the reference kernels use.

Test infrastructure only. ``make_golden.py`` puts this directory first on
``sys.path`` so that the reference's own ``warp_vp_solver/kernels.py`` and
``warp_vp_solver/solver.py`` import it in place of ``warp`` (which is not
installable offline). Each ``wp.launch`` then runs the reference's
``@wp.kernel`` body once per thread index, in row-major thread order, on
NumPy float64 arrays. That reproduces the reference arithmetic
(IEEE float64, no fused multiply-add) so its outputs can be recorded as
golden vectors.

Only what the reference's legacy forward/backward and its single-stage
kernels touch is provided: ``kernel``, ``func``, ``launch``, ``tid``,
``array``/``array2d``, ``zeros``, ``float64``, ``int32``, ``floor`` and
``atomic_add``. ``tile_fft`` is deliberately absent, so
``warp_vp_solver/poisson.py`` takes its host-FFT branch exactly as it does on
a Warp build without tile FFTs.
"""

from __future__ import annotations

import numpy as np

float64 = np.float64


def int32(x):
    """Warp's int32 constructor: C-style truncation toward zero."""
    return int(x)


def floor(x):
    return np.floor(x)


class array:
    """A host array standing in for ``wp.array`` (float64 or int32 data)."""

    def __init__(self, data=None, dtype=float64, shape=None, device=None):
        np_dtype = np.int64 if dtype is int32 else np.float64
        if data is None:
            self._a = np.zeros(shape, dtype=np_dtype)
        else:
            src = data._a if isinstance(data, array) else data
            self._a = np.array(src, dtype=np_dtype, copy=True)
        self.device = device

    @property
    def shape(self):
        return self._a.shape

    def __getitem__(self, idx):
        return self._a[idx]

    def __setitem__(self, idx, value):
        self._a[idx] = value

    def numpy(self):
        return self._a.copy()

    def assign(self, src):
        src = src._a if isinstance(src, array) else np.asarray(src)
        self._a[...] = src

    def zero_(self):
        self._a[...] = 0


def array2d(dtype=None):  # only ever used inside (unevaluated) annotations
    return array


def zeros(shape, dtype=float64, device=None):
    return array(None, dtype=dtype, shape=shape, device=device)


_TID = None


def tid():
    return _TID


def kernel(fn):
    fn.__warp_kernel__ = True
    return fn


def func(fn):
    return fn


def launch(kernel, dim, inputs, device=None, **_unused):
    """Run ``kernel`` once per thread index, in row-major order."""
    global _TID
    args = list(inputs)
    if isinstance(dim, (tuple, list)):
        if len(dim) == 1:
            dim = int(dim[0])
        else:
            n0, n1 = int(dim[0]), int(dim[1])
            for i in range(n0):
                for j in range(n1):
                    _TID = (i, j)
                    kernel(*args)
            _TID = None
            return
    for i in range(int(dim)):
        _TID = i
        kernel(*args)
    _TID = None


def atomic_add(arr, *args):
    *idx, value = args
    key = tuple(int(k) for k in idx)
    arr._a[key] = arr._a[key] + value
    return None


def init():
    return None
