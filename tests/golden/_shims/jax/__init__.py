"""Import-time stand-in for ``jax`` (test infrastructure only).

The reference's ``warp_vp_solver/solver.py`` imports ``jax`` and
``jax.numpy`` at module top but only touches them inside
``_build_jax_callable``. ``make_golden.py`` calls the solver's NumPy entry
points (``run_forward``, ``_run_backward``) directly, so this stub only has
to make the import succeed.
"""

from . import numpy  # noqa: F401


def custom_vjp(*_args, **_kwargs):  # pragma: no cover - never reached
    raise NotImplementedError("jax is not available; golden generation uses the NumPy entry points")
