"""``jax.numpy`` stand-in: NumPy itself (test infrastructure only)."""

from numpy import *  # noqa: F401,F403
from numpy import asarray  # noqa: F401
