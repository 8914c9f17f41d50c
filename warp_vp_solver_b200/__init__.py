"""B200-native (sm_100a) Vlasov-Poisson Strang step and discrete adjoint.

A drop-in for the ``WarpVlasovPoissonSolver`` path of Forgotten/warp_vp_solver: the same
``Mesh``/``make_mesh``, the same solver constructor and ``run_forward`` contract, torch autograd
in place of ``jax.custom_vjp``, and torch versions of the control/cost utilities. The compute
runs in hand-written CUDA kernels reached through the C ABI in ``include/vp_b200.h``.
"""

from .mesh import Mesh, make_mesh
from .solver import WarpVlasovPoissonSolver, run_forward_jax_compatible
from .utils import (
    electric_energy_in_time,
    external_electric_field,
    kl_divergence,
    make_cost_function_ee,
    make_cost_function_eet,
    make_cost_function_kl,
)

__all__ = [
    "Mesh",
    "WarpVlasovPoissonSolver",
    "electric_energy_in_time",
    "external_electric_field",
    "kl_divergence",
    "make_cost_function_ee",
    "make_cost_function_eet",
    "make_cost_function_kl",
    "make_mesh",
    "run_forward_jax_compatible",
]
__version__ = "0.1.0"
