"""kelp_b200 -- KELP's compiled time-stepping path on the NVIDIA B200 (sm_100a).

Host code mirrors KELP's types and step signature; the work runs in
hand-written CUDA kernels behind the C ABI of ``include/kelp_cuda.h``.
"""
from .particles import ParticleState, ParticleStatus, FailureReason, make_state
from .fields import VelocityField, LazyLerpField
from .mesh import Mesh, build_search, build_grid_hash, build_node_to_elems, make_mesh, set_exact_nearest
from .diffusion import DiffusionStepArgs
from .integrators import euler_step, rk2_step, rk4_step, get_integrator, INTEGRATORS

__all__ = ["ParticleState", "ParticleStatus", "FailureReason", "make_state", "VelocityField",
           "LazyLerpField", "Mesh", "build_search", "build_grid_hash", "build_node_to_elems", "make_mesh",
           "set_exact_nearest", "DiffusionStepArgs", "euler_step", "rk2_step", "rk4_step",
           "get_integrator", "INTEGRATORS"]
