"""Per-step diffusion arguments (KELP ``src/kelp/numerics/diffusion.py:84-131``).

The random walk itself runs inside the CUDA step kernels: the counter RNG keyed
by ``(seed, real_id, pid_offset + particle index, step_i, component)``
(``diffusion.py:180-249``), the uniform-Kh split kick and its great-circle
move (``diffusion.py:485-575``, ``integrators.py:673-818``).
"""
from __future__ import annotations

from typing import NamedTuple


class DiffusionStepArgs(NamedTuple):
    scheme: str
    kh_x: float
    kh_y: float
    seed: int
    real_id: int
    step_i: int
    composition: str = "split"
    dres_m: float = 0.0
    kh_eval_position: str = "end"
    az_enabled: bool = False
    az_const: float = 0.0
    az_requires_field: bool = False
    pid_offset: int = 0


COMP_HORIZONTAL = 0
COMP_VERTICAL = 1
