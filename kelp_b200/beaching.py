"""Beaching and resuspension after each step, on the B200.

Mirrors KELP's post-step hook: the configuration (``BeachingConfig``,
``src/kelp/core/config.py:213-266``), the per-run constants
(``BeachRunConfig``, ``src/kelp/numerics/beaching.py:79-93``, resolved as in
``src/kelp/tracking.py:2080-2101``) and ``apply_beaching_hook``
(``src/kelp/tracking.py:199-364`` with ``numerics.beaching.evaluate_beaching``,
``beaching.py:95-181``): the on_failure remap of particles the step killed,
the depth / coastal_element / stochastic criteria and the automatic /
stochastic resuspension.  One kernel launch (``kc_beach``) per hook call; the
stochastic draws use the same counter hash as the diffusion kick with
components 10 and 11, keyed by the particle's original index.

With ``use_eta`` the payload's free surface is added to the anchor's depth,
and with ``dry_mask_var`` the payload's scalar of that name (its surface
layer) marks dry nodes: both node arrays are formed on the host as the
payload forms them and handed to the kernel per hook call
(``kc_beach_surface``).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from typing import Any, List, NamedTuple, Optional

import numpy as np

from . import _native as N
from .device import default_context
from .mesh import build_boundary_info
from .particles import ParticleState

VALID_CRITERIA = ("depth", "coastal_element", "on_failure", "stochastic")
RESUSP_CODES = {"never": 0, "auto": 1, "stochastic": 2, "auto_or_stochastic": 3}


@dataclass
class BeachingConfig:
    """``beaching:`` section of a run configuration (config.py:213-266)."""
    enabled: bool = False
    criteria: List[str] = field(default_factory=lambda: ["depth"])
    depth_min: float = 0.3
    use_eta: bool = False
    dry_mask_var: Optional[str] = None
    zone_depth: Optional[float] = None
    t_beach: Optional[float] = 86400.0
    resuspension: str = "never"
    rewet_hysteresis: float = 0.1
    min_wet_steps: int = 1
    t_resuspend: Optional[float] = None
    seed: Optional[int] = None

    def __post_init__(self) -> None:
        if isinstance(self.criteria, str):
            self.criteria = [self.criteria]
        if not self.enabled:
            return
        bad = [c for c in self.criteria if c not in VALID_CRITERIA]
        if bad or not self.criteria:
            raise ValueError(f"beaching.criteria must be a non-empty subset of {VALID_CRITERIA}, "
                             f"got {self.criteria!r}")
        if self.resuspension not in RESUSP_CODES:
            raise ValueError(f"beaching.resuspension must be one of {tuple(RESUSP_CODES)}, "
                             f"got {self.resuspension!r}")
        if "stochastic" in self.criteria and (self.t_beach is None or self.t_beach <= 0):
            raise ValueError("beaching.t_beach (s) must be > 0 when the 'stochastic' criterion is enabled")
        if self.resuspension in ("stochastic", "auto_or_stochastic") and (
                self.t_resuspend is None or self.t_resuspend <= 0):
            raise ValueError("beaching.t_resuspend (s) must be > 0 for stochastic resuspension")
        if self.min_wet_steps < 1:
            raise ValueError(f"beaching.min_wet_steps must be >= 1, got {self.min_wet_steps}")
        if self.depth_min <= 0:
            raise ValueError(f"beaching.depth_min must be > 0, got {self.depth_min}")
        if self.seed is not None and not (0 <= int(self.seed) < 2 ** 64):
            raise ValueError("beaching.seed must be in [0, 2**64)")


class BeachRunConfig(NamedTuple):
    """Per-run constants of the hook (beaching.py:79-93)."""
    cfg: Any
    crit: frozenset
    need_topo: bool
    elem_coastal: Optional[np.ndarray]
    seed: int
    zone: float
    pid_offset: int = 0


def make_run_config(cfg: BeachingConfig, mesh, diffusion_seed: int = 0,
                    particle_offset: int = 0) -> BeachRunConfig:
    """The run's startup gate (tracking.py:2080-2101): topology is built when
    the coastal or stochastic criterion is on; the seed falls back to the
    diffusion seed and the zone depth to twice ``depth_min``."""
    crit = frozenset(cfg.criteria)
    need_topo = bool({"coastal_element", "stochastic"} & crit)
    elem_coastal = None
    if need_topo:
        build_boundary_info(mesh)
        elem_coastal = mesh._elem_is_coastal
    seed = cfg.seed if cfg.seed is not None else diffusion_seed
    zone = cfg.zone_depth if cfg.zone_depth is not None else 2.0 * cfg.depth_min
    return BeachRunConfig(cfg=cfg, crit=crit, need_topo=need_topo, elem_coastal=elem_coastal,
                          seed=int(seed), zone=float(zone), pid_offset=int(particle_offset))


def beach_args(run_cfg: BeachRunConfig, real_id: int, step_i: int, dt: float) -> N.BeachArgs:
    """The kernel's argument block for one hook call.  The probabilities are
    1 - exp(-|dt| / t) with the host's exp, as the reference evaluates them
    (beaching.py:135, :170)."""
    cfg = run_cfg.cfg
    crit = run_cfg.crit
    a = N.BeachArgs()
    a.use_depth = int("depth" in crit)
    a.use_coastal = int("coastal_element" in crit)
    a.use_stochastic = int("stochastic" in crit)
    a.on_failure = int("on_failure" in crit)
    a.resuspension = RESUSP_CODES[cfg.resuspension]
    a.min_wet_steps = int(cfg.min_wet_steps)
    a.depth_min = float(cfg.depth_min)
    a.zone_depth = float(run_cfg.zone)
    a.rewet_hysteresis = float(cfg.rewet_hysteresis)
    t_b = float(cfg.t_beach or 0.0)
    t_r = float(cfg.t_resuspend or 0.0)
    a.p_beach = float(1.0 - np.exp(-abs(dt) / t_b)) if t_b > 0 else 0.0
    a.p_resusp = float(1.0 - np.exp(-abs(dt) / t_r)) if t_r > 0 else 0.0
    a.seed = int(run_cfg.seed) % (1 << 64)
    a.real_id = int(real_id)
    a.step_i = int(step_i)
    a.pid_offset = int(run_cfg.pid_offset)
    return a


def _payload_node(vel, get):
    """A node array of the step's payload as the reference reads it: a
    LazyLerpField's is (1 - alpha) a + alpha b of its pair, in the arrays'
    own dtype (io.py:68-117, :499-513)."""
    if all(hasattr(vel, k) for k in ("vel_a", "vel_b", "alpha")):
        a, b = get(vel.vel_a), get(vel.vel_b)
        if a is None or b is None:
            return None
        return (1.0 - float(vel.alpha)) * np.asarray(a) + float(vel.alpha) * np.asarray(b)
    return get(vel)


def payload_surfaces(vel, cfg: BeachingConfig):
    """(eta, dry_mask) node arrays the hook reads from the payload
    (tracking.py:236-327): eta when ``use_eta``, the surface layer of the
    ``dry_mask_var`` scalar when the payload carries it; None otherwise."""
    eta = dry = None
    if cfg.use_eta:
        eta = _payload_node(vel, lambda v: getattr(v, "eta", None))
        if eta is None:
            raise ValueError("beaching.use_eta needs the payload's eta")
    if cfg.dry_mask_var:
        def surface(v):
            x = (getattr(v, "scalars", None) or {}).get(cfg.dry_mask_var)
            if x is None:
                return None
            x = np.asarray(x)
            return x[0] if x.ndim > 1 else x
        dry = _payload_node(vel, surface)
    return eta, dry


def apply_beaching_hook(state: ParticleState, prev_status, mesh, vel, run_cfg: BeachRunConfig, wet_streak,
                        real_id: int, step_i: int, dt: float, ctx=None):
    """Beaching + resuspension of a post-step state (tracking.py:199-364).
    Returns ``(state, wet_streak)``; the input state is not modified."""
    a = beach_args(run_cfg, real_id, step_i, dt)
    P = state.n_particles
    wet = (np.zeros(P, np.int32) if wet_streak is None
           else np.ascontiguousarray(wet_streak, dtype=np.int32))
    if P == 0:
        return state, wet.copy()
    ctx = ctx or default_context()
    ctx.ensure_mesh(mesh)
    if run_cfg.need_topo:
        ctx.ensure_coastal(mesh, run_cfg.elem_coastal)
    ctx.upload_particles(state.lon, state.lat, state.z, state.status, state.nearest_node,
                         fr=state.failure_reason)
    ctx.beach_state_upload(prev_status, wet)
    ctx.beach_surface(*payload_surfaces(vel, run_cfg.cfg))
    ctx.beach(a)
    out = ctx.download_particles()
    ws = ctx.beach_state_download()
    err = ctx.device_errors()
    if err:
        raise N.KcError(N.KC_ERR_DEVICE, N.describe_device_errors(err))
    return state.replace(status=out["status"], nearest_node=out["nearest_node"],
                         failure_reason=None if state.failure_reason is None else out["failure_reason"]), ws
