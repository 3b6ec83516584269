"""The named benchmark workloads: seeded synthetic inputs with the shapes of
KELP's benchmark configurations, and the per-step schedule a run loop feeds
the step kernel (bracket snapshots, bracket fraction, stage alphas), built
like ``tracking._build_vel_payload`` (``src/kelp/tracking.py:3136-3206``) with
``on_exhausted: cycle`` (period = span of the records + one interval).
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import Callable, List, Optional

import numpy as np

from . import _native as N
from . import synthetic as S


@dataclass
class Workload:
    name: str
    mesh: object
    snaps: list
    lon: np.ndarray
    lat: np.ndarray
    z: np.ndarray
    scheme: str
    dt: float
    interval: float                 # seconds between snapshots
    n_steps_run: int                # the configuration's horizon
    dims: int = 2
    w_interp: str = "nearest"
    kh: Optional[tuple] = None      # (kh_x, kh_y) of the split uniform kick
    seed: int = 0
    description: dict = field(default_factory=dict)

    @property
    def P(self) -> int:
        return self.lon.size

    def bracket(self, k: int):
        """(idx_a, idx_b, alpha0, dt_to_next) of global step k (forward)."""
        n = len(self.snaps)
        t = k * self.dt
        period = n * self.interval
        tw = t - period * np.floor(t / period)
        ia = int(np.floor(tw / self.interval + 1e-9)) % n
        ta = ia * self.interval
        alpha = (tw - ta) / self.interval
        if abs(alpha) < 1e-12:
            alpha = 0.0
        return ia, (ia + 1) % n, alpha, (ta + self.interval) - tw

    def step_args(self, k: int, slots) -> N.StepArgs:
        ia, ib, alpha0, dtn = self.bracket(k)
        a = N.StepArgs()
        a.scheme = {"euler": N.KC_EULER, "rk2": N.KC_RK2, "rk4": N.KC_RK4}[self.scheme]
        a.dims = self.dims
        a.slot_a, a.slot_b, a.slot_t = slots[ia], slots[ib], slots[ib]
        a.alpha0 = alpha0
        cc = {"euler": (0.0,), "rk2": (0.0, 0.5), "rk4": (0.0, 0.5, 0.5, 1.0)}[self.scheme]
        if self.scheme != "euler":
            for j, c in enumerate(cc):
                a.alpha_k[j] = float(c) * self.dt / dtn
        a.dt = self.dt
        a.time_dir = 1.0
        a.w_code = 0 if self.w_interp == "nearest" else 1
        if self.kh is not None:
            a.kick = 1
            a.kh_x, a.kh_y = self.kh
            a.seed, a.real_id, a.step_i, a.pid_offset = self.seed, 0, k, 0
        a.global_step = -1
        return a


def c1(P: int = 100_000, spacing: float = 0.5625) -> Workload:
    """2-D FESOM2-style: jittered (+-20 %) lon/lat lattice with a 30 % land mask
    (~127 k wet nodes, ~250 k triangles), u/v float32 on nodes (solid-body
    rotation + double gyre, 0.5 m/s), 2 snapshots 24 h apart cycled, 100 k
    particles uniform over the wet area, RK2, dt 1 h, 240 steps, no diffusion."""
    m = S.lattice_mesh(spacing, 80.0, jitter=0.2, land_frac=0.3)
    snaps = S.gyre_snapshots(m, 2, amp=0.5)
    lon, lat, z = S.release_uniform(m, P, seed=3)
    return Workload("c1_fesom2_2d_rk2", m, snaps, lon, lat, z, "rk2", 3600.0, 86400.0, 240,
                    description={"mesh": "jittered 0.5625 deg lattice, 30% land", "nodes": int(m.n_nodes),
                                 "elements": int(m.n_elements), "particles": P, "scheme": "rk2",
                                 "dt_s": 3600, "steps_run": 240, "fields": "f32 node u,v, 2 snapshots 24 h"})


WORKLOADS: dict = {"c1": c1}
