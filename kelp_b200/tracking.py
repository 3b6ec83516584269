"""The caller side of the step on the B200: a device-resident tracking loop.

``Tracker.run`` follows the per-step order of KELP's
``tracking.run_single_realization`` (``src/kelp/tracking.py:2384-2860``):
delayed release (in the step kernel), the velocity payload of the step's time
bracket, the step, the beaching hook, the clock, and a record every
``output_freq`` global steps; only the records cross PCIe.  The mesh, the
snapshots in use (a ring of device slots) and the particles stay resident;
the particles are re-sorted by hash cell every ``sort_every`` steps (results do
not depend on the order).  Several realizations that start together run as
one array with per-particle realization ids (``run_realizations``), each with
the draws of its own run.

The time axis restates ``_resolve_time_bracket`` / ``_build_vel_payload``
(``tracking.py:2910-3206``): brackets on the record times, ``stop`` or
``cycle`` (period = span of the records + the last interval) when the records
are exhausted, the on-snapshot shifts of forward and backward steps within the
clock's roundoff band (``_snapshot_band``, ``:1667``).

``run_tracking(config, ...)`` takes KELP's configuration schema (the
``mode``, ``numerics`` (with ``diffusion`` and ``beaching``) and ``time``
sections, as a dict or YAML file) with ``numerics.backend: cuda``.  KELP's
readers (netCDF / zarr / healpy) are not part of this package: the mesh, the
snapshot records and the seeds are passed in, or read from ``.npz`` files named
in the ``data`` section (``mesh_npz``, ``velocity_npz``, ``seeds``).
"""
from __future__ import annotations

import os
from dataclasses import dataclass, field
from typing import List, Optional, Sequence

import numpy as np

from . import _native as N
from . import integrators as KI
from .beaching import BeachingConfig, beach_args, make_run_config, payload_surfaces
from .device import default_context
from .diffusion import DiffusionStepArgs
from .fields import LazyLerpField, VelocityField
from .particles import ParticleState, ParticleStatus, make_state

# ---------------------------------------------------------------------------
# time axis
# ---------------------------------------------------------------------------


def snapshot_band(dt: float) -> float:
    """Seconds within which a step that reaches a record is on it
    (tracking.py:1667-1679)."""
    return 1e-5 * max(abs(float(dt)), 1.0)


def _last_interval(ft) -> float:
    return float(ft[-1] - ft[-2]) if len(ft) > 1 else 1.0


def cycle_period(file_times) -> float:
    """Period of ``on_exhausted: cycle``: the span of the records plus the
    last interval (tracking.py:2910-2916)."""
    ft = np.asarray(file_times, dtype=np.float64)
    return float(ft[-1] - ft[0]) + _last_interval(ft)


def wrap_time(t: float, file_times, on_exhausted: str) -> float:
    ft = np.asarray(file_times, dtype=np.float64)
    if on_exhausted != "cycle":
        return float(t)
    return float(ft[0] + ((t - ft[0]) % cycle_period(ft)))


def resolve_time_bracket(t: float, file_times, on_exhausted: str = "stop", direction: int = 1,
                         snap: float = 0.0):
    """``(idx_a, idx_b, ta, tb, t_in_bracket)`` of the records around time
    ``t``, or None past the records in ``stop`` mode (tracking.py:2947-3071).

    A forward query within ``snap`` below a record starts the interval above
    it; a backward query on (or within the band above) a record takes the
    interval below it, its position at the top."""
    ft = np.asarray(file_times, dtype=np.float64)
    n = ft.size
    cyc = on_exhausted == "cycle"
    tw = wrap_time(t, ft, on_exhausted)
    if not cyc and (tw < ft[0] - 1e-6 or tw > ft[-1] + 1e-6):
        return None
    ib = int(np.searchsorted(ft, tw, side="right"))
    ia = ib - 1
    if cyc:
        ia, ib = ia % n, ib % n
    else:
        ia, ib = max(0, min(ia, n - 1)), max(0, min(ib, n - 1))
    ta, tb = float(ft[ia]), float(ft[ib])
    if cyc and tb <= ta:
        tb = ta + _last_interval(ft)
    if direction > 0 and snap > 0.0 and ia != ib and tb - tw <= snap:
        s = ib
        s_next = (s + 1) % n if cyc else min(s + 1, n - 1)
        ta2, tb2 = float(ft[s]), float(ft[s_next])
        if cyc and tb2 <= ta2:
            tb2 = ta2 + _last_interval(ft)
        return s, s_next, ta2, tb2, ta2
    if direction < 0 and tw <= ta + max(1e-6, snap):
        ib2 = ia
        ia2 = (ia - 1) % n if cyc else ia - 1
        if ia2 < 0 or ia2 == ib2:
            return ib2, ib2, ta, ta, tw
        ta2, tb2 = float(ft[ia2]), float(ft[ib2])
        if tb2 <= ta2:
            tb2 = ta2 + _last_interval(ft)
        return ia2, ib2, ta2, tb2, tb2
    return ia, ib, ta, tb, tw


def resolve_recon_stencil(bracket, n_records: int):
    """tracking.py:3075-3094 _resolve_recon_stencil: the 4-record PCHIP
    stencil ``((idx_a - 1, idx_a, idx_b, idx_b + 1), t_in_bracket)`` of a
    bracket, or None at the first / last interval, on a record, or across a
    cycle seam (the step then blends linearly)."""
    ia, ib = int(bracket[0]), int(bracket[1])
    if ib != ia + 1:
        return None
    if ia - 1 < 0 or ib + 1 >= n_records:
        return None
    return (ia - 1, ia, ib, ib + 1), float(bracket[4])


def step_end_on_record(sim_time: float, pos: float, dt_to_next: float, direction: int, file_times,
                       on_exhausted: str) -> float:
    """tracking.py:2930-2944 _step_end_on_record: the clock after a step that
    ends on the record ahead (``pos`` is the step's start in the bracket's
    frame; under ``cycle`` the offset is taken modulo the period)."""
    delta = pos - wrap_time(sim_time, file_times, on_exhausted)
    if on_exhausted == "cycle":
        period = cycle_period(file_times)
        delta -= period * np.round(delta / period)
    return sim_time + delta + dt_to_next * direction


def record_view(s: dict, prev_status: np.ndarray, direction: int) -> dict:
    """The recorded values of one observation (output format 2): dormant
    (NOT_RELEASED) rows get NaN positions and velocities
    (core/release.py:132-167), a velocity exists only where the particle was
    ALIVE through the whole step (:170-201), and a backward run records the
    flow velocity (tracking.py:2770-2776)."""
    out = dict(s)
    dormant = s["status"] == int(ParticleStatus.NOT_RELEASED)
    if np.any(dormant):
        for k in ("lon", "lat", "z", "u", "v", "w"):
            if out.get(k) is not None:
                out[k] = np.where(dormant, np.nan, np.asarray(out[k], dtype=np.float64))
    alive = int(ParticleStatus.ALIVE)
    bad = (s["status"] != alive) | (np.asarray(prev_status) != alive)
    for k in ("u", "v", "w"):
        if out.get(k) is not None:
            v = np.where(bad, np.nan, np.asarray(out[k], dtype=np.float64))
            out[k] = -v if direction < 0 else v
    return out


def vel_payload(bracket, fields: Sequence, direction: int = 1):
    """``(vel, vel_next, dt_to_next)`` of a bracket (tracking.py:3136-3206):
    the field at the query time (a snapshot, or a lazy pair with alpha), the
    snapshot the step moves toward and the seconds to it; a degenerate bracket
    gives the steady field."""
    ia, ib, ta, tb, tw = bracket
    a = fields[ia]
    if ia == ib:
        return a, None, None
    b = fields[ib]
    interval = tb - ta
    alpha = (tw - ta) / interval if interval > 0 else 0.0
    if abs(alpha) < 1e-12:
        vel = a
    elif abs(alpha - 1.0) < 1e-12:
        vel = b
    else:
        vel = LazyLerpField(a, b, alpha)
    if direction >= 0:
        return vel, b, tb - tw
    dt_prev = tw - ta
    if dt_prev <= 1e-6:
        return vel, None, None
    return vel, a, dt_prev


# ---------------------------------------------------------------------------
# records
# ---------------------------------------------------------------------------


@dataclass
class TrajectoryRecord:
    """Snapshots of one realization at its record steps (tracking.py:50-80):
    positions, velocity diagnostics, status and failure reason per record,
    times in seconds on the forcing axis at the end of the recorded step."""
    lons: List[np.ndarray] = field(default_factory=list)
    lats: List[np.ndarray] = field(default_factory=list)
    zs: List[np.ndarray] = field(default_factory=list)
    times: List[float] = field(default_factory=list)
    us: List[np.ndarray] = field(default_factory=list)
    vs: List[np.ndarray] = field(default_factory=list)
    ws: List[np.ndarray] = field(default_factory=list)
    status: List[np.ndarray] = field(default_factory=list)
    failure_reason: List[np.ndarray] = field(default_factory=list)
    release_lon: Optional[np.ndarray] = None
    release_lat: Optional[np.ndarray] = None
    release_z: Optional[np.ndarray] = None
    release_time: Optional[np.ndarray] = None

    def append(self, s: dict, t: float, dims: int) -> None:
        self.lons.append(s["lon"])
        self.lats.append(s["lat"])
        self.zs.append(s["z"])
        self.times.append(float(t))
        self.us.append(s["u"])
        self.vs.append(s["v"])
        if dims == 3:
            self.ws.append(s["w"])
        self.status.append(s["status"])
        self.failure_reason.append(s["failure_reason"])

    def as_arrays(self) -> dict:
        """(n_records, P) arrays of every recorded quantity."""
        out = {"time": np.asarray(self.times)}
        for name in ("lons", "lats", "zs", "us", "vs", "ws", "status", "failure_reason"):
            seq = getattr(self, name)
            if seq:
                out[name] = np.stack(seq)
        return out


# ---------------------------------------------------------------------------
# the device-resident loop
# ---------------------------------------------------------------------------


@dataclass
class RunResult:
    records: List[TrajectoryRecord]
    final: List[ParticleState]
    wet_streak: List[Optional[np.ndarray]]
    steps: int


class Tracker:
    """A tracking run whose mesh, snapshots and particles stay on the GPU.

    ``fields`` are the snapshot records (``VelocityField``-like, node layout)
    at ``file_times`` seconds; ``integrator`` is euler / rk2 / rk4;
    ``diffusion`` a ``DiffusionConfig``-like object (``enabled``, ``scheme``
    uniform, ``kh_zonal``, ``kh_meridional``, ``seed``) or None;
    ``beaching`` a ``BeachingConfig`` or None.  ``precision`` and ``snapshots``
    select the numerical form as for the step functions.  ``elem_search``
    "walk" carries each particle's containing element from step to step
    (tracking.py:2236-2253: seeded once at the start by the local search
    around the exact anchor unless the initial state carries them).
    ``temporal_reconstruction`` "pchip" hands the RK stages the 4-record
    monotone-cubic stencil wherever one exists (tracking.py:2415-2436).
    ``prefetch`` starts uploading the records of the next few steps as soon
    as a step is launched (kc_field_upload_async), so an upload runs beside
    the steps before the record is needed instead of in front of it."""

    def __init__(self, mesh, fields: Sequence, file_times, *, integrator: str = "rk2", dt: float,
                 time_dir: float = 1.0, uv_interp: str = "barycentric", w_interp: str = "barycentric",
                 diffusion=None, beaching: Optional[BeachingConfig] = None, on_exhausted: str = "stop",
                 precision: str = "plain", snapshots: Optional[str] = None, sort_every: int = 16,
                 elem_search: str = "local", temporal_reconstruction: str = "linear", prefetch: bool = True,
                 ctx=None):
        if integrator not in ("euler", "rk2", "rk4"):
            raise NotImplementedError(f"integrator {integrator!r} is not built on the CUDA backend")
        if on_exhausted not in ("stop", "cycle"):
            raise ValueError(f"on_exhausted must be 'stop' or 'cycle', got {on_exhausted!r}")
        if float(dt) <= 0:
            raise ValueError(f"dt must be > 0, got {dt!r}")
        if float(time_dir) not in (1.0, -1.0):
            raise ValueError(f"time_dir must be +1 or -1, got {time_dir!r}")
        if elem_search not in ("local", "walk"):
            raise ValueError(f"elem_search must be 'local' or 'walk', got {elem_search!r}")
        if temporal_reconstruction not in ("linear", "pchip"):
            raise ValueError(f"temporal_reconstruction must be 'linear' or 'pchip', got {temporal_reconstruction!r}")
        self.pchip = temporal_reconstruction == "pchip"
        self.prefetch = bool(prefetch)
        self.prefetch_steps = 4   # steps ahead whose records are uploaded early (at most 4 records)
        self.walk = elem_search == "walk"
        # sigma meshes: every step gets the surfaces at its start and end times
        # from one function of time (tracking.py:2562-2596), evaluated on the
        # device from the resident records (_surface)
        self.sigma = KI._sigma_mesh(mesh)
        self.mesh = mesh
        self.fields = list(fields)
        self.file_times = np.asarray(file_times, dtype=np.float64)
        if self.file_times.size != len(self.fields) or self.file_times.size == 0:
            raise ValueError("one record time per snapshot is required")
        if np.any(np.diff(self.file_times) <= 0):
            raise ValueError("record times must increase")
        self.integrator = integrator
        self.dt = float(dt)
        self.direction = 1 if float(time_dir) > 0 else -1
        self.kw = {"uv_interp": uv_interp, "w_interp": w_interp, "cuda_precision": precision}
        if snapshots is not None:
            self.kw["cuda_snapshots"] = snapshots
        self.diffusion = diffusion if (diffusion is not None and getattr(diffusion, "enabled", True)) else None
        if self.diffusion is not None:
            if getattr(self.diffusion, "scheme", "uniform") != "uniform":
                raise NotImplementedError("only the uniform-Kh split kick is built on the CUDA backend")
            if getattr(self.diffusion, "composition", "split") != "split":
                raise NotImplementedError("only the split kick composition is built on the CUDA backend")
        self.beaching = beaching if (beaching is not None and beaching.enabled) else None
        self.on_exhausted = on_exhausted
        self.sort_every = int(sort_every)
        self.ctx = ctx or default_context()
        self.dims = 3 if getattr(self.fields[0], "w", None) is not None else 2

    def _surface(self, which: int, t: float, multistage: bool, steady: bool, band: float) -> None:
        """The sigma surface at time ``t`` as tracking.py:3097-3133
        _eta_at_time defines it -- a record itself on a record, the PCHIP
        stencil's value where PCHIP is on for a multistage step and a stencil
        exists, else the linear blend of the bracket -- computed on the device
        from the resident records into the start (which 0) or end (1)
        surface of the next step; outside the data the step keeps the
        payload's own surface."""
        ctx, ft = self.ctx, self.file_times
        b = resolve_time_bracket(t, ft, self.on_exhausted, self.direction, band)
        if b is None:
            ctx.sigma_surface_records(which, 0, steady=steady)
            return
        ia, ib, ta, tb, tw = b
        interval = tb - ta
        alpha = (tw - ta) / interval if interval > 0 else 0.0
        times, q = None, 0.0
        if ia == ib or abs(alpha) < 1e-12:
            recs, kind = [ia], 1
        elif abs(alpha - 1.0) < 1e-12:
            recs, kind = [ib], 1
        else:
            stencil = resolve_recon_stencil(b, ft.size) if (self.pchip and multistage) else None
            if stencil is not None:
                recs, kind = list(stencil[0]), 3
                times, q = [float(ft[i]) for i in recs], float(stencil[1])
            else:
                recs, kind = [ia, ib], 2
        slots = ctx.slots_for([self.fields[i] for i in recs], KI.snapshot_storage(self.kw))
        ctx.sigma_surface_records(which, kind, slots, alpha, times, q, steady)

    def _diffusion_args(self, realization: int, step_i: int, particle_offset: int):
        """The step's DiffusionStepArgs as tracking.py:2595-2611 builds them
        (None when diffusion is off): Kh, the draws' keys, the Az switch and
        source."""
        d = self.diffusion
        if d is None:
            return None
        return DiffusionStepArgs(
            scheme="uniform", kh_x=float(getattr(d, "kh_zonal", getattr(d, "kh_x", 0.0))),
            kh_y=float(getattr(d, "kh_meridional", getattr(d, "kh_y", 0.0))), seed=int(d.seed),
            real_id=int(realization), step_i=int(step_i),
            az_enabled=bool(getattr(d, "az_enabled", False)), az_const=float(getattr(d, "az_const", 0.0)),
            az_requires_field=bool(getattr(d, "var_az", None)) or bool(getattr(d, "az_requires_field", False)),
            pid_offset=int(particle_offset))

    def run(self, init_state: ParticleState, n_steps: int, *, start_time: Optional[float] = None,
            realization_id: int = 0, start_step_i: int = 0, output_freq: int = 1, particle_offset: int = 0,
            release_step: Optional[np.ndarray] = None, start_wet_streak=None, writer=None,
            checkpoint_freq: int = 0) -> RunResult:
        """One realization; the result holds one record and final state.
        ``writer`` (kelp_b200.writers.TrajectoryWriter) receives every
        record and, every ``checkpoint_freq`` global steps, a restart
        checkpoint (tracking.py:2778-2792); resume with the checkpoint's
        state, ``start_step_i = step_i + 1`` and the wet streaks."""
        return self.run_realizations(init_state, n_steps, realizations=(realization_id,), start_time=start_time,
                                     start_step_i=start_step_i, output_freq=output_freq,
                                     particle_offset=particle_offset, release_step=release_step,
                                     start_wet_streak=start_wet_streak, writer=writer,
                                     checkpoint_freq=checkpoint_freq)

    def run_realizations(self, init_state: ParticleState, n_steps: int, *, realizations: Sequence[int] = (0,),
                         start_time: Optional[float] = None, start_step_i: int = 0, output_freq: int = 1,
                         particle_offset: int = 0, release_step: Optional[np.ndarray] = None,
                         start_wet_streak=None, writer=None, checkpoint_freq: int = 0) -> RunResult:
        """Every realization of ``realizations`` from the same seeds and start
        time, as one particle array (per-particle realization ids): one record
        and final state per realization, each as its own run would give."""
        ctx, mesh = self.ctx, self.mesh
        R = len(realizations)
        if writer is not None and R != 1:
            raise ValueError("a trajectory writer holds one realization: run them one by one")
        P = init_state.n_particles
        ft = self.file_times
        t0 = float(ft[0] if start_time is None else start_time)
        band = snapshot_band(self.dt)
        # resident particles: realization-major copies of the seeds
        rep = (lambda a: np.concatenate([np.asarray(a)] * R)) if R > 1 else (lambda a: np.asarray(a))
        fr0 = init_state.failure_reason if init_state.failure_reason is not None else np.zeros(P, np.int8)
        rs = None
        if release_step is not None:
            rs = rep(np.asarray(release_step, dtype=np.int32))
        elif init_state.release_step is not None:
            rs = rep(np.asarray(init_state.release_step, dtype=np.int32))
        ctx.ensure_mesh(mesh)
        ctx.upload_particles(rep(init_state.lon), rep(init_state.lat), rep(init_state.z), rep(init_state.status),
                             rep(init_state.nearest_node), rep(fr0), rep(np.arange(P, dtype=np.int64)), rs)
        if R > 1:
            ctx.set_realization(np.repeat(np.asarray(realizations, dtype=np.int32), P))
        if self.walk:
            ctx.ensure_elem_neighbors(mesh)
            e0 = init_state.elem
            if e0 is None:   # one local search around the exact anchor at the start
                e0 = ctx.find_elements(init_state.lon, init_state.lat)
            ctx.set_elem(rep(np.asarray(e0, dtype=np.int32)))
        beach_cfg = None
        surfaces = False
        if self.beaching is not None:
            surfaces = bool(self.beaching.use_eta or self.beaching.dry_mask_var)
            seed = int(getattr(self.diffusion, "seed", 0)) if self.diffusion is not None else 0
            beach_cfg = make_run_config(self.beaching, mesh, diffusion_seed=seed, particle_offset=particle_offset)
            if beach_cfg.need_topo:
                ctx.ensure_coastal(mesh, beach_cfg.elem_coastal)
            ws0 = None if start_wet_streak is None else rep(np.asarray(start_wet_streak, dtype=np.int32))
            ctx.beach_state_upload(None, ws0)
            ctx.beach_surface(None, None)
        records = [TrajectoryRecord() for _ in range(R)]
        for r in range(R):
            records[r].release_lon = np.array(init_state.lon, copy=True)
            records[r].release_lat = np.array(init_state.lat, copy=True)
            records[r].release_z = np.array(init_state.z, copy=True)
        sim_time = t0
        done = 0
        multistage = self.integrator in ("rk2", "rk4")
        for k in range(int(n_steps)):
            g = start_step_i + k
            bracket = resolve_time_bracket(sim_time, ft, self.on_exhausted, self.direction, band)
            if bracket is None:
                break
            stencil = resolve_recon_stencil(bracket, ft.size) if (self.pchip and multistage) else None
            vel, vnext, dtn = vel_payload(bracket, self.fields, self.direction)
            recon = None
            if stencil is not None:
                idx4, q_time = stencil
                recon = ([self.fields[i] for i in idx4], [float(ft[i]) for i in idx4], q_time,
                         float(self.direction))
            # tracking.py:2524-2560: a multistage step that reaches the record
            # ahead within the band ends ON it (its length is the distance,
            # the clock is set to the record); a step longer than the bracket
            # falls back to steady velocity
            step_len = self.dt
            sim_time_end = None
            if multistage and dtn is not None and abs(self.dt - dtn) <= band:
                step_len = dtn
                sim_time_end = step_end_on_record(sim_time, bracket[4], dtn, self.direction, ft, self.on_exhausted)
            elif dtn is not None and dtn < self.dt <= dtn + band:
                dtn = self.dt
            if dtn is not None and step_len > dtn:
                vnext, dtn, recon = None, None, None
            kw = dict(self.kw, vel_next=vnext, dt_to_next=dtn)
            if recon is not None:
                kw["recon"] = recon
            recording = (g + 1) % max(int(output_freq), 1) == 0
            if recording:   # the status after the release activation and before the step
                prev = ctx.download_status()
                if rs is not None:
                    prev[(prev == int(ParticleStatus.NOT_RELEASED)) & (rs <= g)] = int(ParticleStatus.ALIVE)
            if self.sort_every > 0 and k % self.sort_every == 0:
                ctx.sort()
            # the draws' keys: the realization of each particle (its own when R > 1)
            diff = self._diffusion_args(realizations[0], g, particle_offset)
            kw["diffusion"] = diff
            kick = KI._kick_args(diff)
            if self.sigma and self.dims == 3:
                steady = recon is None and vnext is None
                t_end = sim_time_end if sim_time_end is not None else sim_time + self.dt * self.direction
                self._surface(0, sim_time, multistage, steady, band)
                self._surface(1, t_end, multistage, steady, band)
            a, _ = KI.prepare_step(vel, mesh, step_len, float(self.direction), self.integrator, kw, ctx, kick=kick)
            a.global_step = g
            ctx.step(a)
            if beach_cfg is not None:
                if surfaces:
                    ctx.beach_surface(*payload_surfaces(vel, beach_cfg.cfg))
                ctx.beach(beach_args(beach_cfg, realizations[0], g, self.dt))
            sim_time = sim_time_end if sim_time_end is not None else sim_time + self.dt * self.direction
            if self.prefetch and k + 1 < int(n_steps):
                # the records of the next few steps upload while this one runs
                need, seen = [], set()
                for j in range(min(self.prefetch_steps, int(n_steps) - k - 1)):
                    nb = resolve_time_bracket(sim_time + j * self.dt * self.direction, ft, self.on_exhausted,
                                              self.direction, band)
                    if nb is None:
                        break
                    nst = resolve_recon_stencil(nb, ft.size) if (self.pchip and multistage) else None
                    for i in (nst[0] if nst is not None else (nb[0], nb[1])):
                        if i not in seen and len(seen) < 4:
                            seen.add(i)
                            need.append(self.fields[i])
                ctx.prefetch(need, KI.snapshot_storage(self.kw))
            done += 1
            s = None
            if recording:
                s = ctx.download_particles()
                t_rec = t0 + (g + 1 - start_step_i) * self.dt * self.direction
                view = record_view(s, prev, self.direction)
                for r in range(R):
                    sl = slice(r * P, (r + 1) * P)
                    records[r].append({k2: (None if v is None else v[sl]) for k2, v in view.items()}, t_rec,
                                      self.dims)
                if writer is not None:
                    writer.append(ParticleState(lon=view["lon"], lat=view["lat"], z=view["z"],
                                                status=view["status"], nearest_node=view["nearest_node"],
                                                u=view["u"], v=view["v"], w=view["w"] if self.dims == 3 else None,
                                                failure_reason=view["failure_reason"]), t_rec)
            if writer is not None and checkpoint_freq > 0 and (g + 1) % checkpoint_freq == 0:
                s = s if s is not None else ctx.download_particles()
                ck = init_state.replace(lon=s["lon"], lat=s["lat"], z=s["z"], status=s["status"],
                                        nearest_node=s["nearest_node"], failure_reason=s["failure_reason"],
                                        elem=ctx.get_elem() if self.walk else None)
                writer.write_checkpoint(ck, g, int(bracket[0]),
                                        wet_streak=ctx.beach_state_download() if beach_cfg is not None else None,
                                        release_step=rs, particle_offset=particle_offset,
                                        uv_vertical=getattr(self.fields[0], "uv_vertical", "layer"))
        if self.sigma and self.dims == 3:   # later steps on this context take their own surfaces again
            ctx.sigma_surfaces(None, None, False)
        err = ctx.device_errors()
        if err:
            raise N.KcError(N.KC_ERR_DEVICE, N.describe_device_errors(err))
        s = ctx.download_particles()
        ws = ctx.beach_state_download() if beach_cfg is not None else None
        el = ctx.get_elem() if self.walk else None
        finals, wets = [], []
        for r in range(R):
            sl = slice(r * P, (r + 1) * P)
            finals.append(init_state.replace(lon=s["lon"][sl], lat=s["lat"][sl], z=s["z"][sl],
                                             status=s["status"][sl], nearest_node=s["nearest_node"][sl],
                                             failure_reason=s["failure_reason"][sl], u=s["u"][sl], v=s["v"][sl],
                                             w=s["w"][sl] if self.dims == 3 else None,
                                             elem=None if el is None else el[sl]))
            wets.append(None if ws is None else ws[sl])
        return RunResult(records=records, final=finals, wet_streak=wets, steps=done)


# ---------------------------------------------------------------------------
# run_tracking: KELP's configuration schema, numerics.backend: cuda
# ---------------------------------------------------------------------------


def _section(cfg, name) -> dict:
    v = cfg.get(name) if isinstance(cfg, dict) else getattr(cfg, name, None)
    if v is None:
        return {}
    if isinstance(v, dict):
        return v
    return {k: getattr(v, k) for k in dir(v) if not k.startswith("_") and not callable(getattr(v, k))}


class _Diffusion:
    def __init__(self, d: dict):
        self.enabled = bool(d.get("enabled", False))
        self.scheme = d.get("scheme", "uniform")
        self.kh_zonal = float(d.get("kh_zonal", 0.0))
        self.kh_meridional = float(d.get("kh_meridional", 0.0))
        self.seed = int(d.get("seed", 0))
        self.composition = d.get("composition", "split")
        self.az_enabled = bool(d.get("az_enabled", False))
        self.az_const = float(d.get("az_const", 0.0))
        self.var_az = d.get("var_az")


def load_config(path_or_dict):
    """A configuration dict from a YAML path or a dict (KELP's schema)."""
    if isinstance(path_or_dict, (str, os.PathLike)):
        import yaml
        with open(path_or_dict) as fh:
            return yaml.safe_load(fh) or {}
    return path_or_dict


def load_mesh_npz(path: str):
    """A mesh from an .npz of KELP Mesh arrays (nodes_lon, nodes_lat, depth,
    elem_nodes and optionally z_levels): connectivity and the grid hash are
    built here."""
    from .mesh import make_mesh
    d = np.load(path)
    sigma = d["z_levels"] if "z_levels" in d else None
    return make_mesh(os.path.basename(path), d["nodes_lon"], d["nodes_lat"], d["depth"], d["elem_nodes"],
                     sigma=sigma)


def load_velocity_npz(path: str):
    """Snapshot records from an .npz with ``times`` (R,), ``u``, ``v`` (R, N) or
    (R, L, N) and optionally ``w`` (R, K, N), ``az`` (R, K, N) and
    ``uv_vertical``."""
    d = np.load(path)
    times = d["times"]
    placement = str(d["uv_vertical"]) if "uv_vertical" in d else "layer"
    fields = []
    for r in range(times.size):
        u, v = d["u"][r], d["v"][r]
        w = d["w"][r] if "w" in d else None
        az = d["az"][r] if "az" in d else None
        fields.append(VelocityField(u=u, v=v, w=w, eta=np.zeros(u.shape[-1]), uv_layout="node",
                                    uv_vertical=placement if w is not None else "layer", az=az))
    return fields, times


def load_seeds(path: str):
    """KELP's seed text file (lon lat [depth] [release_sec] per line, '#'
    comments) or an .npz with lon, lat[, z, release_sec]."""
    if path.endswith(".npz"):
        d = np.load(path)
        return d["lon"], d["lat"], d.get("z"), d.get("release_sec")
    rows = [l.split() for l in open(path) if l.strip() and not l.lstrip().startswith("#")]
    a = np.asarray([[float(x) for x in r] for r in rows])
    z = a[:, 2] if a.shape[1] > 2 else None
    rel = a[:, 3] if a.shape[1] > 3 else None
    return a[:, 0], a[:, 1], z, rel


def run_tracking(config, *, mesh=None, fields=None, file_times=None, seeds=None, ctx=None) -> List[TrajectoryRecord]:
    """Run every realization of a configuration on the GPU (tracking.py:3288).

    ``config``: KELP's schema (dict or YAML path): ``mode`` (Fdrift3D,
    time_dir), ``numerics`` (backend: cuda, integrator, dt, output_freq,
    uv_interp, w_interp, temporal_interp, diffusion, beaching, and the
    backend keywords cuda_precision / cuda_snapshots / sort_every), ``time``
    (start_time_idx, n_steps, on_exhausted, num_runs, run_interval, n_pulses,
    pulse_interval).  ``mesh``, ``fields`` + ``file_times`` and ``seeds``
    ((lon, lat[, z[, release_sec]])) come from the arguments or from the
    ``data`` section's ``mesh_npz``, ``velocity_npz`` and ``seeds`` paths.
    Realizations that start together run as one particle array."""
    cfg = load_config(config)
    mode, num, tim, data = (_section(cfg, k) for k in ("mode", "numerics", "time", "data"))
    backend = num.get("backend", "cuda")
    if backend != "cuda":
        raise ValueError(f"numerics.backend must be 'cuda' for this package, got {backend!r}")
    if not num.get("temporal_interp", True):
        raise NotImplementedError("the CUDA backend runs with temporal_interp: true")
    if num.get("periodic_lon") is not None or num.get("periodic_lat") is not None:
        raise NotImplementedError("periodic windows are not built on the CUDA backend")
    if mesh is None:
        mesh = load_mesh_npz(data["mesh_npz"])
    if fields is None:
        fields, file_times = load_velocity_npz(data["velocity_npz"])
    if seeds is None:
        seeds = load_seeds(data["seeds"])
    lon, lat = np.asarray(seeds[0], dtype=np.float64), np.asarray(seeds[1], dtype=np.float64)
    z = None if len(seeds) < 3 or seeds[2] is None else np.asarray(seeds[2], dtype=np.float64)
    rel_sec = None if len(seeds) < 4 or seeds[3] is None else np.asarray(seeds[3], dtype=np.float64)
    dt = float(num["dt"])
    ft = np.asarray(file_times, dtype=np.float64)
    direction = 1.0 if float(mode.get("time_dir", 1.0)) > 0 else -1.0
    # release pulses (TimeConfig n_pulses / pulse_interval) and per-seed release times
    n_pulses = int(tim.get("n_pulses", 1))
    pulse = float(tim.get("pulse_interval", 0.0))
    if n_pulses > 1:
        lon, lat = np.tile(lon, n_pulses), np.tile(lat, n_pulses)
        z = None if z is None else np.tile(z, n_pulses)
        base = np.zeros(lon.size) if rel_sec is None else np.tile(rel_sec, n_pulses)
        rel_sec = base + np.repeat(np.arange(n_pulses) * pulse, lon.size // n_pulses)
    state = make_state(lon, lat, z).replace(failure_reason=np.zeros(lon.size, np.int8))
    release_step = None
    if rel_sec is not None:
        release_step = np.ceil(rel_sec / dt - 1e-9).astype(np.int32)
        state = state.replace(status=np.where(release_step > 0, int(ParticleStatus.NOT_RELEASED),
                                              int(ParticleStatus.ALIVE)).astype(np.int32))
    diff = _Diffusion(num.get("diffusion") or {})
    beach = num.get("beaching") or {}
    beach_cfg = BeachingConfig(**beach) if beach else None
    tracker = Tracker(mesh, fields, ft, integrator=num.get("integrator", "rk2"), dt=dt, time_dir=direction,
                      uv_interp=num.get("uv_interp", "barycentric"), w_interp=num.get("w_interp", "barycentric"),
                      diffusion=diff if diff.enabled else None, beaching=beach_cfg,
                      on_exhausted=tim.get("on_exhausted", "stop"),
                      precision=num.get("cuda_precision", "plain"), snapshots=num.get("cuda_snapshots"),
                      sort_every=int(num.get("sort_every", 16)),
                      elem_search=num.get("elem_search", "local"),
                      temporal_reconstruction=num.get("temporal_reconstruction", "linear"), ctx=ctx)
    start_idx = int(tim.get("start_time_idx", 0))
    n_steps = tim.get("n_steps")
    if n_steps is None:
        end_idx = tim.get("end_time_idx")
        if end_idx is None:
            raise ValueError("time.n_steps (or time.end_time_idx) is required")
        n_steps = int(round((ft[int(end_idx)] - ft[start_idx]) / dt))
    num_runs = int(tim.get("num_runs", 1))
    run_interval = int(tim.get("run_interval", 0))
    output_freq = int(num.get("output_freq", 1))
    out: List[TrajectoryRecord] = []
    if run_interval == 0:
        res = tracker.run_realizations(state, int(n_steps), realizations=list(range(num_runs)),
                                       start_time=float(ft[start_idx]), output_freq=output_freq,
                                       release_step=release_step)
        out.extend(res.records)
    else:
        for r in range(num_runs):
            res = tracker.run(state, int(n_steps), start_time=float(ft[start_idx + r * run_interval]),
                              realization_id=r, output_freq=output_freq, release_step=release_step)
            out.extend(res.records)
    return out
