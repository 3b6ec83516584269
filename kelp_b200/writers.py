"""Trajectory output and restart checkpoints of a tracking run.

Mirrors KELP's ``TrajectoryWriter`` / ``load_restart``
(``src/kelp/writers.py:1209-1716``, ``:1541``): one observation per record
(``time``, ``lon``, ``lat``, ``z``, ``status``, ``vel_u``/``vel_v``/``vel_w``,
``failure_reason``), the release positions, and a restart block with the
reference's variable names (``restart_lon`` ... ``restart_valid``).  netCDF4
and zarr are not available to this package, so the store is a directory of
``.npy`` arrays (``<path>/``): observations are appended as one file per
record and gathered on read; a checkpoint is written to a temporary file and
moved into place, so an interrupted checkpoint leaves the previous one valid
(the reference's ``restart_valid`` protocol, writers.py:584-662).
"""
from __future__ import annotations

import json
import os
from typing import Dict, Optional

import numpy as np

from .particles import ParticleState

_OBS = ("lon", "lat", "z", "status")


class TrajectoryWriter:
    """Streaming trajectory store with restart checkpoints (writers.py:1209)."""

    def __init__(self, path: str, n_particles: int, metadata: Optional[Dict[str, object]] = None):
        self.path = path
        self.n_particles = int(n_particles)
        self.metadata = dict(metadata or {})
        self._n_obs = 0

    def open(self) -> "TrajectoryWriter":
        """Open (or reopen) the store.  Reopening a store that holds a
        checkpoint resumes numbering at the checkpoint's record count: records
        written after the checkpoint (by a run that stopped before its next
        one) are dropped, as the resumed run writes them again."""
        obs_dir = os.path.join(self.path, "obs")
        os.makedirs(obs_dir, exist_ok=True)
        self._write_json("attrs.json", {"n_particles": self.n_particles, **self.metadata})
        files = sorted(f for f in os.listdir(obs_dir) if f.endswith(".npz") and ".tmp" not in f)
        kept = len(files)
        rst = os.path.join(self.path, "restart.npz")
        if os.path.exists(rst):
            with np.load(rst) as d:
                if "restart_n_obs" in d.files:
                    kept = min(kept, int(d["restart_n_obs"]))
        for f in files[kept:]:
            os.remove(os.path.join(obs_dir, f))
        self._n_obs = kept
        return self

    def __enter__(self):
        return self.open()

    def __exit__(self, *exc):
        self.close()

    def close(self) -> None:
        pass

    @property
    def n_obs(self) -> int:
        return self._n_obs

    def _write_json(self, name, obj):
        tmp = os.path.join(self.path, name + ".tmp")
        with open(tmp, "w") as fh:
            json.dump(obj, fh)
        os.replace(tmp, os.path.join(self.path, name))

    def _check(self, a, name):
        a = np.asarray(a)
        if a.shape != (self.n_particles,):
            raise ValueError(f"{name}: expected shape ({self.n_particles},), got {a.shape}")
        return a

    def append(self, state: ParticleState, time_value: float) -> None:
        """One observation of every particle (writers.py:1275-1304)."""
        if not np.isfinite(float(time_value)):
            raise ValueError(f"time_value must be finite, got {time_value!r}")
        rec = {"time": np.float64(time_value)}
        for name in _OBS:
            rec[name] = self._check(getattr(state, name), name)
        for src, dst in (("u", "vel_u"), ("v", "vel_v"), ("w", "vel_w"), ("failure_reason", "failure_reason")):
            val = getattr(state, src, None)
            if val is not None:
                rec[dst] = self._check(val, src)
        path = os.path.join(self.path, "obs", f"{self._n_obs:08d}.npz")
        np.savez(path + ".tmp.npz", **rec)
        os.replace(path + ".tmp.npz", path)
        self._n_obs += 1

    def write_release(self, lon, lat, z, time) -> None:
        np.savez(os.path.join(self.path, "release.npz"), release_lon=self._check(lon, "lon"),
                 release_lat=self._check(lat, "lat"), release_z=self._check(z, "z"),
                 release_time=np.asarray(time, dtype=np.float64))

    def write_checkpoint(self, state: ParticleState, step_i: int, file_idx: int, wet_streak=None,
                         release_step=None, particle_offset: Optional[int] = None,
                         uv_vertical: Optional[str] = None) -> None:
        """The restart block (writers.py:567-662): positions, status, anchors,
        the global step and record index, and the optional failure reasons,
        release steps, carried elements, release positions and wet streaks."""
        blk = {"restart_lon": self._check(state.lon, "lon").astype(np.float64),
               "restart_lat": self._check(state.lat, "lat").astype(np.float64),
               "restart_z": self._check(state.z, "z").astype(np.float64),
               "restart_status": self._check(state.status, "status").astype(np.int32),
               "restart_nearest_node": self._check(state.nearest_node, "nearest_node").astype(np.int32),
               "restart_step_i": np.int64(step_i), "restart_file_idx": np.int64(file_idx),
               "restart_n_obs": np.int64(self._n_obs)}   # the records that belong to this checkpoint
        optional = []
        for name, val, dt in (("failure_reason", state.failure_reason, np.int8),
                              ("release_step", release_step, np.int32),
                              ("elem", state.elem, np.int32),
                              ("release_lon", getattr(state, "release_lon", None), np.float64),
                              ("release_lat", getattr(state, "release_lat", None), np.float64),
                              ("release_z", getattr(state, "release_z", None), np.float64),
                              ("wet_streak", wet_streak, np.int32)):
            if val is not None:
                blk["restart_" + name] = self._check(val, name).astype(dt)
                optional.append("restart_" + name)
        if particle_offset is not None:
            blk["restart_particle_offset"] = np.int64(particle_offset)
        if uv_vertical is not None:
            blk["restart_uv_vertical"] = np.array(str(uv_vertical))
        blk["restart_optional"] = np.array(" ".join(optional))
        tmp = os.path.join(self.path, "restart.tmp.npz")
        np.savez(tmp, **blk)
        os.replace(tmp, os.path.join(self.path, "restart.npz"))   # the valid flag: the file exists whole


def read_trajectory(path: str) -> dict:
    """The observations of a store as (n_obs, P) arrays plus ``time`` (n_obs,)."""
    obs_dir = os.path.join(path, "obs")
    files = sorted(f for f in os.listdir(obs_dir) if f.endswith(".npz") and ".tmp" not in f)
    recs = [dict(np.load(os.path.join(obs_dir, f))) for f in files]
    out = {}
    for k in recs[0] if recs else ():
        out[k] = np.stack([r[k] for r in recs]) if recs[0][k].ndim else np.array([r[k] for r in recs])
    rel = os.path.join(path, "release.npz")
    if os.path.exists(rel):
        out.update(dict(np.load(rel)))
    return out


def load_restart(path: str) -> dict:
    """The last valid checkpoint (writers.py:1541-1716): ``state``,
    ``step_i``, ``file_idx``, ``wet_streak``, ``release_step`` (also on
    ``state.release_step``), ``particle_offset``, ``uv_vertical``,
    ``rotation_angles`` (None: rotated frames are not written here); the
    carried elements and release positions are attached to the state."""
    f = os.path.join(path, "restart.npz")
    if not os.path.exists(f):
        raise ValueError(f"No valid restart checkpoint in {path}")
    d = dict(np.load(f))
    get = lambda k: d.get("restart_" + k)
    state = ParticleState(lon=get("lon"), lat=get("lat"), z=get("z"), status=get("status"),
                          nearest_node=get("nearest_node"), failure_reason=get("failure_reason"),
                          elem=get("elem"), release_step=get("release_step"),
                          release_lon=get("release_lon"), release_lat=get("release_lat"), release_z=get("release_z"))
    po = get("particle_offset")
    uv = get("uv_vertical")
    return {"state": state, "step_i": int(get("step_i")), "file_idx": int(get("file_idx")),
            "wet_streak": get("wet_streak"), "release_step": get("release_step"),
            "particle_offset": None if po is None else int(po), "uv_vertical": None if uv is None else str(uv),
            "rotation_angles": None}
