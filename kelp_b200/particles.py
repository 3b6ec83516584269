"""Particle state: the structure-of-arrays record every step consumes and returns.

Mirrors KELP's ``src/kelp/core/particles.py``: status codes (``:18-31``), the
per-particle failure reason (``:34-71``), ``ParticleState`` (``:153``) with its
immutable ``replace`` idiom, and ``make_state`` (``:384``).  A step never mutates
its input state; it returns a new one whose arrays are freshly allocated.
"""
from __future__ import annotations

from dataclasses import dataclass, fields
from enum import IntEnum
from typing import Optional

import numpy as np


class ParticleStatus(IntEnum):
    ALIVE = 1
    BEACHED = 2
    OUTSIDE = 3
    NOT_RELEASED = 4


class FailureReason(IntEnum):
    NONE = 0
    INTERPOLATION_FAILED = 1
    OUT_OF_BOUNDS = 2
    SURFACE_HIT = 3
    BOTTOM_HIT = 4


@dataclass
class ParticleState:
    """Positions (degrees, metres positive down), status and diagnostics of P
    particles.  Optional arrays stay ``None`` when a feature is not tracked."""
    lon: np.ndarray
    lat: np.ndarray
    z: np.ndarray
    status: np.ndarray
    nearest_node: np.ndarray
    u: Optional[np.ndarray] = None
    v: Optional[np.ndarray] = None
    w: Optional[np.ndarray] = None
    failure_reason: Optional[np.ndarray] = None
    release_step: Optional[np.ndarray] = None
    elem: Optional[np.ndarray] = None
    release_lon: Optional[np.ndarray] = None
    release_lat: Optional[np.ndarray] = None
    release_z: Optional[np.ndarray] = None

    _OPTIONAL_ARRAYS = ("u", "v", "w", "failure_reason", "release_step",
                        "elem", "release_lon", "release_lat", "release_z")

    @property
    def n_particles(self) -> int:
        return self.lon.shape[0]

    @property
    def alive_mask(self) -> np.ndarray:
        return self.status == ParticleStatus.ALIVE

    def replace(self, **kw) -> "ParticleState":
        d = {f.name: getattr(self, f.name) for f in fields(self)}
        d.update(kw)
        return ParticleState(**d)

    def subset(self, index) -> "ParticleState":
        kw = {name: np.asarray(getattr(self, name))[index].copy()
              for name in ("lon", "lat", "z", "status", "nearest_node")}
        for name in self._OPTIONAL_ARRAYS:
            a = getattr(self, name)
            kw[name] = None if a is None else np.asarray(a)[index].copy()
        return ParticleState(**kw)


def make_state(lon, lat, z=None) -> ParticleState:
    """A fresh all-ALIVE state with unknown anchors (``particles.py:384``)."""
    lon = np.asarray(lon, dtype=np.float64)
    lat = np.asarray(lat, dtype=np.float64)
    P = lon.shape[0]
    z = np.zeros(P, dtype=np.float64) if z is None else np.asarray(z, dtype=np.float64)
    return ParticleState(lon=lon, lat=lat, z=z,
                         status=np.full(P, int(ParticleStatus.ALIVE), dtype=np.int32),
                         nearest_node=np.full(P, -1, dtype=np.int32))


def count_by_status(status: np.ndarray) -> dict:
    out = {
        "alive": int(np.sum(status == ParticleStatus.ALIVE)),
        "beached": int(np.sum(status == ParticleStatus.BEACHED)),
        "outside": int(np.sum(status == ParticleStatus.OUTSIDE)),
        "total": int(status.size),
    }
    n_dormant = int(np.sum(status == ParticleStatus.NOT_RELEASED))
    if n_dormant:
        out["not_released"] = n_dormant
    return out
