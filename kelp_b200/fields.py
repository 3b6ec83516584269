"""Velocity snapshot payloads: one snapshot, and the lazily blended pair.

Mirrors KELP's ``src/kelp/core/io.py``: ``VelocityField`` (``:180``) holds one
snapshot (``u``/``v`` node- or element-valued, ``(N,)`` in 2-D or ``(L, N)`` in
3-D, ``w`` ``(K, N)`` on the interfaces, ``eta`` ``(N,)``), and ``LazyLerpField``
(``:386``) names a bracket pair plus the fraction ``alpha`` between them.  The
CUDA step kernels never materialise the blend: they read the raw pair and blend
per vertex with the arithmetic of ``io.py:52-65``.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import Optional

import numpy as np

_VALID_UV_LAYOUTS = ("element", "node", "nemo_cgrid")
_VALID_UV_VERTICAL = ("layer", "level", "layer_linear")


@dataclass
class VelocityField:
    u: np.ndarray
    v: np.ndarray
    eta: np.ndarray
    w: Optional[np.ndarray] = None
    uv_layout: str = "element"
    uv_vertical: str = "layer"
    kh_zonal: Optional[np.ndarray] = None
    kh_meridional: Optional[np.ndarray] = None
    kh_layout: Optional[str] = None
    az: Optional[np.ndarray] = None
    scalars: Optional[dict] = None
    meta: dict = field(default_factory=dict)

    def __post_init__(self):
        if self.uv_layout not in _VALID_UV_LAYOUTS:
            raise ValueError(f"uv_layout must be one of {_VALID_UV_LAYOUTS}, got {self.uv_layout!r}")
        if self.uv_vertical not in _VALID_UV_VERTICAL:
            raise ValueError(f"uv_vertical must be one of {_VALID_UV_VERTICAL}, got {self.uv_vertical!r}")
        if self.u.shape != self.v.shape:
            raise ValueError(f"u/v shape mismatch {self.u.shape} vs {self.v.shape}")


def _lerp(a, b, alpha: float) -> np.ndarray:
    """(1 - alpha) a + alpha b in float64, the expression of io.py:68-117
    _blend (float32 snapshots are widened first, so they blend in float64 as
    the reference's do, io.py:110-117)."""
    return (1.0 - alpha) * np.asarray(a, dtype=np.float64) + alpha * np.asarray(b, dtype=np.float64)


class LazyLerpField:
    """``(vel_a, vel_b, alpha)``: the field at a time between two snapshots.

    Only the raw pair and ``alpha`` are consumed by the CUDA kernels; the
    metadata checks mirror ``io.py:407-466`` so an inconsistent pair fails in
    Python before any device work."""

    def __init__(self, vel_a, vel_b, alpha: float):
        if vel_a.uv_layout != vel_b.uv_layout:
            raise ValueError(f"LazyLerpField: uv_layout mismatch {vel_a.uv_layout!r} vs {vel_b.uv_layout!r}")
        if getattr(vel_a, "uv_vertical", "layer") != getattr(vel_b, "uv_vertical", "layer"):
            raise ValueError("LazyLerpField: uv_vertical mismatch")
        for fname in ("u", "v", "eta"):
            fa, fb = getattr(vel_a, fname), getattr(vel_b, fname)
            if fa.shape != fb.shape:
                raise ValueError(f"LazyLerpField: {fname} shape mismatch {fa.shape} vs {fb.shape}")
        if vel_a.w is not None and vel_b.w is not None and vel_a.w.shape != vel_b.w.shape:
            raise ValueError(f"LazyLerpField: w shape mismatch {vel_a.w.shape} vs {vel_b.w.shape}")
        self.vel_a = vel_a
        self.vel_b = vel_b
        self.alpha = float(alpha)
        self.uv_layout = vel_a.uv_layout
        self.uv_vertical = getattr(vel_a, "uv_vertical", "layer")

    def _blend(self, name):
        a, b = getattr(self.vel_a, name), getattr(self.vel_b, name)
        if a is None or b is None:
            return None
        return _lerp(a, b, self.alpha)

    @property
    def u(self):
        return self._blend("u")

    @property
    def v(self):
        return self._blend("v")

    @property
    def w(self):
        if self.vel_a.w is None or self.vel_b.w is None:
            return None
        return self._blend("w")

    @property
    def eta(self):
        return self._blend("eta")

    @property
    def scalars(self):
        """The snapshots' node scalars blended key by key (io.py:499-513),
        None unless both carry them."""
        sa, sb = getattr(self.vel_a, "scalars", None), getattr(self.vel_b, "scalars", None)
        if sa is None or sb is None:
            return None
        if set(sa) != set(sb):
            raise ValueError(f"LazyLerpField: scalars key mismatch {sorted(sa)} vs {sorted(sb)}")
        return {k: _lerp(sa[k], sb[k], self.alpha) for k in sa}

    @property
    def az(self):
        """The blended vertical diffusivity, None unless both snapshots carry one."""
        if getattr(self.vel_a, "az", None) is None or getattr(self.vel_b, "az", None) is None:
            return None
        return self._blend("az")
