"""The depth-linear u/v data-point table (node layout).

Mirrors KELP's ``src/kelp/numerics/vertical_uv.py:181-278``
(``_build_depth_points``) and ``depth_points`` (``:328``): for placement
``"level"`` the data points are the level depths, for ``"layer_linear"`` the
layer centres; ``last[i]`` is the deepest point of node ``i`` whose lower
bound lies at or above the node's bed (capped by the reader's optional
declaration ``mesh.metadata["uv_data_last"]``); ``bed`` is the node depth.
On a sigma mesh (``"layer_linear"`` only) the points are the layer centres in
the sigma fraction s = z / H, every node reads every layer and is wet at every
s (``bed`` = +inf).  The CUDA kernels read the table for fields whose
``uv_vertical`` is ``"level"`` or ``"layer_linear"``.
"""
from __future__ import annotations

from typing import NamedTuple

import numpy as np

PLACEMENTS = ("level", "layer_linear")


class DepthPoints(NamedTuple):
    p: np.ndarray      # (M,) data-point depths, positive down
    last: np.ndarray   # (N,) int32 last usable point per node
    bed: np.ndarray    # (N,) float64 bed depth per node


def depth_points(mesh, placement: str) -> DepthPoints:
    if placement not in PLACEMENTS:
        raise ValueError(f"depth_points: placement must be one of {PLACEMENTS}, got {placement!r}")
    if getattr(mesh, "vertical_coord", "zlevel") == "sigma":
        # vertical_uv.py:196-211: interfaces at s_k = 1 - sigma_k
        if placement != "layer_linear":
            raise ValueError(f"depth-linear u/v ({placement!r}) on a sigma mesh: only 'layer_linear' is defined")
        sg = np.asarray(mesh.sigma, dtype=np.float64)
        if sg.ndim != 1 or sg.size < 2:
            raise ValueError(f"depth-linear u/v ({placement!r}) needs a 3-D sigma mesh with >= 2 interfaces "
                             f"in mesh.sigma, got shape {sg.shape}")
        p = 1.0 - 0.5 * (sg[:-1] + sg[1:])
        n = np.asarray(mesh.nodes_lon).shape[0]
        return DepthPoints(p=p, last=np.full(n, p.size - 1, np.int32), bed=np.full(n, np.inf))
    z = np.abs(np.asarray(mesh.sigma, dtype=np.float64))
    need = 1 if placement == "level" else 2
    if z.ndim != 1 or z.size < need:
        raise ValueError(f"depth-linear u/v ({placement!r}) needs >= {need} levels in mesh.sigma")
    if not np.all(np.isfinite(z)):
        raise ValueError(f"depth-linear u/v ({placement!r}) needs finite level depths")
    if np.any(np.diff(z) < 0.0):
        raise ValueError(f"depth-linear u/v ({placement!r}) needs non-decreasing level depths")
    if placement == "level":
        p = z.copy()
        lower = p
    else:
        p = 0.5 * (z[:-1] + z[1:])
        lower = z[1:]
    m = p.size
    d = np.asarray(mesh.depth, dtype=np.float64)
    geo = np.searchsorted(lower, d, side="right").astype(np.int64) - 1
    geo[np.isnan(d)] = 0
    last = np.minimum(geo, m - 1)
    decl = (getattr(mesh, "metadata", None) or {}).get("uv_data_last")
    if decl is not None:
        dl = np.asarray(decl)
        if dl.shape != d.shape or not np.issubdtype(dl.dtype, np.integer):
            raise ValueError("mesh.metadata['uv_data_last'] must be an integer array of shape (N,)")
        if dl.size and int(dl.min()) < -1:
            raise ValueError("mesh.metadata['uv_data_last'] must be >= -1")
        last = np.minimum(last, dl.astype(np.int64))
    last = np.maximum(last, 0).astype(np.int32)
    return DepthPoints(p=p, last=last, bed=d.copy())
