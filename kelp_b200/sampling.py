"""Scalar field sampling at particle positions on the device.

The counterpart of KELP's ``kelp.numerics.sampling.sample_field``
(numerics/sampling.py:727-933): the same signature, argument meaning,
validation errors and results (NaN for dead or anchorless particles, the
anchor's raw value as the fallback of every rule).  The work runs in the
native library (``kc_sample_field``, one thread per particle).

Covered: node fields ``(N,)``, z-level mid-layer fields ``(K-1, N)`` and
interface fields ``(K, N)`` (through the W interpolation of the method, as
the reference hands them over, sampling.py:876-890) with the methods
``nearest``, ``leastsq``, ``barycentric`` and ``idw``, and on sigma meshes
(sampling.py:620-723: the node columns max(depth + eta, Dmin)) with
``nearest``, ``leastsq`` and ``idw``; barycentric sampling on sigma meshes
raises ``NotImplementedError``.
"""
from __future__ import annotations

import numpy as np

METHOD_CODES = {"nearest": 0, "leastsq": 1, "barycentric": 2, "idw": 3}
_VALID = sorted(METHOD_CODES)


def _n_nodes(mesh) -> int:
    return int(np.asarray(mesh.nodes_lon).shape[0])


def sample_field(values, mesh, lons, lats, zs=None, *, nearest=None, alive=None, eta=None, method="leastsq",
                 Dmin=0.5, ctx=None) -> np.ndarray:
    """Sample a node scalar field at particle positions (sampling.py:727).

    values (N,), (K-1, N) or (K, N); lons, lats (P,) degrees; zs (P,)
    positive-down metres, required for a 3-D field; nearest (P,) anchors
    (None: the exact nearest node); alive (P,) mask (None: all alive);
    method one of nearest / leastsq / barycentric / idw; on a sigma mesh
    eta (N,) the free surface of the columns and Dmin their floor.
    """
    from .device import default_context
    if method not in METHOD_CODES:
        raise ValueError(f"Unknown method '{method}'. Valid method values are: {_VALID}")
    values = np.asarray(values, dtype=np.float64)
    lons = np.asarray(lons, dtype=np.float64)
    lats = np.asarray(lats, dtype=np.float64)
    N = _n_nodes(mesh)
    if values.shape[-1] != N:
        raise ValueError(f"values.shape[-1]={values.shape[-1]} does not match mesh.n_nodes={N}. "
                         "Element-based fields are not supported; provide a node-based field.")
    z_mids = None
    if values.ndim == 2:
        if zs is None:
            raise ValueError("zs (particle depths) is required for 3D field sampling")
        if getattr(mesh, "vertical_coord", "zlevel") == "sigma":   # sampling.py:620-723 _sample_sigma_3d
            if eta is None:
                raise ValueError("eta (free-surface elevation) is required for sigma mesh sampling")
            if method == "barycentric":
                raise NotImplementedError("barycentric sampling on sigma meshes is not built on the CUDA backend "
                                          "(nearest, leastsq and idw are)")
            K = np.asarray(mesh.sigma).size
            if values.shape[0] not in (K, K - 1):
                raise ValueError(f"sigma 3D field shape[0]={values.shape[0]} does not match "
                                 f"K={K} (interface) or K-1={K - 1} (mid-layer) from mesh.sigma")
            ctx = ctx or default_context()
            ctx.ensure_mesh(mesh)
            return ctx.sample_field_sigma(values, lons, lats, zs, eta, Dmin, nearest, alive, METHOD_CODES[method])
        zl = np.abs(np.asarray(mesh.sigma, dtype=np.float64))
        K = zl.size
        if values.shape[0] not in (K, K - 1):
            raise ValueError(f"3D z-level field shape[0]={values.shape[0]} does not match "
                             f"K={K} (interface) or K-1={K - 1} (mid-layer) from mesh.sigma")
        # an interface field (K, N) goes through the W interpolation
        # (sampling.py:876-890): no mid-layer depths
        z_mids = None if values.shape[0] == K else 0.5 * (zl[:-1] + zl[1:])
    elif values.ndim != 1:
        raise ValueError(f"values must be 1D (N,) or 2D (K, N) or (K-1, N), got shape {values.shape}")
    ctx = ctx or default_context()
    ctx.ensure_mesh(mesh)
    return ctx.sample_field(values, lons, lats, zs, z_mids, nearest, alive, METHOD_CODES[method])
