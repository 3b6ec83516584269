"""The exact C-grid quad mesh of a regional NEMO raster (mesh.nemo_grid: cgrid).

Restates ``build_nemo_cgrid_mesh`` (``src/kelp/readers/nemo/_mesh.py:16-264``)
for a closed regional raster (no E-W periodic halo, no north fold: every
raster point is its own canonical point): nodes are the F-points referenced
by a kept cell, elements are the wet T-cells (``T(j, i)`` with corners
``SW=F(j-1,i-1)``, ``SE=F(j-1,i)``, ``NE=F(j,i)``, ``NW=F(j,i-1)``, ``j, i >=
1``) followed by one ring of dry cells (8-neighbourhood) that read zero
velocity.  The mesh carries the tables ``numerics/nemo_cgrid.py`` reads
(``_nemo_cgrid_corners``, ``_elem_ji``, ``_nlev``, ``_nlev_raster``, ``_zw``,
``_area``, ``_e3b``, ``_kbu``/``_e3u``, ``_kbv``/``_e3v``, ``_e2u``/``_e1v``) and
is uploaded by ``DeviceContext.ensure_mesh`` (``kc_cgrid_upload``).
"""
from __future__ import annotations

from typing import Optional

import numpy as np

from .mesh import Mesh, build_node_to_elems, build_search


def partial_level(zw, e3, shape):
    """``_partial_level`` (readers/nemo/_vertical.py:74-88): per column the
    first level whose thickness differs from the reference layer (relative
    1e-4) and that thickness, flat ``(kb int32, th)``; ``kb = -1`` where none
    does (also for ``e3`` None)."""
    n = shape[0] * shape[1]
    if e3 is None:
        return np.full(n, -1, np.int32), np.zeros(n)
    e3 = np.asarray(e3, np.float64)
    ref = np.diff(zw)[:, None, None]
    diff = np.abs(e3 - ref) > 1e-4 * ref
    kb = np.where(diff.any(0), diff.argmax(0), -1)
    th = np.take_along_axis(e3, np.maximum(kb, 0)[None], 0)[0]
    return kb.astype(np.int32).reshape(-1), np.where(kb >= 0, th, 0.0).reshape(-1)


def _nonconvex(quads, lon, lat) -> np.ndarray:
    """Quads whose four corner turns in the tangent plane at their centroid
    are not all of one sign (or flat): the ring cells the builder drops
    (mesh.py:2920-3000 find_nonconvex_quads)."""
    la, lo = np.radians(lat[quads]), np.radians(lon[quads])
    v = np.stack((np.cos(la) * np.cos(lo), np.cos(la) * np.sin(lo), np.sin(la)), -1)
    c = v.mean(1)
    c /= np.linalg.norm(c, axis=1, keepdims=True)
    e1 = np.stack((-c[:, 1], c[:, 0], np.zeros(len(c))), -1)
    e1 /= np.maximum(np.linalg.norm(e1, axis=1, keepdims=True), 1e-300)
    e2 = np.cross(c, e1)
    x = np.einsum("qvk,qk->qv", v, e1)
    y = np.einsum("qvk,qk->qv", v, e2)
    ex, ey = np.roll(x, -1, 1) - x, np.roll(y, -1, 1) - y
    z = ex * np.roll(ey, -1, 1) - ey * np.roll(ex, -1, 1)
    scale = (ex ** 2 + ey ** 2).max(1, keepdims=True)
    flat = np.abs(z) <= 1e-12 * scale
    return np.flatnonzero(flat.any(1) | ~((z > 0).all(1) | (z < 0).all(1)))


def build_cgrid_mesh(glamf, gphif, tmask2d, *, depth2d=None, e2u=None, e1v=None, nlev2d=None, zw=None,
                     area=None, e3b=None, e3u0=None, e3v0=None, name: str = "nemo",
                     partial_cells: str = "shrunk", r_earth: Optional[float] = None,
                     exact_nearest: bool = True) -> Mesh:
    """The C-grid quad mesh of a regional raster (arguments as the
    reference's builder: F-point lon/lat, the surface T mask, optional model
    face widths, and in 3-D the wet levels per column, the reference layer
    interfaces ``zw (K+1)``, the T-cell areas, the bottom cell thickness and
    the model face thicknesses ``(K, ny, nx)``)."""
    lon2d = np.asarray(glamf, dtype=np.float64)
    lat2d = np.asarray(gphif, dtype=np.float64)
    if lon2d.ndim != 2 or lon2d.shape != lat2d.shape:
        raise ValueError(f"glamf/gphif must be 2-D (y, x) of equal shape, got {lon2d.shape} and {lat2d.shape}")
    ny, nx = lon2d.shape
    wet0 = np.asarray(tmask2d) > 0.5
    if wet0.shape != (ny, nx):
        raise ValueError(f"tmask shape {wet0.shape} != grid {(ny, nx)}")
    if partial_cells not in ("shrunk", "porous"):
        raise ValueError(f"partial_cells must be 'shrunk' or 'porous', got {partial_cells!r}")
    jj, ii = np.mgrid[0:ny, 0:nx]
    wet = wet0 & (jj >= 1) & (ii >= 1)
    if not wet.any():
        raise ValueError("NEMO C-grid mesh has no wet T-cells")
    flat_lon, flat_lat = lon2d.reshape(-1), lat2d.reshape(-1)

    def quads(j, i):
        return np.stack([(j + dj) * nx + (i + di) for dj, di in ((-1, -1), (-1, 0), (0, 0), (0, -1))], axis=1)

    ej, ei = np.nonzero(wet)
    quad_raster = quads(ej, ei)
    n_wet = int(ej.size)
    pd_ = np.pad(wet, 1)
    dil = np.zeros_like(wet)
    for dj in range(3):
        for di in range(3):
            dil |= pd_[dj:dj + ny, di:di + nx]
    rj, ri = np.nonzero(dil & ~wet)
    keep = (rj >= 1) & (ri >= 1)
    rj, ri = rj[keep], ri[keep]
    rq = quads(rj, ri)
    bad = _nonconvex(rq, flat_lon, flat_lat)
    keep = np.ones(rq.shape[0], dtype=bool)
    keep[bad] = False
    rj, ri, rq = rj[keep], ri[keep], rq[keep]
    n_ring = int(rj.size)
    ej = np.concatenate([ej, rj])
    ei = np.concatenate([ei, ri])
    quad_raster = np.concatenate([quad_raster, rq], axis=0)
    referenced = np.unique(quad_raster)
    n_nodes = int(referenced.size)
    remap = np.full(ny * nx, -1, dtype=np.int64)
    remap[referenced] = np.arange(n_nodes, dtype=np.int64)
    corners = remap[quad_raster].astype(np.int32)
    nodes_lon = np.ascontiguousarray(flat_lon[referenced])
    nodes_lat = np.ascontiguousarray(flat_lat[referenced])
    eb = None
    if zw is not None:
        nf = np.asarray(nlev2d, np.int32)
        eb = (np.diff(np.asarray(zw, np.float64))[np.maximum(nf - 1, 0)] if e3b is None
              else np.asarray(e3b, np.float64))
        eb = np.where(nf > 0, eb, 0.0)
        if depth2d is None:
            depth2d = np.where(nf > 0, np.asarray(zw, np.float64)[np.maximum(nf - 1, 0)] + eb, 0.0)
    depth = np.zeros(n_nodes)
    if depth2d is not None:
        d = np.where(wet0, np.nan_to_num(np.abs(np.asarray(depth2d, dtype=np.float64))), 0.0)
        dp = np.zeros((ny + 1, nx + 1))
        dp[:ny, :nx] = d                       # F(j, i) touches T(j..j+1, i..i+1)
        dm = np.maximum.reduce([dp[:ny, :nx], dp[1:, :nx], dp[:ny, 1:], dp[1:, 1:]]).reshape(-1)
        depth = np.ascontiguousarray(dm[referenced])
    elon, elat = nodes_lon[corners], nodes_lat[corners]
    ref = elon[:, [0]]
    elon_unw = ref + ((elon - ref + 180.0) % 360.0 - 180.0)
    n2e, cnt = build_node_to_elems(n_nodes, corners)
    mesh = Mesh(name=name, nodes_lon=nodes_lon, nodes_lat=nodes_lat, depth=depth, elem_nodes=corners.copy(),
                elem_center_lon=np.ascontiguousarray(((elon_unw.mean(axis=1) + 180.0) % 360.0) - 180.0),
                elem_center_lat=np.ascontiguousarray(elat.mean(axis=1)), node_to_elems=n2e,
                node_to_elems_count=cnt, sigma=np.array([], dtype=np.float64), vertical_coord="zlevel",
                **({} if r_earth is None else {"r_earth": float(r_earth)}))
    mesh._structured_shape = (ny, nx)
    mesh._nemo_cgrid = True
    mesh._nemo_cgrid_partial = partial_cells
    mesh._nemo_cgrid_elem_ji = np.stack([ej, ei], axis=1).astype(np.int64)
    mesh._nemo_cgrid_corners = corners
    nl = np.ones(n_wet) if nlev2d is None else np.asarray(nlev2d)[ej[:n_wet], ei[:n_wet]]
    mesh._nemo_cgrid_nlev = np.r_[nl, np.zeros(n_ring)].astype(np.int32)
    mesh._nemo_cgrid_nlev_raster = np.zeros((ny, nx), dtype=np.int32)
    mesh._nemo_cgrid_nlev_raster[ej[:n_wet], ei[:n_wet]] = nl
    mesh._nemo_cgrid_zw = np.empty(0) if zw is None else np.asarray(zw, np.float64)
    mesh._nemo_cgrid_area = np.empty(0) if area is None else np.ascontiguousarray(area, np.float64).reshape(-1)
    mesh._nemo_cgrid_e3b = np.empty(0)
    for nm in ("u", "v"):
        setattr(mesh, f"_nemo_cgrid_kb{nm}", np.empty(0, np.int32))
        setattr(mesh, f"_nemo_cgrid_e3{nm}", np.empty(0))
    if zw is not None:
        mesh.sigma = mesh._nemo_cgrid_zw
        mesh._nemo_cgrid_e3b = np.ascontiguousarray(eb).reshape(-1)
        for nm, e3 in (("u", e3u0), ("v", e3v0)):
            kb, th = partial_level(mesh._nemo_cgrid_zw, e3, (ny, nx))
            setattr(mesh, f"_nemo_cgrid_kb{nm}", kb)
            setattr(mesh, f"_nemo_cgrid_e3{nm}", th)
    if (e2u is None) != (e1v is None):
        raise ValueError("pass both e2u and e1v, or neither")
    for nm, a in (("_nemo_cgrid_e2u", e2u), ("_nemo_cgrid_e1v", e1v)):
        setattr(mesh, nm, np.empty(0, dtype=np.float64) if a is None
                else np.ascontiguousarray(np.asarray(a, dtype=np.float64).reshape(-1)))
    build_search(mesh)
    mesh.metadata["exact_nearest"] = bool(exact_nearest)
    return mesh
