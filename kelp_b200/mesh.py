"""Unstructured-mesh container and the host-side search set-up.

Mirrors KELP's ``src/kelp/core/mesh.py``: the ``Mesh`` container (``:40-166``),
``build_node_to_elems`` (``:2716``), the uniform longitude/latitude grid hash
(``build_grid_hash`` ``:844-1001`` with ``_gh_lon_branch`` ``:799``,
``_gh_grid_geometry`` ``:814``, ``_gh_cell_index`` ``:831``), the exact-search
row budget (``_gh_max_edge_for`` ``:1008``, ``_gh_far_rows_for`` ``:1042``) and
the unit-sphere node table (``_node_xyz_fill`` ``:712``).

All of it is once-per-run host set-up.  The CSR hash follows the reference's
layout exactly (``cell = cj * nx + ci``; nodes of a cell in increasing node
index) because the nearest-node scan order decides ties.  The node table is
evaluated by the native library's host routine with the C library's ``cos``/
``sin`` -- the same functions the reference's Numba fill calls -- never by
numpy, whose SIMD trigonometry rounds differently in the last place.

The step functions accept any object with these attribute names, so a mesh
built by KELP itself (``kelp.core.mesh.Mesh`` after ``build_search``) works
unchanged.
"""
from __future__ import annotations

import warnings
from dataclasses import dataclass, field
from typing import Any, Dict, Optional

import numpy as np

from .geometry import DEG2RAD, RAD2DEG, R_EARTH_STANDARD

_GRID_HASH_MAX_CELLS = 50_000_000
_GH_FAR_ROWS_MIN = 4
_GH_FAR_ROWS_MAX = 4096


@dataclass
class Mesh:
    name: str
    nodes_lon: np.ndarray
    nodes_lat: np.ndarray
    depth: np.ndarray
    elem_nodes: np.ndarray
    elem_center_lon: np.ndarray
    elem_center_lat: np.ndarray
    node_to_elems: np.ndarray
    node_to_elems_count: np.ndarray
    sigma: np.ndarray = field(default_factory=lambda: np.array([], dtype=np.float64))
    vertical_coord: str = "zlevel"
    r_earth: float = R_EARTH_STANDARD
    metadata: Dict[str, Any] = field(default_factory=dict)

    _gh_offsets: Optional[np.ndarray] = field(default=None, repr=False)
    _gh_node_ids: Optional[np.ndarray] = field(default=None, repr=False)
    _gh_cell_size: float = field(default=0.0, repr=False)
    _gh_lon_min: float = field(default=0.0, repr=False)
    _gh_lat_min: float = field(default=0.0, repr=False)
    _gh_nx: int = field(default=0, repr=False)
    _gh_ny: int = field(default=0, repr=False)
    _gh_wrap_lon: bool = field(default=False, repr=False)
    _gh_far_rows: int = field(default=16, repr=False)
    _gh_max_edge_deg: Optional[float] = field(default=None, repr=False)
    _node_xyz: Optional[np.ndarray] = field(default=None, repr=False)
    _elem_neighbors: Optional[np.ndarray] = field(default=None, repr=False)
    _elem_is_coastal: Optional[np.ndarray] = field(default=None, repr=False)

    @property
    def n_nodes(self) -> int:
        return self.nodes_lon.shape[0]

    @property
    def n_elements(self) -> int:
        return self.elem_nodes.shape[0]

    @property
    def z_levels(self) -> np.ndarray:
        if self.vertical_coord != "zlevel":
            raise NotImplementedError("mesh.z_levels is only valid for z-level meshes")
        return np.abs(self.sigma)


def build_node_to_elems(n_nodes: int, elem_nodes: np.ndarray):
    """Dense ``(N, max_conn)`` node->element table, -1 padded, elements of a
    node in increasing element order, a vertex repeated within one element
    counted once (``mesh.py:2716-2762``)."""
    en = np.asarray(elem_nodes)
    E, mv = en.shape
    # de-duplicate vertices repeated inside one element (FESOM-C tri-as-quad)
    keep = en >= 0
    for k in range(1, mv):
        for j in range(k):
            keep[:, k] &= en[:, k] != en[:, j]
    e_idx = np.repeat(np.arange(E, dtype=np.int64), mv).reshape(E, mv)[keep]
    n_idx = en[keep].astype(np.int64)
    order = np.lexsort((e_idx, n_idx))          # by node, then element
    n_sorted = n_idx[order]
    e_sorted = e_idx[order]
    counts = np.bincount(n_sorted, minlength=n_nodes).astype(np.int32)
    max_conn = int(counts.max()) if n_nodes > 0 else 0
    starts = np.zeros(n_nodes + 1, dtype=np.int64)
    np.cumsum(counts, out=starts[1:])
    col = np.arange(n_sorted.size, dtype=np.int64) - starts[n_sorted]
    n2e = np.full((n_nodes, max_conn), -1, dtype=np.int32)
    n2e[n_sorted, col] = e_sorted.astype(np.int32)
    return n2e, counts


def _gh_lon_branch(nodes_lon: np.ndarray):
    lon_0360 = (nodes_lon + 360.0) % 360.0
    lon_signed = (nodes_lon + 180.0) % 360.0 - 180.0
    span_0360 = lon_0360.max() - lon_0360.min()
    span_signed = lon_signed.max() - lon_signed.min()
    wrap = bool(min(span_0360, span_signed) > 350.0)
    if wrap or span_0360 <= span_signed:
        return lon_0360, wrap
    return lon_signed, wrap


def _gh_grid_geometry(lon, lat, cell_size, wrap):
    lat_min = lat.min() - cell_size
    lat_max = lat.max() + cell_size
    ny = int(np.ceil((lat_max - lat_min) / cell_size))
    if wrap:
        lon_min = 0.0
        nx = int(np.ceil(360.0 / cell_size))
    else:
        lon_min = lon.min() - cell_size
        lon_max = lon.max() + cell_size
        nx = int(np.ceil((lon_max - lon_min) / cell_size))
    return lon_min, lat_min, nx, ny


def _gh_cell_index(lon, lat, cell_size, lon_min, lat_min, nx, ny, wrap):
    if wrap:
        ci = np.minimum((lon / cell_size).astype(np.int32), nx - 1)
    else:
        ci = np.clip(((lon - lon_min) / cell_size).astype(np.int32), 0, nx - 1)
    cj = np.clip(((lat - lat_min) / cell_size).astype(np.int32), 0, ny - 1)
    return cj * nx + ci


def node_xyz_table(nodes_lon: np.ndarray, nodes_lat: np.ndarray) -> np.ndarray:
    """Unit-sphere coordinates ``(N, 3)`` of every node, evaluated with the C
    library's ``cos``/``sin`` by the native library (``mesh.py:712-737``)."""
    from . import _native
    lon = np.ascontiguousarray(nodes_lon, dtype=np.float64)
    lat = np.ascontiguousarray(nodes_lat, dtype=np.float64)
    out = np.empty((lon.shape[0], 3), dtype=np.float64)
    _native.node_xyz_fill(lon, lat, out)
    return out


def ensure_node_xyz(mesh) -> np.ndarray:
    """The mesh's unit-sphere node table, computed on first use (KELP's
    ``build_search`` fills it at once; here building the grid hash does not
    load the native library, so the arrays of a mesh can be prepared without
    it)."""
    if getattr(mesh, "_node_xyz", None) is None:
        mesh._node_xyz = node_xyz_table(mesh.nodes_lon, mesh.nodes_lat)
    return mesh._node_xyz


def _gh_max_edge_for(mesh) -> float:
    en = mesh.elem_nodes
    if en is None or en.size == 0:
        return 0.0
    lon = np.asarray(mesh.nodes_lon, dtype=np.float64)
    lat = np.asarray(mesh.nodes_lat, dtype=np.float64)
    nv = en.shape[1]
    max_edge = 0.0
    step = 1_000_000
    for e0 in range(0, en.shape[0], step):
        blk = en[e0:e0 + step]
        last_valid = np.clip((blk >= 0).sum(axis=1) - 1, 0, nv - 1)
        pairs = [(blk[:, k], blk[:, (k + 1) % nv]) for k in range(nv)]
        pairs.append((blk[np.arange(blk.shape[0]), last_valid], blk[:, 0]))
        for a, b in pairs:
            ok = (a >= 0) & (b >= 0)
            if not ok.any():
                continue
            a = a[ok]
            b = b[ok]
            d = lon[b] - lon[a]
            dl = (((d + 180.0) % 360.0) - 180.0) * DEG2RAD
            la1 = lat[a] * DEG2RAD
            la2 = lat[b] * DEG2RAD
            cosd = np.sin(la1) * np.sin(la2) + np.cos(la1) * np.cos(la2) * np.cos(dl)
            dd = np.arccos(np.clip(cosd, -1.0, 1.0)) * RAD2DEG
            max_edge = max(max_edge, float(dd.max()))
    return max_edge


def _gh_far_rows_for(mesh, cell_size: float) -> int:
    if getattr(mesh, "_gh_max_edge_deg", None) is None:
        mesh._gh_max_edge_deg = _gh_max_edge_for(mesh)
    rows = int(np.ceil(mesh._gh_max_edge_deg / cell_size - 1.0e-9)) + 2
    if rows > _GH_FAR_ROWS_MAX:
        warnings.warn("grid hash: exact-search row budget capped at "
                      f"{_GH_FAR_ROWS_MAX} cells", RuntimeWarning)
        rows = _GH_FAR_ROWS_MAX
    if rows < _GH_FAR_ROWS_MIN:
        rows = _GH_FAR_ROWS_MIN
    return int(rows)


def build_grid_hash(mesh, cell_size: float = 0.0, ctx=None) -> None:
    """Uniform lon/lat CSR hash over the mesh nodes (``mesh.py:844-1001``).

    ``cell_size`` 0 takes ``metadata["grid_hash_cell"]`` when pinned, else the
    reference's automatic size ``max(0.05, 2 sqrt(area / N))`` degrees.  With
    a device context ``ctx`` the cells, the stable sort and the offsets are
    computed on the GPU (kc_grid_hash_build, equal bit for bit); the lon
    branch and the grid geometry are host decisions either way."""
    lon, wrap = _gh_lon_branch(np.asarray(mesh.nodes_lon, dtype=np.float64))
    lon_span = lon.max() - lon.min()
    lat = np.asarray(mesh.nodes_lat, dtype=np.float64)
    N = len(lon)
    if not cell_size > 0:
        md = mesh.metadata or {}
        if "grid_hash_cell" in md:
            pinned = float(md["grid_hash_cell"])
            if not np.isfinite(pinned) or not (0.0 < pinned < 45.0):
                raise ValueError("mesh.metadata['grid_hash_cell'] must be a finite "
                                 f"cell size in (0, 45) degrees, got {md['grid_hash_cell']!r}")
            cell_size = pinned
        else:
            lat_span = lat.max() - lat.min()
            area = max(lon_span * lat_span, 1.0)
            cell_size = max(0.05, np.sqrt(area / N) * 2)
    lon_min, lat_min, nx, ny = _gh_grid_geometry(lon, lat, cell_size, wrap)
    n_cells = nx * ny
    if n_cells > _GRID_HASH_MAX_CELLS:
        raise ValueError(f"grid hash: cell size {cell_size:.6g} deg needs {n_cells} cells "
                         f"(> {_GRID_HASH_MAX_CELLS}); use a larger cell.")
    if ctx is not None:
        offsets, node_ids = ctx.grid_hash(lon, lat, cell_size, lon_min, lat_min, nx, ny, wrap)
    else:
        cell_idx = _gh_cell_index(lon, lat, cell_size, lon_min, lat_min, nx, ny, wrap)
        counts = np.bincount(cell_idx, minlength=n_cells).astype(np.int32)
        offsets = np.zeros(n_cells + 1, dtype=np.int32)
        np.cumsum(counts, out=offsets[1:])
        node_ids = np.argsort(cell_idx, kind="stable").astype(np.int32)

    mesh._node_xyz = None   # filled on first use by ensure_node_xyz (the native library's C-library trig)
    mesh._gh_offsets = offsets
    mesh._gh_node_ids = node_ids
    mesh._gh_cell_size = cell_size
    mesh._gh_lon_min = lon_min
    mesh._gh_lat_min = lat_min
    mesh._gh_nx = nx
    mesh._gh_ny = ny
    mesh._gh_wrap_lon = wrap
    mesh._gh_far_rows = _gh_far_rows_for(mesh, cell_size)


def build_boundary_info(mesh) -> None:
    """Coastal element flags: an element owning an edge that no other element
    shares (``mesh.py:2764-2821``).  Each element's edge ring runs over its
    compacted valid vertices (the closing edge included), an undirected edge
    counted once per element."""
    if getattr(mesh, "_elem_is_coastal", None) is not None:
        return
    en = np.asarray(mesh.elem_nodes)
    E, mv = en.shape
    if E == 0:
        mesh._elem_is_coastal = np.zeros(0, dtype=np.bool_)
        return
    mask = en >= 0
    if mv == 4:
        mask[:, 3] &= ~((en[:, 3] == en[:, 0]) & (en[:, 0] >= 0))
    nv = mask.sum(axis=1)
    # compact each row's valid vertices to the front, in order
    order = np.argsort(~mask, axis=1, kind="stable")
    verts = np.take_along_axis(en, order, axis=1).astype(np.int64)
    rows = np.arange(E)
    e_all, k_all = [], []
    base = np.int64(mesh.nodes_lon.shape[0] + 1)
    for j in range(mv):
        ok = (nv >= 3) & (j < nv)
        nxt = np.where(ok, (j + 1) % np.maximum(nv, 1), 0)
        a = verts[rows, j]
        b = verts[rows, nxt]
        ok &= a != b
        lo, hi = np.minimum(a, b), np.maximum(a, b)
        e_all.append(rows[ok])
        k_all.append(lo[ok] * base + hi[ok])
    coastal = np.zeros(E, dtype=np.bool_)
    if e_all:
        e_cat = np.concatenate(e_all)
        k_cat = np.concatenate(k_all)
        if e_cat.size:
            # an undirected edge counts once per element
            pairs = np.unique(np.stack([k_cat, e_cat.astype(np.int64)], axis=1), axis=0)
            _, inv, cnt = np.unique(pairs[:, 0], return_inverse=True, return_counts=True)
            coastal[pairs[cnt[inv] == 1, 1]] = True
    mesh._elem_is_coastal = coastal


def build_elem_neighbors(mesh) -> np.ndarray:
    """Element adjacency across shared edges (``mesh.py:2824-2910``): slot k of
    row e holds the element sharing edge (v_k, v_{k+1}) of e's compacted
    vertex ring (-1 pads and repeats of the first vertex dropped), -1 on a
    boundary edge or an unused slot.  An edge of more than two elements (a
    non-manifold mesh) raises.  Cached as ``mesh._elem_neighbors``."""
    cached = getattr(mesh, "_elem_neighbors", None)
    if cached is not None:
        return cached
    en = np.asarray(mesh.elem_nodes)
    E, mv = en.shape
    out = np.full((E, mv), -1, dtype=np.int32)
    if E == 0:
        mesh._elem_neighbors = out
        return out
    # compacted ring: keep a slot unless it is -1 or repeats the first valid vertex
    first = np.full(E, -1, dtype=np.int64)
    keep = np.zeros((E, mv), dtype=bool)
    for j in range(mv):
        v = en[:, j].astype(np.int64)
        ok = v >= 0
        ok &= ~((first >= 0) & (v == first))
        keep[:, j] = ok
        first = np.where((first < 0) & ok, v, first)
    nv = keep.sum(axis=1)
    order = np.argsort(~keep, axis=1, kind="stable")
    verts = np.take_along_axis(en, order, axis=1).astype(np.int64)
    rows = np.arange(E)
    base = np.int64(np.asarray(mesh.nodes_lon).shape[0] + 1)
    e_all, k_all, key_all = [], [], []
    for k in range(mv):
        ok = (nv >= 3) & (k < nv)
        nxt = np.where(ok, (k + 1) % np.maximum(nv, 1), 0)
        a = verts[rows, k]
        b = verts[rows, nxt]
        ok &= a != b
        e_all.append(rows[ok])
        k_all.append(np.full(int(ok.sum()), k, dtype=np.int64))
        key_all.append(np.minimum(a, b)[ok] * base + np.maximum(a, b)[ok])
    e_cat = np.concatenate(e_all)
    k_cat = np.concatenate(k_all)
    key = np.concatenate(key_all)
    if key.size:
        # a ring repeating an edge keeps its first slot (per-element dedup)
        o = np.lexsort((k_cat, e_cat, key))
        key, e_cat, k_cat = key[o], e_cat[o], k_cat[o]
        dup = np.r_[False, (key[1:] == key[:-1]) & (e_cat[1:] == e_cat[:-1])]
        key, e_cat, k_cat = key[~dup], e_cat[~dup], k_cat[~dup]
        starts = np.flatnonzero(np.r_[True, key[1:] != key[:-1]])
        counts = np.diff(np.r_[starts, key.size])
        if (counts > 2).any():
            s0 = starts[counts > 2][0]
            raise ValueError(f"non-manifold mesh: edge key {int(key[s0])} is shared by {int(counts[counts > 2][0])} "
                             "elements")
        pairs = starts[counts == 2]
        out[e_cat[pairs], k_cat[pairs]] = e_cat[pairs + 1]
        out[e_cat[pairs + 1], k_cat[pairs + 1]] = e_cat[pairs]
    mesh._elem_neighbors = out
    return out


def build_search(mesh) -> None:
    """Build the grid hash (``mesh.py:237``)."""
    build_grid_hash(mesh)


def set_grid_hash_cell(mesh, cell_size: float) -> None:
    """Pin an explicit cell size and rebuild (``mesh.py:287``)."""
    cs = float(cell_size)
    if not np.isfinite(cs) or not 0.0 < cs < 45.0:
        raise ValueError(f"grid-hash cell_size must be a finite value in (0, 45) degrees, got {cell_size!r}")
    mesh.metadata["grid_hash_cell"] = cs
    build_grid_hash(mesh, cell_size=cs)


def set_exact_nearest(mesh, flag: bool) -> None:
    """Switch the exact nearest-node anchor on/off (``mesh.py:321``)."""
    mesh.metadata["exact_nearest"] = bool(flag)


def make_mesh(name, nodes_lon, nodes_lat, depth, elem_nodes, *, sigma=None,
              vertical_coord="zlevel", r_earth=R_EARTH_STANDARD,
              cell_size: float = 0.0, exact_nearest: bool = True) -> Mesh:
    """Assemble a ``Mesh`` from node/element arrays and build its search
    structures (node->element table, grid hash, node table)."""
    lon = np.ascontiguousarray(nodes_lon, dtype=np.float64)
    lat = np.ascontiguousarray(nodes_lat, dtype=np.float64)
    en = np.ascontiguousarray(elem_nodes, dtype=np.int32)
    n2e, cnt = build_node_to_elems(lon.size, en)
    valid = en >= 0
    nvalid = valid.sum(axis=1)
    ref = lon[en[:, 0]]
    d = np.where(valid, ((lon[np.where(valid, en, 0)] - ref[:, None] + 180.0) % 360.0) - 180.0, 0.0)
    ecl = ((ref + d.sum(axis=1) / nvalid + 180.0) % 360.0) - 180.0
    ecla = np.where(valid, lat[np.where(valid, en, 0)], 0.0).sum(axis=1) / nvalid
    mesh = Mesh(name=name, nodes_lon=lon, nodes_lat=lat,
                depth=np.ascontiguousarray(depth, dtype=np.float64), elem_nodes=en,
                elem_center_lon=ecl, elem_center_lat=ecla,
                node_to_elems=n2e, node_to_elems_count=cnt,
                sigma=np.array([], dtype=np.float64) if sigma is None else np.asarray(sigma, dtype=np.float64),
                vertical_coord=vertical_coord, r_earth=float(r_earth))
    if cell_size > 0:
        mesh.metadata["grid_hash_cell"] = float(cell_size)
    build_grid_hash(mesh)
    set_exact_nearest(mesh, exact_nearest)
    return mesh
