"""Seeded synthetic meshes, velocity snapshots and particle releases.

The reference measures on synthetic data only; these generators build inputs
of the shapes its benchmark configurations name (no readers, no files):

* ``lattice_mesh`` -- a jittered lon/lat lattice triangulated cell by cell
  (the seam column joins back across +-180 deg like KELP's own band meshes in
  ``tests/test_fused_bary_tinterp.py``), optionally with a fraction of cells
  kept as convex quads, and a land mask from smooth spherical noise;
* ``gyre_snapshots`` -- node-layout u/v (solid-body rotation plus a
  double gyre) and, for 3-D, u/v per layer and w on the interfaces from the
  continuity of the same stream-function flow;
* ``release_uniform`` -- particles uniform in area over the wet elements
  (and uniform in depth over the local column for 3-D).
"""
from __future__ import annotations

import numpy as np

from .fields import VelocityField
from .geometry import DEG2RAD
from .mesh import make_mesh


def _sphere_noise(lon, lat, n_modes=32, seed=2):
    rng = np.random.default_rng(seed)
    x = np.cos(lat * DEG2RAD) * np.cos(lon * DEG2RAD)
    y = np.cos(lat * DEG2RAD) * np.sin(lon * DEG2RAD)
    z = np.sin(lat * DEG2RAD)
    f = np.zeros_like(lon)
    for _ in range(n_modes):
        d = rng.normal(size=3)
        d /= np.linalg.norm(d)
        k = rng.uniform(1.0, 6.0)
        ph = rng.uniform(0, 2 * np.pi)
        amp = rng.uniform(0.5, 1.0) / k
        f += amp * np.cos(k * (d[0] * x + d[1] * y + d[2] * z) * np.pi + ph)
    return f


def lattice_mesh(spacing: float = 0.5625, lat_max: float = 80.0, *, lon_min: float = -180.0,
                 lon_max: float = 180.0, jitter: float = 0.2, land_frac: float = 0.3,
                 quad_frac: float = 0.0, seed_jitter: int = 1, seed_land: int = 2, seed_quad: int = 4,
                 depth=None, sigma=None, cell_size: float = 0.0, name: str = "lattice"):
    """Jittered lon/lat lattice mesh.  ``lon_max - lon_min == 360`` joins the
    seam column.  Land (``land_frac`` of the nodes by smooth noise) removes
    every element touching a land node, then orphaned nodes."""
    glob = abs((lon_max - lon_min) - 360.0) < 1e-9
    nlon = int(round((lon_max - lon_min) / spacing)) + (0 if glob else 1)
    nlat = int(round(2 * lat_max / spacing)) + 1 if lat_max > 0 else 1
    lon1 = lon_min + spacing * np.arange(nlon)
    lat1 = -lat_max + spacing * np.arange(nlat)
    gx, gy = np.meshgrid(lon1, lat1)
    lon = gx.ravel().astype(np.float64)
    lat = gy.ravel().astype(np.float64)
    rng = np.random.default_rng(seed_jitter)
    lon = lon + rng.uniform(-jitter, jitter, lon.size) * spacing
    lat = lat + rng.uniform(-jitter, jitter, lat.size) * spacing
    lat = np.clip(lat, -89.9, 89.9)
    lon = ((lon + 180.0) % 360.0) - 180.0
    ncx = nlon if glob else nlon - 1
    jj, ii = np.meshgrid(np.arange(nlat - 1), np.arange(ncx), indexing="ij")
    jj = jj.ravel()
    ii = ii.ravel()
    i2 = (ii + 1) % nlon
    n0 = jj * nlon + ii
    n1 = jj * nlon + i2
    n2 = (jj + 1) * nlon + ii
    n3 = (jj + 1) * nlon + i2
    qrng = np.random.default_rng(seed_quad)
    is_quad = qrng.uniform(size=n0.size) < quad_frac
    tris_a = np.stack([n0, n1, n2, np.full_like(n0, -1)], 1)
    tris_b = np.stack([n1, n3, n2, np.full_like(n0, -1)], 1)
    quads = np.stack([n0, n1, n3, n2], 1)
    elems = np.concatenate([quads[is_quad], tris_a[~is_quad], tris_b[~is_quad]])
    if land_frac > 0:
        noise = _sphere_noise(lon, lat, seed=seed_land)
        land = noise < np.quantile(noise, land_frac)
        valid = elems >= 0
        touches = (land[np.where(valid, elems, 0)] & valid).any(axis=1)
        elems = elems[~touches]
    if quad_frac <= 0:
        elems = elems[:, :3]
    used = np.zeros(lon.size, bool)
    used[elems[elems >= 0]] = True
    remap = np.full(lon.size, -1, np.int64)
    remap[used] = np.arange(used.sum())
    elems = np.where(elems >= 0, remap[np.where(elems >= 0, elems, 0)], -1).astype(np.int32)
    lon = lon[used]
    lat = lat[used]
    if depth is None:
        d = np.full(lon.size, 4000.0)
    elif callable(depth):
        d = depth(lon, lat)
    else:
        d = np.asarray(depth)[used]
    return make_mesh(name, lon, lat, d, elems, sigma=sigma, cell_size=cell_size)


def stretched_levels(k_levels: int = 47, top: float = 5.0, bottom: float = 6000.0):
    """0 then ``top * r**(k-1)`` up to ``bottom`` (positive down)."""
    n = k_levels - 1
    r = (bottom / top) ** (1.0 / (n - 1))
    return np.concatenate([[0.0], top * r ** np.arange(n)])


def smooth_bathymetry(lon, lat, dmin=50.0, dmax=6000.0, seed=5):
    f = _sphere_noise(lon, lat, n_modes=16, seed=seed)
    f = (f - f.min()) / (f.max() - f.min() + 1e-300)
    return dmin + (dmax - dmin) * f


def _gyre_uv(lon, lat, phase, amp):
    """Solid-body rotation plus a double gyre (m/s), smooth on the sphere."""
    la = lat * DEG2RAD
    lo = lon * DEG2RAD
    u_sb = 0.5 * amp * np.cos(la)
    # stream function psi = sin(2 lo + phase) * sin(2 la)^2 ; u = -dpsi/dy, v = dpsi/dx
    s = np.sin(2 * lo + phase)
    c = np.cos(2 * lo + phase)
    u_g = -amp * 0.5 * s * 2 * np.sin(2 * la) * np.cos(2 * la) * 2
    v_g = amp * 0.5 * 2 * c * np.sin(2 * la) ** 2
    return u_sb + u_g, v_g


def gyre_snapshots(mesh, n_snap: int = 2, *, amp: float = 0.5, dtype=np.float32,
                   z_levels=None, decay: float = 1000.0, w_scale: float = 1e-4, placement: str = "layer"):
    """``n_snap`` node-layout snapshots, the phase advancing by 0.7 rad per
    snapshot.  With ``z_levels`` (K interfaces): u/v scaled by
    ``exp(-z / decay)`` at the layer mid-depths ((K-1, N), placement
    ``"layer"`` or ``"layer_linear"``) or on the levels ((K, N), placement
    ``"level"``), and w (K, N) from continuity of the divergent part
    (positive down, w = 0 at the surface)."""
    lon = np.asarray(mesh.nodes_lon)
    lat = np.asarray(mesh.nodes_lat)
    out = []
    for k in range(n_snap):
        u, v = _gyre_uv(lon, lat, 0.7 * k, amp)
        if z_levels is None:
            out.append(VelocityField(u=u.astype(dtype), v=v.astype(dtype), eta=np.zeros(lon.size),
                                     uv_layout="node"))
            continue
        zl = np.asarray(z_levels, dtype=np.float64)
        zm = zl if placement == "level" else 0.5 * (zl[:-1] + zl[1:])
        dec = np.exp(-zm / decay)[:, None]
        div = np.sin(3 * lon * DEG2RAD + 0.7 * k) * np.cos(3 * lat * DEG2RAD)
        uu = (u[None, :] * dec).astype(dtype)
        vv = (v[None, :] * dec).astype(dtype)
        # w(z) = -int_0^z div * f(z') dz', f = exp(-z/decay): closed form
        ww = (w_scale * div[None, :] * (1.0 - np.exp(-zl / decay))[:, None]).astype(dtype)
        out.append(VelocityField(u=uu, v=vv, w=ww, eta=np.zeros(lon.size), uv_layout="node",
                                 uv_vertical=placement))
    return out


def vortex_snapshots(mesh, n_snap: int = 2, *, n_vortex: int = 256, rms: float = 0.3, z_levels=None,
                     decay: float = 1000.0, w_amp: float = 1e-5, dtype=np.float32, seed: int = 3):
    """Eddying node-layout field: a sum of ``n_vortex`` Gaussian vortices
    (centres uniform on the sphere, radii 30-300 km, random sign), scaled to
    ``rms`` m/s over the nodes; successive snapshots drift the centres
    westward by one radius.  3-D: u/v per layer decaying as exp(-z/decay), and
    a small smooth w (``w_amp`` m/s) on the interfaces, zero at the surface."""
    rng = np.random.default_rng(seed)
    lon = np.asarray(mesh.nodes_lon)
    lat = np.asarray(mesh.nodes_lat)
    zc = rng.uniform(-1, 1, n_vortex)
    clat = np.degrees(np.arcsin(zc))
    clon = rng.uniform(-180, 180, n_vortex)
    rad = rng.uniform(30e3, 300e3, n_vortex)
    sgn = rng.choice([-1.0, 1.0], n_vortex)
    R_E = 6371000.0
    out = []
    for s in range(n_snap):
        u = np.zeros(lon.size)
        v = np.zeros(lon.size)
        for k in range(n_vortex):
            band = 4.0 * np.degrees(rad[k] / R_E)
            sel = np.flatnonzero(np.abs(lat - clat[k]) < band)
            cl = clon[k] - s * np.degrees(rad[k] / R_E) / max(np.cos(np.radians(clat[k])), 0.05)
            dx = (((lon[sel] - cl + 180.0) % 360.0) - 180.0) * DEG2RAD * R_E * np.cos(np.radians(clat[k]))
            dy = (lat[sel] - clat[k]) * DEG2RAD * R_E
            g = np.exp(-(dx * dx + dy * dy) / (2 * rad[k] ** 2))
            # stream function sgn * exp(-r^2 / 2R^2): u = -dpsi/dy, v = dpsi/dx
            u[sel] += sgn[k] * g * dy / rad[k]
            v[sel] -= sgn[k] * g * dx / rad[k]
        scale = rms / max(np.sqrt(np.mean(u * u + v * v)), 1e-30)
        u *= scale
        v *= scale
        if z_levels is None:
            out.append(VelocityField(u=u.astype(dtype), v=v.astype(dtype), eta=np.zeros(lon.size),
                                     uv_layout="node"))
            continue
        zl = np.asarray(z_levels, dtype=np.float64)
        zm = 0.5 * (zl[:-1] + zl[1:])
        dec = np.exp(-zm / decay).astype(dtype)[:, None]
        wpat = np.sin(3 * lon * DEG2RAD + 0.9 * s) * np.cos(4 * lat * DEG2RAD)
        wz = (1.0 - np.exp(-zl / decay)).astype(dtype)[:, None]
        out.append(VelocityField(u=dec * u.astype(dtype)[None, :], v=dec * v.astype(dtype)[None, :],
                                 w=(w_amp * wz) * wpat.astype(dtype)[None, :], eta=np.zeros(lon.size),
                                 uv_layout="node", uv_vertical="layer"))
    return out


def release_uniform(mesh, P: int, seed: int = 3, *, depth_uniform: bool = False):
    """``P`` positions uniform in area over the mesh's elements (lon, lat, z)."""
    rng = np.random.default_rng(seed)
    en = np.asarray(mesh.elem_nodes)
    lon = np.asarray(mesh.nodes_lon)
    lat = np.asarray(mesh.nodes_lat)
    # split every element into fan triangles (0, k, k+1)
    tris = []
    for k in range(1, en.shape[1] - 1):
        t = np.stack([en[:, 0], en[:, k], en[:, k + 1]], 1)
        tris.append(t[(t >= 0).all(1)])
    t = np.concatenate(tris)
    la = lat[t]
    lo0 = lon[t[:, :1]]
    lo = lo0 + (((lon[t] - lo0) + 180.0) % 360.0 - 180.0)
    area = 0.5 * np.abs((lo[:, 1] - lo[:, 0]) * (la[:, 2] - la[:, 0]) - (lo[:, 2] - lo[:, 0]) * (la[:, 1] - la[:, 0]))
    area *= np.cos(la.mean(1) * DEG2RAD)
    pick = rng.choice(t.shape[0], size=P, p=area / area.sum())
    r1 = np.sqrt(rng.uniform(size=P))
    r2 = rng.uniform(size=P)
    b = np.stack([1 - r1, r1 * (1 - r2), r1 * r2], 1)
    plon = (b * lo[pick]).sum(1)
    plat = (b * la[pick]).sum(1)
    plon = ((plon + 180.0) % 360.0) - 180.0
    z = np.zeros(P)
    if depth_uniform:
        dep = np.asarray(mesh.depth)[t[pick]].min(1)
        z = rng.uniform(size=P) * dep
    return plon, plat, z


def sort_seeds(lon, lat, z, cell: float = 1.0):
    """Seed order for memory locality, as KELP's utils/sort_seeds.py prepares
    seed files before a run: a stable sort by lon/lat cell (``cell`` degrees,
    rows south to north) with the depth as the secondary key.  Returns the
    permuted (lon, lat, z)."""
    nx = int(np.ceil(360.0 / cell))
    key = (np.floor((np.asarray(lat) + 90.0) / cell).astype(np.int64) * nx
           + np.floor((np.asarray(lon) + 180.0) / cell).astype(np.int64) % nx)
    order = np.lexsort((np.asarray(z), key))
    return np.asarray(lon)[order], np.asarray(lat)[order], np.asarray(z)[order]


def tripolar_grid(ny: int, nx: int, *, fold: str = "T", cap_lat: float = 20.0, pole_lat: float = 65.0,
                  pole_lon: float = 73.0, south_lat: float = -78.0):
    """An ORCA-like tripolar raster in canonical form: ``(layout, glamf,
    gphif, glamt, gphit)``.  East-west periodic with one halo column each
    side (nx - 2 columns, 360 / (nx - 2) degrees apart) and a north fold
    pivoting on T or F points with one halo row.  South of ``cap_lat`` the
    rows are latitude circles, uniformly spaced from ``south_lat``; north of
    it a bipolar cap: in polar stereographic coordinates (the cap boundary
    the unit circle) a column runs straight from its boundary point to that
    point's projection on the segment between the two grid poles (at
    ``pole_lat``, ``pole_lon`` and ``pole_lon + 180``), which is the fold
    line; a column and its mirror image about the poles' meridian plane meet
    there.  The fold copies are set from their canonical points."""
    from .nemo import CgridLayout, to_canonical
    lay = CgridLayout((ny, nx), periodic=True, fold=fold)
    c0, w, J = lay.first_col, lay.width, lay.fold_row
    step = 360.0 / w
    fold_r = J + (0.5 if fold == "F" else 0.0)             # the fold line's row coordinate
    axis = np.radians(pole_lon - (0.5 * step if fold == "F" else 0.0))
    t_cap = np.tan(np.radians(90.0 - cap_lat) / 2.0)
    a = np.tan(np.radians(90.0 - pole_lat) / 2.0) / t_cap
    r_cap = round(fold_r * (cap_lat - south_lat) / (cap_lat - south_lat + (90.0 - cap_lat)))

    def points(oy, ox):
        r, i = np.meshgrid(np.arange(ny) + 0.5 * oy, np.arange(nx) + 0.5 * ox, indexing="ij")
        lam = np.radians(pole_lon + (i - c0) * step)
        lon = np.degrees(lam)
        lat = south_lat + (cap_lat - south_lat) * r / r_cap
        cap = r > r_cap
        s = (r[cap] - r_cap) / (fold_r - r_cap)
        proj = a * np.cos(lam[cap] - axis)
        px = (1.0 - s) * np.cos(lam[cap]) + s * proj * np.cos(axis)
        py = (1.0 - s) * np.sin(lam[cap]) + s * proj * np.sin(axis)
        rho = np.hypot(px, py)
        lon[cap] = np.degrees(np.arctan2(py, px))
        lat[cap] = 90.0 - np.degrees(2.0 * np.arctan(rho * t_cap))
        return ((lon + 180.0) % 360.0) - 180.0, lat

    flon, flat = points(1, 1)
    tlon, tlat = points(0, 0)
    return (lay, to_canonical(flon, lay, "F"), to_canonical(flat, lay, "F"), to_canonical(tlon, lay, "T"),
            to_canonical(tlat, lay, "T"))


def cgrid_stream_flow(glamf, gphif, amp: float = 5e5):
    """Face velocities of a smooth non-divergent flow on a C-grid raster, from
    a streamfunction psi (m^2/s) sampled at the F-points: the east-face (u)
    transport psi(F(j,i)) - psi(F(j-1,i)) over the face's great-circle length
    e2u, the north-face (v) transport psi(F(j,i-1)) - psi(F(j,i)) over e1v;
    every cell's net transport is zero.  psi is a smooth function of the
    unit-sphere position, so halo and fold copies agree.  Returns
    (u, v, e2u, e1v) rasters (the first row / column: the raster's own
    neighbours, edge-clamped)."""
    la, lo = np.radians(gphif), np.radians(glamf)
    x, y, z = np.cos(la) * np.cos(lo), np.cos(la) * np.sin(lo), np.sin(la)
    psi = amp * (0.6 * x * y + 0.5 * np.sin(2.0 * z + 0.3) * x + 0.4 * np.cos(3.0 * y) * z + 0.3 * z * z)

    def arc(j0, i0, j1, i1):
        dot = x[j0, i0] * x[j1, i1] + y[j0, i0] * y[j1, i1] + z[j0, i0] * z[j1, i1]
        return 6371000.0 * np.arccos(np.clip(dot, -1.0, 1.0))

    ny, nx = glamf.shape
    jj, ii = np.indices((ny, nx))
    js, iw = np.maximum(jj - 1, 0), np.maximum(ii - 1, 0)
    e2u = np.maximum(arc(js, ii, jj, ii), 1.0)
    e1v = np.maximum(arc(jj, iw, jj, ii), 1.0)
    u = (psi[jj, ii] - psi[js, ii]) / e2u
    v = (psi[jj, iw] - psi[jj, ii]) / e1v
    return u, v, e2u, e1v
