"""HEALPix NEST geometry and the dual mesh (pixel centres = nodes, corner
cells = elements) without healpy.

Written from the HEALPix projection (Gorski et al. 2005, ApJ 622:759;
Calabretta & Roukema 2007, MNRAS 381:865).  A NEST pixel id splits into a
base face (0-3 north, 4-7 equatorial, 8-11 south) and face-local integer
coordinates (ix, iy) by bit de-interleaving.  A face-local point (x, y) lies
on the iso-latitude ring j = jr[face] * nside - x - y (counted from the north
pole, 0 .. 4 nside) at longitude index x - y; in the polar caps
(j < nside, j > 3 nside) the longitude is compressed by j / nside.

The dual mesh follows KELP's ``build_healpix_dual_mesh``
(``src/kelp/readers/healpix.py:93-330``): one element per pixel corner whose
incident pixels are all wet (3 at the 8 valence-3 corners -> triangle, else a
quad), members in counter-clockwise order starting at the smallest pixel id,
elements ordered by (owner pixel, corner index N/E/S/W), orphan pixels
dropped, nodes in increasing NEST id.  Here the incident pixels of a corner
are found by grouping all pixels on an exact integer key of the corner point
instead of healpy's neighbour lists.
"""
from __future__ import annotations

import numpy as np

from .mesh import make_mesh

# ring of the southern corner of each base face, in units of nside
_JR = np.array([2, 2, 2, 2, 3, 3, 3, 3, 4, 4, 4, 4], dtype=np.int64)
# longitude of each base face's southern corner, in units of pi/4
_JP = np.array([1, 3, 5, 7, 0, 2, 4, 6, 1, 3, 5, 7], dtype=np.int64)


def nest_to_xyf(nside: int, pix: np.ndarray):
    """(face, ix, iy) of NEST pixel ids."""
    pix = np.asarray(pix, dtype=np.int64)
    npface = nside * nside
    face = pix // npface
    ipf = pix % npface
    ix = np.zeros_like(ipf)
    iy = np.zeros_like(ipf)
    bit = 0
    while (1 << (2 * bit)) < npface:
        ix |= ((ipf >> (2 * bit)) & 1) << bit
        iy |= ((ipf >> (2 * bit + 1)) & 1) << bit
        bit += 1
    return face, ix, iy


def xyf_to_zphi(nside: int, face, x, y):
    """(z = sin(lat), phi) of face-local points (x, y), continuous."""
    face = np.asarray(face, dtype=np.int64)
    x = np.asarray(x, dtype=np.float64)
    y = np.asarray(y, dtype=np.float64)
    ns = float(nside)
    j = _JR[face] * ns - x - y
    d = x - y
    phi_c = _JP[face] * (np.pi / 4.0)
    z = np.empty_like(j)
    phi = np.empty_like(j)
    north = j < ns
    south = j > 3 * ns
    eq = ~(north | south)
    z[eq] = (2 * ns - j[eq]) * 2.0 / (3 * ns)
    phi[eq] = (_JP[face[eq]] * ns + d[eq]) * (np.pi / (4 * ns))
    for m, jj, sgn in ((north, j, 1.0), (south, 4 * ns - j, -1.0)):
        if not m.any():
            continue
        jm = jj[m]
        z[m] = sgn * (1.0 - jm * jm / (3 * ns * ns))
        with np.errstate(divide="ignore", invalid="ignore"):
            ph = phi_c[m] + d[m] * np.pi / (4.0 * jm)
        phi[m] = np.where(jm > 0, ph, phi_c[m])
    return z, phi


def pix2lonlat(nside: int, pix: np.ndarray):
    """Centre longitude (wrapped to [-180, 180)) and latitude, degrees."""
    f, ix, iy = nest_to_xyf(nside, pix)
    z, phi = xyf_to_zphi(nside, f, ix + 0.5, iy + 0.5)
    lat = np.degrees(np.arcsin(np.clip(z, -1.0, 1.0)))
    lon = np.degrees(phi)
    return ((lon + 180.0) % 360.0) - 180.0, lat


def corner_key(nside: int, face, x, y) -> np.ndarray:
    """Exact integer key of the face-local integer corner (x, y): the ring j
    and the position around it (8 nside positions per ring)."""
    face = np.asarray(face, dtype=np.int64)
    x = np.asarray(x, dtype=np.int64)
    y = np.asarray(y, dtype=np.int64)
    j = _JR[face] * nside - x - y
    d = x - y
    idx = np.empty_like(j)
    eq = (j >= nside) & (j <= 3 * nside)
    idx[eq] = (_JP[face[eq]] * nside + d[eq]) % (8 * nside)
    for m, jj in ((j < nside, j), (j > 3 * nside, 4 * nside - j)):
        if not m.any():
            continue
        jm = jj[m]
        k = ((2 * (_JP[face[m]] // 2) + 1) * jm + d[m]) // 2
        idx[m] = np.where(jm > 0, k % np.maximum(4 * jm, 1), 0)
    return j * (8 * nside) + idx


def dual_mesh(nside: int, wet: np.ndarray | None = None, depth: np.ndarray | None = None, *, sigma=None,
              cell_size: float = 0.0, name: str = "healpix"):
    """The dual mesh of a NEST HEALPix grid (see the module docstring)."""
    npix = 12 * nside * nside
    wet = np.ones(npix, bool) if wet is None else np.asarray(wet, bool)
    pix = np.arange(npix, dtype=np.int64)
    f, ix, iy = nest_to_xyf(nside, pix)
    # corners k = 0 N, 1 E, 2 S, 3 W of every pixel
    cx = np.stack([ix + 1, ix + 1, ix, ix], 1)
    cy = np.stack([iy + 1, iy, iy, iy + 1], 1)
    keys = corner_key(nside, np.repeat(f, 4), cx.ravel(), cy.ravel())
    owner = np.repeat(pix, 4)
    kidx = np.tile(np.arange(4, dtype=np.int64), npix)
    order = np.lexsort((owner, keys))
    ks, ps, kk = keys[order], owner[order], kidx[order]
    starts = np.flatnonzero(np.r_[True, ks[1:] != ks[:-1]])
    counts = np.diff(np.r_[starts, ks.size])
    if not set(np.unique(counts)) <= {3, 4}:
        raise AssertionError("HEALPix corner grouping: a corner with other than 3 or 4 pixels")
    # members (up to 4) per corner, and the owner's corner index
    mem = np.full((starts.size, 4), -1, np.int64)
    for t in range(4):
        sel = counts > t
        mem[sel, t] = ps[starts[sel] + t]
    kown = kk[starts]                      # lexsort put the smallest pixel id first
    allwet = np.all(np.where(mem >= 0, wet[np.clip(mem, 0, npix - 1)], True), axis=1)
    mem, kown = mem[allwet], kown[allwet]
    # counter-clockwise order around the corner point, starting at the owner
    lon_all, lat_all = pix2lonlat(nside, np.clip(mem, 0, npix - 1).ravel())
    lon_all = lon_all.reshape(mem.shape)
    lat_all = lat_all.reshape(mem.shape)
    valid = mem >= 0
    ref_lon = lon_all[:, :1]
    dl = ((lon_all - ref_lon + 180.0) % 360.0) - 180.0
    cl = np.cos(np.radians(lat_all))
    nvalid = valid.sum(1, keepdims=True)
    mx = np.where(valid, dl * cl, 0.0).sum(1, keepdims=True) / nvalid
    my = np.where(valid, lat_all, 0.0).sum(1, keepdims=True) / nvalid
    ang = np.arctan2(np.where(valid, lat_all - my, 0.0), np.where(valid, dl * cl - mx, 0.0))
    # the two pole cells are degenerate in that chart: counter-clockwise seen
    # from outside is increasing longitude at the north pole, decreasing at
    # the south pole
    ckey = ks[starts][allwet]
    for pole_key, sgn in ((0, 1.0), (4 * nside * 8 * nside, -1.0)):
        pm = ckey == pole_key
        if pm.any():
            ang[pm] = sgn * np.radians(np.where(valid[pm], lon_all[pm], 0.0))
    ang = np.where(valid, ang, np.inf)
    a0 = ang[:, :1]
    with np.errstate(invalid="ignore"):
        rel = np.where(valid, (ang - a0) % (2 * np.pi), np.inf)
    perm = np.argsort(rel, axis=1, kind="stable")
    rows = np.take_along_axis(mem, perm, axis=1)
    ekey = (rows[:, 0] << 2) | kown
    o = np.argsort(ekey, kind="stable")
    rows = rows[o]
    node_pix = np.unique(rows[rows >= 0])
    remap = np.full(npix, -1, np.int64)
    remap[node_pix] = np.arange(node_pix.size)
    en = np.where(rows >= 0, remap[np.clip(rows, 0, npix - 1)], -1).astype(np.int32)
    lon, lat = pix2lonlat(nside, node_pix)
    d = np.zeros(node_pix.size) if depth is None else np.abs(np.asarray(depth, np.float64))[node_pix]
    m = make_mesh(name, lon, lat, d, en, sigma=sigma, cell_size=cell_size)
    m.metadata.update({"healpix_nside": nside, "healpix_npix": npix,
                       "n_triangles": int((en[:, 3] < 0).sum()), "n_quads": int((en[:, 3] >= 0).sum())})
    m.node_pix = node_pix
    return m
