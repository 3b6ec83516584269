"""The pruned 3x3 windows of the nearest-node scan: on query sets built to
stress the pruning -- points on grid-hash cell edges and corners, on the
bisectors of neighbouring nodes (ties and near-ties), on the nodes, near the
poles and the dateline -- the device's nearest node with pruned windows is the
whole-window scan's, bit for bit, and both equal the oracle's exact nearest
(mesh.py:1611-1859) wherever the query is not an engineered tie; on a global
HEALPix dual mesh and on the golden meshes."""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _healpix_mesh(nside=64):
    from kelp_b200 import healpix as H
    from kelp_b200 import synthetic as S
    pix = np.arange(12 * nside * nside)
    plon, plat = H.pix2lonlat(nside, pix)
    wet = S._sphere_noise(plon, plat, seed=2) >= np.quantile(S._sphere_noise(plon, plat, seed=2), 0.3)
    return H.dual_mesh(nside, wet, S.smooth_bathymetry(plon, plat, 50.0, 6000.0))


def _stress_queries(m, n=60_000, seed=7):
    """(lon, lat, tie): the query set, and which queries were built to sit on a
    bisector (exact or near ties, where the last ulp of the query's trig --
    CUDA's against the C library's -- may pick either node): node-pair
    midpoints, element centroids, and the dateline, where a mesh symmetric
    about 180 degrees (HEALPix rings) puts two nodes at the same distance."""
    rng = np.random.default_rng(seed)
    lon0, lat0 = np.asarray(m.nodes_lon), np.asarray(m.nodes_lat)
    cell, lo, la = m._gh_cell_size, m._gh_lon_min, m._gh_lat_min
    q = [np.c_[rng.uniform(-180, 180, n), np.degrees(np.arcsin(rng.uniform(-1, 1, n)))]]
    # cell edges and corners, exactly and one rounding either side
    i = rng.integers(0, m._gh_nx + 1, n)
    j = rng.integers(0, m._gh_ny + 1, n)
    e_lon = lo + i * cell
    e_lat = np.clip(la + j * cell, -90.0, 90.0)
    for s in (-1, 0, 1):
        q.append(np.c_[np.nextafter(e_lon, e_lon + s), rng.uniform(-90, 90, n)])
        q.append(np.c_[rng.uniform(-180, 180, n), np.clip(np.nextafter(e_lat, e_lat + s), -90, 90)])
        q.append(np.c_[np.nextafter(e_lon, e_lon + s), np.clip(np.nextafter(e_lat, e_lat + s), -90, 90)])
    q.append(np.c_[lon0, lat0])
    q.append(np.c_[rng.uniform(-180, 180, n), rng.uniform(80, 90, n) * rng.choice([-1, 1], n)])
    n_plain = sum(a.shape[0] for a in q)
    # the dateline: on a mesh symmetric about 180 degrees every such point is a tie
    q.append(np.c_[rng.choice([-180.0, 180.0, np.nextafter(180.0, 0), np.nextafter(-180.0, 0)], n),
                   rng.uniform(-89, 89, n)])
    # bisectors of node pairs that share an element: midpoints, and a hair either way
    en = np.asarray(m.elem_nodes)
    k = rng.integers(0, en.shape[0], n)
    a, b = en[k, 0], en[k, 1]
    xyz = O.node_xyz(lon0, lat0)
    mid = xyz[a] + xyz[b]
    mid /= np.linalg.norm(mid, axis=1, keepdims=True)
    mlon, mlat = np.degrees(np.arctan2(mid[:, 1], mid[:, 0])), np.degrees(np.arcsin(np.clip(mid[:, 2], -1, 1)))
    for eps in (0.0, 1e-13, -1e-13, 1e-9, -1e-9):
        q.append(np.c_[mlon + eps, mlat - eps])
    # the mean of an element's first three vertices (three-way near ties)
    c3 = xyz[en[k, 0]] + xyz[en[k, 1]] + xyz[en[k, 2]]
    c3 /= np.linalg.norm(c3, axis=1, keepdims=True)
    q.append(np.c_[np.degrees(np.arctan2(c3[:, 1], c3[:, 0])), np.degrees(np.arcsin(np.clip(c3[:, 2], -1, 1)))])
    Q = np.concatenate(q)
    tie = np.zeros(Q.shape[0], bool)
    tie[n_plain:] = True
    return np.ascontiguousarray(Q[:, 0]), np.ascontiguousarray(Q[:, 1]), tie


def _whole_window_context(monkeypatch, m):
    """A second device context whose mesh upload keeps the whole windows."""
    from kelp_b200.device import DeviceContext
    monkeypatch.setenv("KELP_B200_PRUNED_WINDOWS", "0")
    ctx = DeviceContext(0)
    ctx.ensure_mesh(m)
    monkeypatch.delenv("KELP_B200_PRUNED_WINDOWS")
    return ctx


def _check(monkeypatch, m, lon, lat, tie):
    from kelp_b200.device import default_context
    ctx = default_context()
    ctx.ensure_mesh(m)
    got = ctx.find_nearest(lon, lat)
    whole = _whole_window_context(monkeypatch, m)
    try:
        want = whole.find_nearest(lon, lat)
    finally:
        whole.close()
    # the pruned scan is the whole-window scan, bit for bit, on every query
    bad = np.flatnonzero(got != want)
    assert bad.size == 0, (bad.size, bad[:10], got[bad[:10]], want[bad[:10]])
    # and both are the reference's exact nearest away from engineered ties
    ref = O.find_nearest(m, lon, lat)
    off = np.flatnonzero((got != ref) & ~tie)
    assert off.size == 0, (off.size, lon[off[:5]], lat[off[:5]], got[off[:5]], ref[off[:5]])


def test_pruned_nearest_equals_whole_window_healpix(monkeypatch):
    m = _healpix_mesh()
    _check(monkeypatch, m, *_stress_queries(m))


@pytest.mark.parametrize("fixture", ["golden_band", "golden_quad", "golden_polar"])
def test_pruned_nearest_equals_whole_window_golden(monkeypatch, golden, fixture):
    m = golden(fixture).mesh
    _check(monkeypatch, m, *_stress_queries(m, n=20_000))
