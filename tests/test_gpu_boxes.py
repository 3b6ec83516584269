"""The containment tables change no result.

Each element's box (elem_box in kc_geom.cuh) may only reject a point that the
full element test rejects too, with the barycentric W search's own verdict;
each element's record (elem_record) holds the very vertex coordinates the
test would read through the node ids.  So with both tables, with neither and
with the boxes alone (KELP_B200_ELEM_BOXES=0 / KELP_B200_ELEM_RECORDS=0 at
mesh upload leave them out) every containment, every step and every state
array must be bit-identical:

* kc_find_elements on points that sit on the tolerance band: each element's
  vertices and edge midpoints nudged by +-1e-9 .. 1e-5 degrees, plus uniform
  points over the mesh;
* 48 steps of the 2-D (C1 shape), 3-D HEALPix (C3 shape, W barycentric,
  kick) and tripolar C-grid (C5 shape) workloads, plain and mixed forms.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


CONFIGS = {"both": ("1", "1"), "neither": ("0", "0"), "boxes only": ("1", "0")}


def _ctx(monkeypatch, config, mesh):
    from kelp_b200.device import DeviceContext
    boxes, records = CONFIGS[config]
    monkeypatch.setenv("KELP_B200_ELEM_BOXES", boxes)
    monkeypatch.setenv("KELP_B200_ELEM_RECORDS", records)
    ctx = DeviceContext(0)
    ctx.ensure_mesh(mesh)
    return ctx


def _band_points(mesh, rng, n_max=400_000):
    en = np.asarray(mesh.elem_nodes)
    lon, lat = np.asarray(mesh.nodes_lon), np.asarray(mesh.nodes_lat)
    sel = rng.choice(en.shape[0], size=min(en.shape[0], n_max // 8), replace=False)
    e = en[sel]
    a, b = e[:, 0], e[:, 1]
    pl = np.concatenate([lon[a], 0.5 * (lon[a] + lon[b])])
    pt = np.concatenate([lat[a], 0.5 * (lat[a] + lat[b])])
    pl = np.repeat(pl, 4)
    pt = np.repeat(pt, 4)
    mag = 10.0 ** rng.uniform(-9, -5, pl.size)
    ang = rng.uniform(0, 2 * np.pi, pl.size)
    pl = ((pl + mag * np.cos(ang) + 180.0) % 360.0) - 180.0
    pt = np.clip(pt + mag * np.sin(ang), -90.0, 90.0)
    ul = rng.uniform(lon.min(), lon.max(), n_max // 4)
    ut = rng.uniform(lat.min(), lat.max(), n_max // 4)
    return np.concatenate([pl, ul]), np.concatenate([pt, ut])


@pytest.mark.parametrize("wname", ["c1", "c3small", "c5small"])
def test_find_elements_same_with_and_without_boxes(monkeypatch, wname):
    from kelp_b200 import workloads as W
    wl = W.WORKLOADS[wname]()
    qlon, qlat = _band_points(wl.mesh, np.random.default_rng(7))
    out = {}
    for config in CONFIGS:
        ctx = _ctx(monkeypatch, config, wl.mesh)
        try:
            out[config] = ctx.find_elements(qlon, qlat)
        finally:
            ctx.close()
    diff = {c: int(np.count_nonzero(out[c] != out["both"])) for c in CONFIGS}
    print(f"{wname}: {qlon.size} points, {int(np.count_nonzero(out['both'] >= 0))} inside, differ {diff}")
    assert all(v == 0 for v in diff.values())


def _steps(ctx, wl, form, n, idx):
    from kelp_b200 import _native as N
    if wl.dims == 3 and wl.uv_vertical != "layer":
        ctx.ensure_depth_points(wl.mesh, wl.uv_vertical)
    slots = ctx.slots_for(wl.snaps, np.float32)
    P = idx.size
    ctx.upload_particles(wl.lon[idx], wl.lat[idx], wl.z[idx], np.ones(P, np.int32), np.full(P, -1, np.int32),
                         np.zeros(P, np.int8), np.arange(P, dtype=np.int64))
    code = N.KC_MIXED if form == "mixed" else N.KC_PLAIN
    for k in range(n):
        if k % 16 == 0:
            ctx.sort()
        ctx.step(wl.step_args(k, slots, code))
    ctx.synchronize()
    assert ctx.device_errors() == 0
    return ctx.download_particles()


def _ndiff(a, b):
    a, b = np.asarray(a), np.asarray(b)
    same = a == b
    if a.dtype.kind == "f":
        same |= np.isnan(a) & np.isnan(b)
    return int(np.count_nonzero(~same))


@pytest.mark.parametrize("wname", ["c1", "c3small", "c5small"])
@pytest.mark.parametrize("form", ["plain", "mixed"])
def test_steps_same_with_and_without_boxes(monkeypatch, wname, form):
    from kelp_b200 import workloads as W
    wl = W.WORKLOADS[wname]()
    idx = np.random.default_rng(3).choice(wl.P, size=min(wl.P, 100_000), replace=False)
    out = {}
    for config in CONFIGS:
        ctx = _ctx(monkeypatch, config, wl.mesh)
        try:
            out[config] = _steps(ctx, wl, form, 48, idx)
        finally:
            ctx.close()
    ref = out["both"]
    rep = {c: {k: _ndiff(ref[k], out[c][k]) for k in ref if ref[k] is not None} for c in CONFIGS if c != "both"}
    print(f"{wname} {form}: {rep}")
    assert all(v == 0 for r in rep.values() for v in r.values()), rep
