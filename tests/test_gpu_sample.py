"""kelp_b200.sampling.sample_field (kc_sample_field) against the reference.

* The reference's own outputs (tests/golden/golden_sample_*.npz): 2-D node
  fields on a seam-wrapping band and a tri/quad mesh, a z-level mid-layer
  field on a 3-D band; every method; fill NaNs, points on nodes, dead
  particles, nearest = -1.
* The anchors found on the device (nearest=None) against the oracle's.
* 200 k points on the C3-shaped HEALPix mesh (nside 128, 69 levels) against
  the oracle, every method, 2-D and mid-layer fields.

Bar: the NaN pattern identical; finite values within 1e-12 relative (the
device's cos is correctly rounded where the C library may be 1 ulp off).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
METHODS = ("nearest", "leastsq", "barycentric", "idw")


def _check(got, want, tag):
    got, want = np.asarray(got), np.asarray(want)
    nan_mm = int(np.count_nonzero(np.isnan(got) != np.isnan(want)))
    fin = np.isfinite(want) & np.isfinite(got)
    rel = np.abs(got[fin] - want[fin]) / np.maximum(np.abs(want[fin]), 1e-300)
    worst = float(rel.max()) if rel.size else 0.0
    exact = int(np.count_nonzero(got[fin] == want[fin]))
    print(f"{tag}: {want.size} points, {int(fin.sum())} finite, {exact} bit-equal, max rel {worst:.2e}, "
          f"NaN mismatches {nan_mm}")
    assert nan_mm == 0
    assert worst <= 1e-12


@pytest.mark.parametrize("name", ["band", "quad", "3d"])
@pytest.mark.parametrize("method", METHODS)
def test_sample_matches_reference_goldens(golden, name, method):
    from kelp_b200.sampling import sample_field
    g = golden(f"golden_sample_{name}")
    d = g.d
    got = sample_field(d["v2"], g.mesh, d["lon"], d["lat"], nearest=d["nearest"], alive=d["alive"], method=method)
    _check(got, d[f"o2_{method}"], f"{name} 2-D {method}")
    if "v3" in d:
        got3 = sample_field(d["v3"], g.mesh, d["lon"], d["lat"], d["z"], nearest=d["nearest"], alive=d["alive"],
                            method=method)
        _check(got3, d[f"o3_{method}"], f"{name} mid-layer {method}")


def test_sample_device_anchors(golden):
    from kelp_b200.sampling import sample_field
    from oracle import oracle as O
    g = golden("golden_sample_3d")
    d = g.d
    for method in METHODS:
        got = sample_field(d["v3"], g.mesh, d["lon"], d["lat"], d["z"], method=method)
        want = O.sample_field(d["v3"], g.mesh, d["lon"], d["lat"], d["z"], method=method)
        _check(got, want, f"device anchors {method}")


def test_sample_at_scale_against_oracle():
    from kelp_b200 import workloads as W
    from kelp_b200.sampling import sample_field
    from oracle import oracle as O
    wl = W.WORKLOADS["c3small"]()
    m = wl.mesh
    lo, la = np.asarray(m.nodes_lon), np.asarray(m.nodes_lat)
    zl = np.abs(np.asarray(m.sigma))
    zmid = 0.5 * (zl[:-1] + zl[1:])
    rng = np.random.default_rng(4)
    v2 = 15.0 + 10.0 * np.cos(np.radians(la)) + np.sin(np.radians(3.0 * lo))
    v2[rng.choice(lo.size, lo.size // 50, replace=False)] = np.nan
    v3 = 2.0 + 25.0 * np.exp(-zmid[:, None] / 900.0) * (1.0 + 0.2 * np.cos(np.radians(2.0 * lo)))[None, :]
    v3[zmid[:, None] > np.asarray(m.depth)[None, :]] = np.nan
    P = wl.P
    view = O.MeshView(m)
    nn = O.find_nearest(m, wl.lon, wl.lat, view)
    for method in METHODS:
        got = sample_field(v2, m, wl.lon, wl.lat, method=method)
        _check(got, O.sample_field(v2, m, wl.lon, wl.lat, nearest=nn, method=method, view=view),
               f"c3small 2-D {method} ({P} points)")
        got3 = sample_field(v3, m, wl.lon, wl.lat, wl.z, method=method)
        _check(got3, O.sample_field(v3, m, wl.lon, wl.lat, wl.z, nearest=nn, method=method, view=view),
               f"c3small mid-layer {method}")


@pytest.mark.parametrize("method", METHODS)
def test_interface_field_matches_reference(golden, method):
    """An interface-shaped (K, N) field through the W interpolation of the
    method (sampling.py:876-890), against the reference's own outputs."""
    from kelp_b200.sampling import sample_field
    g = golden("golden_sample_iface")
    d = g.d
    got = sample_field(d["vk"], g.mesh, d["lon"], d["lat"], d["z"], nearest=d["nearest"], alive=d["alive"],
                       method=method)
    _check(got, d[f"ok_{method}"], f"interface {method}")


@pytest.mark.parametrize("method", ("nearest", "leastsq", "idw"))
def test_sigma_fields_match_reference(golden, method):
    """Sigma-mesh sampling (sampling.py:620-723) on the device: interface and
    mid-layer fields with the free surface, against the reference's outputs."""
    from kelp_b200.sampling import sample_field
    g = golden("golden_sample_sigma")
    d = g.d
    for key, out in (("vk", "ok"), ("vm", "om")):
        got = sample_field(d[key], g.mesh, d["lon"], d["lat"], d["z"], nearest=d["nearest"], alive=d["alive"],
                           eta=d["eta"], method=method, Dmin=0.5)
        _check(got, d[f"{out}_{method}"], f"sigma {key} {method}")
