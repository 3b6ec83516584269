"""The mixed-precision form against the plain float64 form on the GPU.

The mixed form keeps the anchor, containment and vertical decisions in
float64 and interpolates in float32 (float32 or scaled float16 snapshots).
Its particles therefore follow the plain form's to within the float32
interpolation error: after the horizons below, p99 great-circle separation
under 1 m with float32 snapshots, and the float16 storage error bound
(relative 2^-11 of each value) with float16 snapshots.
"""
import numpy as np
import pytest

from kelp_b200 import accuracy as A
from kelp_b200 import integrators as KI
from kelp_b200.diffusion import DiffusionStepArgs

pytestmark = pytest.mark.gpu


def _run(g, cname, **kw):
    c = g.case(cname)
    dt, T, n_steps, td, khx, khy, seed, real_id, pid_off = c["params"]
    scheme = cname.split("_")[0]
    w_interp = "barycentric" if "wbary" in cname else "nearest"
    fn = KI.get_integrator(scheme)
    st = g.particles()
    for k in range(int(n_steps)):
        vel, vnext, dtn = g.payload(c["schedule"][k], T)
        diff = None
        if khx >= 0:
            diff = DiffusionStepArgs("uniform", khx, khy, int(seed), int(real_id), k, pid_offset=int(pid_off))
        st = fn(st, vel, g.mesh, dt, td, uv_interp="barycentric", w_interp=w_interp, vel_next=vnext,
                dt_to_next=dtn, diffusion=diff, **kw)
    return {"lon": st.lon, "lat": st.lat, "z": st.z, "status": st.status, "nearest_node": st.nearest_node}


CASES = [("golden_band", "rk2"), ("golden_band", "rk4_kick_aniso"), ("golden_quad", "rk2_kick"),
         ("golden_3d", "rk2_wbary_kick"), ("golden_3d", "rk4_wnear"), ("golden_dl_lev", "rk2_lev_wbary"),
         ("golden_dl_llin", "rk4_llin_wnear_kick")]


@pytest.mark.parametrize("fixture,cname", CASES)
def test_mixed_f32_tracks_plain(golden, fixture, cname):
    g = golden(fixture)
    ref = _run(g, cname)
    mx = _run(g, cname, cuda_precision="mixed")
    s = A.separation_stats(ref, mx)
    print(fixture, cname, s)
    assert s["compared"] > 100
    assert s["status_mismatch"] <= max(2, ref["status"].size // 500)
    assert s["p99_m"] < 1.0, s
    # an unchanged position decides the same anchor: the element path is the plain one
    same = (ref["status"] == 1) & (mx["status"] == 1) & (ref["lon"] == mx["lon"]) & (ref["lat"] == mx["lat"])
    np.testing.assert_array_equal(ref["nearest_node"][same], mx["nearest_node"][same])


@pytest.mark.parametrize("fixture,cname", [("golden_band", "rk2"), ("golden_3d", "rk2_wbary_kick")])
def test_mixed_f16_snapshots_bounded(golden, fixture, cname):
    g = golden(fixture)
    ref = _run(g, cname)
    mx = _run(g, cname, cuda_precision="mixed", cuda_snapshots="f16")
    s = A.separation_stats(ref, mx)
    print(fixture, cname, "f16", s)
    c = g.case(cname)
    dt, T, n_steps = c["params"][:3]
    umax = max(float(np.abs(np.asarray(sn.u)).max()) for sn in g.snaps)
    # each stored value within 2^-11 of its magnitude; a step moves a particle
    # by dt times a weighted mean of such values
    bound = n_steps * dt * umax * 2.0 ** -11
    assert s["p99_m"] < bound, (s, bound)
    assert s["status_mismatch"] <= max(3, ref["status"].size // 200)


def test_plain_rejects_f16_and_mixed_rejects_f64(golden):
    from kelp_b200 import _native as N
    g = golden("golden_quad")   # float64 snapshots
    c = g.case("rk2")
    st = g.particles()
    vel, vnext, dtn = g.payload(c["schedule"][0], c["params"][1])
    with pytest.raises(ValueError):
        KI.rk2_step(st, vel, g.mesh, 3600.0, 1.0, uv_interp="barycentric", vel_next=vnext, dt_to_next=dtn,
                    cuda_snapshots="f16")
    # mixed with float64 inputs stores them as float32: runs
    out = KI.rk2_step(st, vel, g.mesh, 3600.0, 1.0, uv_interp="barycentric", vel_next=vnext, dt_to_next=dtn,
                      cuda_precision="mixed")
    assert np.isfinite(out.lon).all()


@pytest.mark.parametrize("storage,bound_m", [("f32", 1.0), ("f16", 50.0)])
def test_mixed_cgrid_tracks_plain(storage, bound_m):
    """The mixed form's 3-D C-grid step (float32 values and fluxes on float32
    or scaled float16 face rasters, float64 geometry) on the tripolar C5-shaped
    workload against the plain form over 24 one-hour RK4 steps: p99
    separation under 1 m on float32 rasters; float16 rasters within their
    storage error (p99 under 50 m after a day)."""
    from kelp_b200 import workloads as W
    from kelp_b200.fields import LazyLerpField
    from kelp_b200.particles import make_state
    w = W.c5_small(P=20_000)
    out = {}
    for form, snaps in (("plain", None), ("mixed", storage)):
        st = make_state(w.lon, w.lat, w.z).replace(failure_reason=np.zeros(w.P, np.int8))
        for k in range(24):
            ia, ib, a0, dtn = w.bracket(k)
            a, b = w.snaps[ia], w.snaps[ib]
            vel = a if a0 == 0.0 else LazyLerpField(a, b, a0)
            st = KI.rk4_step(st, vel, w.mesh, w.dt, 1.0, uv_interp="nemo_cgrid", vel_next=b, dt_to_next=dtn,
                             cuda_precision=form, cuda_snapshots=snaps)
        out[form] = {"lon": st.lon, "lat": st.lat, "z": st.z, "status": st.status, "nearest_node": st.nearest_node}
    s = A.separation_stats(out["plain"], out["mixed"])
    print("cgrid mixed", storage, s)
    assert s["compared"] > 10_000
    assert s["status_mismatch"] <= 20
    assert s["p99_m"] < bound_m, s
