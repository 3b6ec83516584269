"""The C-grid step on the C5-shaped workload (kelp_b200.workloads.c5_small:
a curvilinear raster with partial bottom cells, 75 levels, the mesh built by
kelp_b200.nemo.build_cgrid_mesh) against the oracle: statuses, anchors and
failure reasons bit-exact, positions and depths within the kernels'
tolerance, over several RK4 steps that cross records."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

POS_TOL_DEG = 1e-9 / 0.017453292519943295


def test_c5small_rk4_matches_oracle():
    from oracle import oracle as O
    from kelp_b200 import integrators as KI
    from kelp_b200.fields import LazyLerpField
    from kelp_b200.particles import make_state
    from kelp_b200 import workloads as W
    w = W.c5_small(P=20_000)
    st = make_state(w.lon, w.lat, w.z).replace(failure_reason=np.zeros(w.P, np.int8))
    ref = st
    view = O.MeshView(w.mesh)
    for k in range(6):
        ia, ib, a0, dtn = w.bracket(k * 20)   # steps spread over the record interval
        a, b = w.snaps[ia], w.snaps[ib]
        vel = a if a0 == 0.0 else LazyLerpField(a, b, a0)
        st = KI.rk4_step(st, vel, w.mesh, w.dt, 1.0, uv_interp="nemo_cgrid", vel_next=b, dt_to_next=dtn)
        out = O.step(ref, vel, w.mesh, w.dt, 1.0, "rk4", vel_next=b, dt_to_next=dtn, view=view)
        ref = ref.replace(lon=out["lon"], lat=out["lat"], z=out["z"], status=out["status"],
                          nearest_node=out["nearest_node"], failure_reason=out["failure_reason"])
        for name in ("status", "nearest_node", "failure_reason"):
            np.testing.assert_array_equal(getattr(st, name), out[name], err_msg=f"step {k} {name}")
        d = np.abs(((st.lon - out["lon"]) + 180.0) % 360.0 - 180.0)
        assert d.max() <= POS_TOL_DEG, f"step {k} lon {d.max():.3e}"
        assert np.abs(st.lat - out["lat"]).max() <= POS_TOL_DEG
        assert np.abs(st.z - out["z"]).max() <= 1e-6
        np.testing.assert_allclose(st.w, out["w"], rtol=0, atol=1e-9)
    assert (st.status == 1).mean() > 0.9
