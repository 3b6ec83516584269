"""A 3-D RK2 step whose payload is an endpoint LazyLerpField (alpha 0).

The reference routes that payload to its unfused RK2
(src/kelp/numerics/integrators.py:5691-5692 -> :5380-5608), which steps the
payload materialised by its own blend.  tests/golden/golden_lazy0.npz holds
the reference's outputs over 10 steps on the 3-D z-level mesh of golden_3d
(W barycentric; W nearest with the split kick), each step's payload
LazyLerpField(record ia, record ia + 1, 0.0) with record ia + 1 as vel_next.

CPU: the oracle, stepping the materialised field, equals the recorded run
bit for bit.  GPU: kelp_b200's rk2_step on the same LazyLerpField payloads,
within the parity tolerances of the other golden runs.
"""
import numpy as np
import pytest

CASES = ("rk2_wbary", "rk2_wnear_kick")


def _schedule(g, k, dt, T):
    from kelp_b200.fields import LazyLerpField
    t = k * dt
    ia = int(np.floor(t / T + 1e-9))
    return LazyLerpField(g.snaps[ia], g.snaps[ia + 1], 0.0), g.snaps[ia + 1], (ia + 1) * T - t


def _diffusion(c, k):
    from kelp_b200.diffusion import DiffusionStepArgs
    dt, T, n, td, khx, khy, seed = c["params"]
    return None if khx < 0 else DiffusionStepArgs("uniform", khx, khy, int(seed), 0, k)


@pytest.mark.parametrize("cname", CASES)
def test_oracle_matches_reference(golden, cname):
    from oracle import oracle as O
    from kelp_b200.integrators import _materialized
    g = golden("golden_lazy0")
    c = g.case(cname)
    dt, T, n = float(c["params"][0]), float(c["params"][1]), int(c["params"][2])
    w_interp = "barycentric" if "wbary" in cname else "nearest"
    st = g.particles()
    view = O.MeshView(g.mesh)
    for k in range(n):
        vel, vnext, dtn = _schedule(g, k, dt, T)
        out = O.step(st, _materialized(vel), g.mesh, dt, 1.0, "rk2", vel_next=vnext, dt_to_next=dtn,
                     w_interp=w_interp, diffusion=_diffusion(c, k), view=view)
        st = st.replace(lon=out["lon"], lat=out["lat"], z=out["z"], status=out["status"],
                        nearest_node=out["nearest_node"], failure_reason=out["failure_reason"],
                        u=out["u"], v=out["v"], w=out["w"])
    for name in ("status", "nearest_node", "failure_reason", "lon", "lat", "z", "u", "v", "w"):
        assert np.array_equal(np.asarray(getattr(st, name)), c[f"s{n}_{name}"]), name


def test_materialized_is_the_payloads_blend():
    from kelp_b200.fields import LazyLerpField, VelocityField
    from kelp_b200.integrators import _materialized
    a = VelocityField(u=np.array([[1.0, -0.0]]), v=np.array([[2.0, 3.0]]), eta=np.zeros(2), w=np.ones((2, 2)),
                      uv_layout="node")
    b = VelocityField(u=np.array([[np.nan, 5.0]]), v=np.array([[4.0, np.inf]]), eta=np.ones(2),
                      w=np.zeros((2, 2)), uv_layout="node")
    m = _materialized(LazyLerpField(a, b, 0.0))
    assert np.isnan(m.u[0, 0]) and m.u[0, 1] == 0.0 and not np.signbit(m.u[0, 1])   # 1.0 a + 0.0 b
    assert m.v[0, 0] == 2.0 and np.isnan(m.v[0, 1]) and np.array_equal(m.eta, [0.0, 0.0])


@pytest.mark.gpu
@pytest.mark.parametrize("cname", CASES)
def test_cuda_matches_reference(golden, cname):
    from kelp_b200 import integrators as KI
    from test_gpu_parity import assert_close_state
    g = golden("golden_lazy0")
    c = g.case(cname)
    dt, T, n = float(c["params"][0]), float(c["params"][1]), int(c["params"][2])
    w_interp = "barycentric" if "wbary" in cname else "nearest"
    st = g.particles()
    for k in range(n):
        vel, vnext, dtn = _schedule(g, k, dt, T)
        st = KI.rk2_step(st, vel, g.mesh, dt, 1.0, uv_interp="barycentric", w_interp=w_interp, vel_next=vnext,
                         dt_to_next=dtn, diffusion=_diffusion(c, k))
    assert_close_state(st, c, f"s{n}_", f"golden_lazy0/{cname}")
