"""CUDA step kernels against the reference's own outputs (golden fixtures) and
against the CPU oracle at larger sizes.

Bar: status, nearest node and failure reason bit-exact; positions within
1e-9 rad (5.7e-8 degrees), depths within 1e-6 m, velocities within 1e-9 m/s.
The floating-point tolerance covers the last-place differences between
CUDA's and the C library's trigonometric functions; the integer bar does not
move.
"""
import numpy as np
import pytest

from kelp_b200 import integrators as KI
from kelp_b200.diffusion import DiffusionStepArgs

from test_oracle_golden import (CGRID_CASES, EDGE_CASES, LSQ_CASES, PCHIP_CASES, SIGMA_CASES, diffusion_args, edge_kw,
                                recon_of, surfaces_of, uv_interp_of, w_interp_of)

pytestmark = pytest.mark.gpu

POS_TOL_DEG = 1e-9 / 0.017453292519943295
Z_TOL = 1e-6
VEL_TOL = 1e-9

CASES = [("golden_band", c) for c in ("rk2", "rk4", "euler", "rk2_bwd", "rk2_kick", "rk4_kick_aniso", "rk2_dt4800")]
CASES += [("golden_quad", c) for c in ("rk2", "rk4", "euler", "rk2_kick")]
CASES += [("golden_polar", "rk2")]
CASES += [("golden_3d", c) for c in ("rk2_wnear", "rk2_wbary", "rk2_wbary_kick", "rk4_wnear", "rk4_wbary_kick", "euler_wbary",
                                     "rk2_wbary_kick_azf", "rk4_wnear_azf_nokh")]
CASES += [("golden_dl_lev", c) for c in ("rk2_lev_wbary", "rk4_lev_wnear_kick", "euler_lev_wnear", "rk2_lev_wbary_azc")]
CASES += [("golden_dl_llin", c) for c in ("rk2_llin_wbary", "rk4_llin_wnear_kick", "euler_llin_wnear")]
CASES += [("golden_wring", c) for c in ("rk2_wlsq", "rk4_wlsq_kick", "euler_wlsq", "rk2_wlsq_bwd", "rk2_widw",
                                        "rk4_widw_kick")]
# elem_search: walk (carried elements in and out of every step)
WALK_CASES = [("golden_band", c) for c in ("rk2_walk", "rk4_walk_kick", "euler_walk")]
WALK_CASES += [("golden_3d", c) for c in ("rk2_wbary_walk", "rk4_wnear_walk_kick")]
CASES += WALK_CASES
CASES += SIGMA_CASES
CASES += CGRID_CASES
CASES += LSQ_CASES
CASES += EDGE_CASES
CASES += PCHIP_CASES


def replay_cuda(g, cname):
    c = g.case(cname)
    dt, T, n_steps, td, khx, khy, seed, real_id, pid_off = c["params"]
    scheme = cname.split("_")[0]
    fn = KI.get_integrator(scheme)
    w_interp = w_interp_of(cname)
    st = g.particles()
    if "elem0" in c:   # elem_search: walk
        st = st.replace(elem=c["elem0"].copy())
    snaps = {}
    for k in range(int(n_steps)):
        vel, vnext, dtn = g.payload(c["schedule"][k], T)
        diff = diffusion_args(c, k)
        uv = uv_interp_of(g)
        rc = recon_of(g, c, k)
        extra = {} if rc is None else {"recon": rc}
        for key, e in zip(("sigma_eta_start", "sigma_eta_end"), surfaces_of(c, k)):
            if e is not None:
                extra[key] = e
        extra.update(edge_kw(g, cname))
        st = fn(st, vel, g.mesh, dt, td, uv_interp=uv, w_interp=w_interp, vel_next=vnext,
                dt_to_next=dtn, diffusion=diff, **extra)
        if f"s{k + 1}_lon" in c:
            snaps[k + 1] = st
    return c, snaps


def assert_close_state(st, c, tag, where):
    for name in ("status", "nearest_node", "failure_reason", "elem"):
        if tag + name not in c:
            continue
        got = np.asarray(getattr(st, name))
        bad = np.flatnonzero(got != c[tag + name])
        assert bad.size == 0, f"{where} {name}: {bad.size} mismatches, first at {bad[:5]}"
    for name, tol in (("lon", POS_TOL_DEG), ("lat", POS_TOL_DEG), ("z", Z_TOL), ("u", VEL_TOL), ("v", VEL_TOL),
                      ("w", VEL_TOL)):
        if tag + name not in c:
            continue
        got = np.asarray(getattr(st, name))
        want = c[tag + name]
        if name == "lon":
            d = np.abs(((got - want) + 180.0) % 360.0 - 180.0)
        else:
            d = np.abs(got - want)
        assert d.max() <= tol, f"{where} {name}: max |diff| {d.max():.3e} > {tol:.1e}"


@pytest.mark.parametrize("fixture,cname", CASES)
def test_cuda_matches_reference(golden, fixture, cname):
    g = golden(fixture)
    c, snaps = replay_cuda(g, cname)
    for k, st in snaps.items():
        assert_close_state(st, c, f"s{k}_", f"{fixture}/{cname} step {k}")


@pytest.mark.parametrize("fixture", ["golden_quad", "golden_polar"])
def test_cuda_exact_nearest(golden, fixture):
    from kelp_b200.device import default_context
    g = golden(fixture)
    ctx = default_context()
    ctx.ensure_mesh(g.mesh)
    got = ctx.find_nearest(g.d["p_q_lon"], g.d["p_q_lat"])
    np.testing.assert_array_equal(got, g.d["p_q_nearest"])


def _c1_like(P=20000, spacing=1.5):
    from kelp_b200 import synthetic as S
    m = S.lattice_mesh(spacing, 80.0)
    snaps = S.gyre_snapshots(m, 2, amp=0.5)
    lon, lat, z = S.release_uniform(m, P, seed=3)
    return m, snaps, lon, lat


@pytest.mark.parametrize("scheme", ["rk2", "rk4"])
def test_cuda_vs_oracle_c1_like(scheme):
    """A C1-shaped 2-D run (global lattice, land mask, f32 fields, temporal
    interpolation, dt 1 h) over 48 steps: CUDA against the oracle."""
    from oracle import oracle as O
    from kelp_b200.particles import make_state
    from kelp_b200.fields import LazyLerpField
    m, snaps, lon, lat = _c1_like()
    T, dt = 86400.0, 3600.0
    st = make_state(lon, lat)
    st = st.replace(failure_reason=np.zeros(lon.size, np.int8))
    so = st
    view = O.MeshView(m)
    fn = KI.get_integrator(scheme)
    for k in range(48):
        t = (k * dt) % T
        a, b = (snaps[0], snaps[1]) if (k * dt) // T % 2 == 0 else (snaps[1], snaps[0])
        alpha = t / T
        vel = a if alpha == 0 else LazyLerpField(a, b, alpha)
        st = fn(st, vel, m, dt, 1.0, uv_interp="barycentric", vel_next=b, dt_to_next=T - t)
        out = O.step(so, vel, m, dt, 1.0, scheme, vel_next=b, dt_to_next=T - t, view=view)
        so = so.replace(lon=out["lon"], lat=out["lat"], status=out["status"], nearest_node=out["nearest_node"],
                        failure_reason=out["failure_reason"], u=out["u"], v=out["v"])
    want = {f"f_{k}": getattr(so, k) for k in ("lon", "lat", "status", "nearest_node", "failure_reason", "u", "v")}
    assert_close_state(st, want, "f_", f"c1-like {scheme}")


def test_resident_loop_with_resort_matches_oracle():
    """The device-resident loop (kc_run over per-step arguments) with a
    re-sort by hash cell every 3 steps returns, in upload order, exactly what
    the oracle computes: the order of the particles does not change any
    result (each keeps its RNG key)."""
    from oracle import oracle as O
    from kelp_b200 import workloads as W
    from kelp_b200.device import DeviceContext
    from kelp_b200.particles import make_state
    from kelp_b200.fields import LazyLerpField
    w = W.c3(P=15000, nside=32)
    ctx = DeviceContext(0)
    ctx.ensure_mesh(w.mesh)
    slots = ctx.slots_for(w.snaps)
    P = w.P
    ctx.upload_particles(w.lon, w.lat, w.z, np.ones(P, np.int32), np.full(P, -1, np.int32), np.zeros(P, np.int8))
    so = make_state(w.lon, w.lat, w.z).replace(failure_reason=np.zeros(P, np.int8))
    view = O.MeshView(w.mesh)
    for k in range(9):
        if k % 3 == 0:
            ctx.sort()
        ctx.run([w.step_args(k, slots)])
        ia, ib, alpha0, dtn = w.bracket(k)
        a, b = w.snaps[ia], w.snaps[ib]
        vel = a if alpha0 == 0.0 else LazyLerpField(a, b, alpha0)
        out = O.step(so, vel, w.mesh, w.dt, 1.0, "rk2", vel_next=b, dt_to_next=dtn, w_interp="barycentric",
                     diffusion=DiffusionStepArgs("uniform", 10.0, 10.0, 0, 0, k), view=view)
        so = so.replace(lon=out["lon"], lat=out["lat"], z=out["z"], status=out["status"],
                        nearest_node=out["nearest_node"], failure_reason=out["failure_reason"],
                        u=out["u"], v=out["v"], w=out["w"])
    got = ctx.download_particles()
    assert ctx.device_errors() == 0
    from kelp_b200.particles import ParticleState
    st = ParticleState(lon=got["lon"], lat=got["lat"], z=got["z"], status=got["status"],
                       nearest_node=got["nearest_node"], failure_reason=got["failure_reason"], u=got["u"],
                       v=got["v"], w=got["w"])
    want = {f"f_{k}": getattr(so, k) for k in ("lon", "lat", "z", "status", "nearest_node", "failure_reason",
                                               "u", "v", "w")}
    assert_close_state(st, want, "f_", "resident loop with re-sort")
    ctx.close()


def test_cuda_vs_oracle_healpix_3d_kick():
    """A C3-shaped run on a reduced HEALPix dual mesh (nside 32: quads, the 8
    valence-3 triangles and the pole cells), 69 levels, W barycentric, the split
    uniform kick, 12 steps of 6 h: CUDA against the oracle."""
    from oracle import oracle as O
    from kelp_b200 import workloads as W
    from kelp_b200.particles import make_state
    from kelp_b200.fields import LazyLerpField
    w = W.c3(P=20000, nside=32)
    st = make_state(w.lon, w.lat, w.z).replace(failure_reason=np.zeros(w.P, np.int8))
    so = st
    view = O.MeshView(w.mesh)
    for k in range(12):
        ia, ib, alpha0, dtn = w.bracket(k)
        a, b = w.snaps[ia], w.snaps[ib]
        vel = a if alpha0 == 0.0 else LazyLerpField(a, b, alpha0)
        diff = DiffusionStepArgs("uniform", 10.0, 10.0, 0, 0, k)
        st = KI.rk2_step(st, vel, w.mesh, w.dt, 1.0, uv_interp="barycentric", w_interp="barycentric",
                         vel_next=b, dt_to_next=dtn, diffusion=diff)
        out = O.step(so, vel, w.mesh, w.dt, 1.0, "rk2", vel_next=b, dt_to_next=dtn, w_interp="barycentric",
                     diffusion=diff, view=view)
        so = so.replace(lon=out["lon"], lat=out["lat"], z=out["z"], status=out["status"],
                        nearest_node=out["nearest_node"], failure_reason=out["failure_reason"],
                        u=out["u"], v=out["v"], w=out["w"])
    want = {f"f_{k}": getattr(so, k) for k in ("lon", "lat", "z", "status", "nearest_node", "failure_reason",
                                               "u", "v", "w")}
    assert_close_state(st, want, "f_", "healpix 3-D rk2 + kick")
    assert (st.status == 1).sum() > 0.5 * w.P


@pytest.mark.parametrize("fixture", ["golden_band", "golden_3d"])
def test_cuda_walk_batch_matches_oracle(golden, fixture):
    """find_containing_elements_walk on the device against the oracle: from
    the true element, from a distant start (walks many edges or gives up and
    falls back), and with no start; points inside, outside and on the mesh
    boundary."""
    from oracle import oracle as O
    from kelp_b200.device import default_context
    g = golden(fixture)
    m = g.mesh
    rng = np.random.default_rng(11)
    lon0, lat0 = np.asarray(m.nodes_lon), np.asarray(m.nodes_lat)
    n = 4000
    lon = rng.uniform(lon0.min() - 1.0, lon0.max() + 1.0, n)
    lat = rng.uniform(lat0.min() - 1.0, lat0.max() + 1.0, n)
    E = np.asarray(m.elem_nodes).shape[0]
    ctx = default_context()
    ctx.ensure_elem_neighbors(m)
    nn = O.find_nearest(m, lon, lat)
    truth = O.contain(m, lon, lat, nn)
    np.testing.assert_array_equal(ctx.find_elements(lon, lat), truth)
    np.testing.assert_array_equal(ctx.find_elements(lon, lat, nn), truth)
    for start in (truth, rng.integers(0, E, n).astype(np.int32), np.full(n, -1, np.int32),
                  np.where(rng.random(n) < 0.5, E + 5, -7).astype(np.int32)):
        want = O.walk(m, lon, lat, start, nn)
        got = ctx.find_elements_walk(lon, lat, start)
        np.testing.assert_array_equal(got, want)


def test_cuda_walk_resident_sort_and_elem_roundtrip(golden):
    """Carried elements through the resident path: set, re-sort, step, read
    back in upload order; equal to the host-buffer step of the same state."""
    from kelp_b200.device import default_context
    g = golden("golden_band")
    c = g.case("rk2_walk")
    dt, T, n_steps, td, *_ = c["params"]
    st = g.particles().replace(elem=c["elem0"].copy())
    vel, vnext, dtn = g.payload(c["schedule"][0], T)
    ref = KI.rk2_step(st, vel, g.mesh, dt, td, uv_interp="barycentric", vel_next=vnext, dt_to_next=dtn)
    ctx = default_context()
    a, _ = KI.prepare_step(vel, g.mesh, dt, td, "rk2", dict(uv_interp="barycentric", vel_next=vnext,
                                                           dt_to_next=dtn), ctx, elem=st.elem)
    ctx.upload_particles(st.lon, st.lat, st.z, st.status, st.nearest_node, st.failure_reason)
    ctx.set_elem(st.elem)
    np.testing.assert_array_equal(ctx.get_elem(), st.elem)
    ctx.sort()
    ctx.step(a)
    out = ctx.download_particles()
    np.testing.assert_array_equal(ctx.get_elem(), ref.elem)
    np.testing.assert_array_equal(out["status"], ref.status)
    np.testing.assert_array_equal(out["lon"], ref.lon)
    np.testing.assert_array_equal(out["lat"], ref.lat)
