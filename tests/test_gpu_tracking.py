"""The device-resident tracking loop (kelp_b200.tracking) against the
reference's recorded run and against the per-call API.

The beaching golden was recorded by running the reference's own step and
beaching hook in the order of its tracking loop; the Tracker, which keeps the
particles on the GPU, re-sorts them and carries their anchors between steps,
must end where that run ends (integers bit-exact, positions within the step
kernels' tolerance).  Several realizations in one array must equal separate
runs bit for bit, and run_tracking with KELP's configuration schema must equal
the Tracker it builds.
"""
import numpy as np
import pytest

from kelp_b200 import tracking as T
from kelp_b200.beaching import BeachingConfig

from test_oracle_golden import beach_kwargs

pytestmark = pytest.mark.gpu

POS_TOL_DEG = 1e-9 / 0.017453292519943295


class Diff:
    enabled = True
    scheme = "uniform"
    composition = "split"
    az_enabled = False

    def __init__(self, kh, seed):
        self.kh_zonal = self.kh_meridional = kh
        self.seed = seed


def _tracker(g, c, sort_every=5):
    kw = beach_kwargs(c)
    dt, Tsnap, n_steps, td, khx, khy, seed, real_id, pid_off = c["params"]
    cfg = BeachingConfig(enabled=True, criteria=kw["criteria"], depth_min=kw["depth_min"],
                         zone_depth=kw["zone_depth"], t_beach=kw["t_beach"] or None,
                         resuspension=kw["resuspension"], rewet_hysteresis=kw["rewet_hysteresis"],
                         min_wet_steps=kw["min_wet_steps"], t_resuspend=kw["t_resuspend"] or None, seed=kw["seed"])
    ft = np.arange(len(g.snaps)) * Tsnap
    diff = Diff(khx, int(seed)) if khx >= 0 else None
    return T.Tracker(g.mesh, g.snaps, ft, integrator="rk2", dt=dt, diffusion=diff, beaching=cfg,
                     sort_every=sort_every), int(n_steps)


def test_tracker_reproduces_the_reference_run(golden):
    g = golden("golden_beach")
    c = g.case("dco_auto")
    tr, n = _tracker(g, c)
    res = tr.run(g.particles(), n, output_freq=4)
    fin = res.final[0]
    for name in ("status", "nearest_node", "failure_reason"):
        np.testing.assert_array_equal(getattr(fin, name), c[f"s{n}_{name}"], err_msg=name)
    np.testing.assert_array_equal(res.wet_streak[0], c[f"s{n}_wet"])
    for name in ("lon", "lat"):
        np.testing.assert_allclose(getattr(fin, name), c[f"s{n}_{name}"], rtol=0, atol=POS_TOL_DEG, err_msg=name)
    rec = res.records[0]
    assert len(rec.times) == n // 4 and rec.times[-1] == n * c["params"][0]
    # the record after step 8 is the reference's state after step 8 (dormant
    # particles are recorded as NaN positions, output format 2)
    np.testing.assert_array_equal(rec.status[1], c["s8_status"])
    want = np.where(c["s8_status"] == 4, np.nan, c["s8_lon"])
    np.testing.assert_allclose(rec.lons[1], want, rtol=0, atol=POS_TOL_DEG, equal_nan=True)


def test_realizations_in_one_array_equal_separate_runs(golden):
    g = golden("golden_beach")
    c = g.case("sto_both")
    tr, n = _tracker(g, c)
    st = g.particles()
    together = tr.run_realizations(st, n, realizations=(0, 1, 2), output_freq=8)
    for r in range(3):
        alone = tr.run(st, n, realization_id=r, output_freq=8)
        for name in ("lon", "lat", "status", "nearest_node", "failure_reason"):
            np.testing.assert_array_equal(getattr(together.final[r], name), getattr(alone.final[0], name),
                                          err_msg=f"realization {r} {name}")
        np.testing.assert_array_equal(together.wet_streak[r], alone.wet_streak[0])
        np.testing.assert_array_equal(np.stack(together.records[r].lons), np.stack(alone.records[0].lons))
    # the members differ: their draws are their own
    assert not np.array_equal(together.final[0].lon, together.final[1].lon)


def test_run_tracking_config_equals_tracker(golden, tmp_path):
    g = golden("golden_beach")
    c = g.case("cd_sresusp")
    dt, Tsnap, n_steps, td, khx, khy, seed, real_id, pid_off = c["params"]
    kw = beach_kwargs(c)
    m = g.mesh
    np.savez(tmp_path / "mesh.npz", nodes_lon=m.nodes_lon, nodes_lat=m.nodes_lat, depth=m.depth,
             elem_nodes=m.elem_nodes)
    np.savez(tmp_path / "vel.npz", times=np.arange(len(g.snaps)) * Tsnap,
             u=np.stack([np.asarray(s.u) for s in g.snaps]), v=np.stack([np.asarray(s.v) for s in g.snaps]))
    st = g.particles()
    np.savez(tmp_path / "seeds.npz", lon=st.lon, lat=st.lat)
    cfg = {"mode": {"time_dir": 1.0},
           "numerics": {"backend": "cuda", "integrator": "rk2", "dt": float(dt), "output_freq": 4,
                        "uv_interp": "barycentric", "temporal_interp": True,
                        "diffusion": {"enabled": True, "scheme": "uniform", "kh_zonal": float(khx),
                                      "kh_meridional": float(khy), "seed": int(seed)},
                        "beaching": {"enabled": True, "criteria": kw["criteria"], "depth_min": kw["depth_min"],
                                     "resuspension": kw["resuspension"], "t_resuspend": kw["t_resuspend"],
                                     "rewet_hysteresis": kw["rewet_hysteresis"]}},
           "time": {"start_time_idx": 0, "n_steps": int(n_steps), "num_runs": 2},
           "data": {"mesh_npz": str(tmp_path / "mesh.npz"), "velocity_npz": str(tmp_path / "vel.npz"),
                    "seeds": str(tmp_path / "seeds.npz")}}
    recs = T.run_tracking(cfg)
    assert len(recs) == 2
    # the same run through a Tracker on the golden's own mesh object
    diff = Diff(khx, int(seed))
    bcfg = BeachingConfig(enabled=True, criteria=kw["criteria"], depth_min=kw["depth_min"],
                          resuspension=kw["resuspension"], t_resuspend=kw["t_resuspend"],
                          rewet_hysteresis=kw["rewet_hysteresis"])
    tr = T.Tracker(g.mesh, g.snaps, np.arange(len(g.snaps)) * Tsnap, integrator="rk2", dt=dt, diffusion=diff,
                   beaching=bcfg)
    alive = st.replace(status=np.ones(st.n_particles, np.int32))   # the seed file carries positions only
    for r in range(2):
        res = tr.run(alive, int(n_steps), realization_id=r, output_freq=4)
        np.testing.assert_array_equal(np.stack(recs[r].status), np.stack(res.records[0].status))
        np.testing.assert_array_equal(np.stack(recs[r].lons), np.stack(res.records[0].lons))


def test_tracker_walk_equals_per_call_walk(golden):
    """elem_search "walk" in the resident loop (seeded by the local search at
    the start, carried through re-sorts) equals stepping the same state
    through the per-call rk2_step with state.elem."""
    from kelp_b200 import integrators as KI
    g = golden("golden_band")
    c = g.case("rk2_walk")
    dt, Tsnap, n_steps, td, *_ = c["params"]
    ft = np.arange(len(g.snaps)) * Tsnap
    n = 6
    tr = T.Tracker(g.mesh, g.snaps, ft, integrator="rk2", dt=dt, sort_every=2, elem_search="walk")
    st0 = g.particles()
    res = tr.run(st0, n)
    fin = res.final[0]
    # the start seed: the local search around the exact anchor (tracking.py:2243-2249)
    np.testing.assert_array_equal(tr.ctx.find_elements(st0.lon, st0.lat), c["elem0"])
    st = st0.replace(elem=c["elem0"].copy())
    t = float(ft[0])
    for k in range(n):
        br = T.resolve_time_bracket(t, ft, "stop", 1, T.snapshot_band(dt))
        vel, vnext, dtn = T.vel_payload(br, g.snaps, 1)
        st = KI.rk2_step(st, vel, g.mesh, dt, 1.0, uv_interp="barycentric", vel_next=vnext, dt_to_next=dtn)
        t += dtn if (dtn is not None and abs(dt - dtn) <= T.snapshot_band(dt)) else dt
    for name in ("status", "nearest_node", "failure_reason", "elem", "lon", "lat"):
        np.testing.assert_array_equal(getattr(fin, name), getattr(st, name), err_msg=name)


def test_tracker_az_kick_equals_per_call(golden):
    """The vertical Az kick (field Az from the snapshots) inside the resident
    loop equals the per-call rk2_step with the DiffusionStepArgs the reference's
    loop builds (tracking.py:2595-2611)."""
    from kelp_b200 import integrators as KI
    from kelp_b200.diffusion import DiffusionStepArgs
    g = golden("golden_3d")
    c = g.case("rk2_wbary_kick_azf")
    dt, Tsnap, n_steps, td, khx, khy, seed, real_id, pid_off = c["params"]
    ft = np.arange(len(g.snaps)) * Tsnap
    n = 5
    d = Diff(khx, int(seed))
    d.az_enabled, d.az_const, d.var_az = True, 0.0, "az"
    tr = T.Tracker(g.mesh, g.snaps, ft, integrator="rk2", dt=dt, w_interp="barycentric", diffusion=d,
                   sort_every=2)
    st0 = g.particles()
    fin = tr.run(st0, n, realization_id=3).final[0]
    st = st0
    t = float(ft[0])
    band = T.snapshot_band(dt)
    for k in range(n):
        vel, vnext, dtn = T.vel_payload(T.resolve_time_bracket(t, ft, "stop", 1, band), g.snaps, 1)
        diff = DiffusionStepArgs("uniform", khx, khy, int(seed), 3, k, az_enabled=True, az_requires_field=True)
        st = KI.rk2_step(st, vel, g.mesh, dt, 1.0, uv_interp="barycentric", w_interp="barycentric",
                         vel_next=vnext, dt_to_next=dtn, diffusion=diff)
        t += dtn if (dtn is not None and abs(dt - dtn) <= band) else dt
    for name in ("status", "nearest_node", "failure_reason", "lon", "lat", "z"):
        np.testing.assert_array_equal(getattr(fin, name), getattr(st, name), err_msg=name)
    assert np.any(fin.z != st0.z)


def test_tracker_pchip_equals_per_call(golden):
    """temporal_reconstruction "pchip" in the resident loop: the RK stages take
    the 4-record stencil where one exists (linear at the first and last
    interval), bit-identical to the per-call rk4_step with the same bundles."""
    from kelp_b200 import integrators as KI
    g = golden("golden_pchip2d")
    dt = 21600.0
    ft = np.arange(len(g.snaps)) * 86400.0
    n = 18
    tr = T.Tracker(g.mesh, g.snaps, ft, integrator="rk4", dt=dt, sort_every=3, temporal_reconstruction="pchip")
    st0 = g.particles()
    fin = tr.run(st0, n).final[0]
    st = st0
    t = float(ft[0])
    band = T.snapshot_band(dt)
    used = 0
    for k in range(n):
        br = T.resolve_time_bracket(t, ft, "stop", 1, band)
        vel, vnext, dtn = T.vel_payload(br, g.snaps, 1)
        sten = T.resolve_recon_stencil(br, ft.size)
        kw = {}
        if sten is not None:
            kw["recon"] = ([g.snaps[i] for i in sten[0]], [float(ft[i]) for i in sten[0]], sten[1], 1.0)
            used += 1
        step_len, t_end = dt, None
        if dtn is not None and abs(dt - dtn) <= band:
            step_len, t_end = dtn, T.step_end_on_record(t, br[4], dtn, 1, ft, "stop")
        st = KI.rk4_step(st, vel, g.mesh, step_len, 1.0, uv_interp="barycentric", vel_next=vnext,
                         dt_to_next=dtn, **kw)
        t = t_end if t_end is not None else t + dt
    assert 0 < used < n
    for name in ("status", "nearest_node", "failure_reason", "lon", "lat"):
        np.testing.assert_array_equal(getattr(fin, name), getattr(st, name), err_msg=name)


def test_checkpoint_restart_is_bit_identical(golden, tmp_path):
    """A run stopped at a checkpoint and resumed from it (state, global step,
    wet streaks, release steps, carried elements) ends bit-identical to the
    uninterrupted run; the trajectory store holds every record (format 2:
    NaN velocities where a particle was not alive through the step)."""
    from kelp_b200.writers import TrajectoryWriter, load_restart, read_trajectory
    g = golden("golden_beach")
    c = g.case("sto_both")
    tr, n = _tracker(g, c)
    st0 = g.particles()
    full = tr.run(st0, n, output_freq=2)
    half = n // 2
    w = TrajectoryWriter(str(tmp_path / "run"), st0.n_particles).open()
    tr.run(st0, half, output_freq=2, writer=w, checkpoint_freq=half)
    rst = load_restart(str(tmp_path / "run"))
    assert rst["step_i"] == half - 1
    dt = float(c["params"][0])
    rest = tr.run(rst["state"], n - half, start_time=half * dt, start_step_i=rst["step_i"] + 1, output_freq=2,
                  start_wet_streak=rst["wet_streak"])
    for name in ("lon", "lat", "status", "nearest_node", "failure_reason"):
        np.testing.assert_array_equal(getattr(rest.final[0], name), getattr(full.final[0], name), err_msg=name)
    np.testing.assert_array_equal(rest.wet_streak[0], full.wet_streak[0])
    traj = read_trajectory(str(tmp_path / "run"))
    assert traj["lon"].shape == (half // 2, st0.n_particles)
    np.testing.assert_array_equal(traj["lon"], np.stack(full.records[0].lons[: half // 2]))
    dead = traj["status"] != 1
    assert np.all(np.isnan(traj["vel_u"][dead]))


@pytest.mark.parametrize("recon", ["linear", "pchip"])
def test_prefetched_records_give_the_same_run(golden, recon):
    """The next step's records uploaded beside the running step
    (kc_field_upload_async, through the ring's eviction with more records
    than slots) give the run of uploads made before each step, bit for bit."""
    from kelp_b200.fields import VelocityField
    from kelp_b200.device import DeviceContext
    g = golden("golden_band")
    recs = [VelocityField(u=np.asarray(s.u) * (1.0 + 0.1 * k), v=np.asarray(s.v) * (1.0 - 0.05 * k), w=None,
                          eta=np.zeros(np.asarray(s.u).shape[-1]), uv_layout="node")
            for k in range(3) for s in g.snaps]           # 12 records, more than the 8 ring slots
    ft = np.arange(len(recs)) * 86400.0
    diff = Diff(5.0e4, 9)
    out = {}
    for pf in (False, True):
        ctx = DeviceContext(0)
        try:
            tr = T.Tracker(g.mesh, recs, ft, integrator="rk4", dt=21600.0, diffusion=diff, sort_every=5,
                           temporal_reconstruction=recon, prefetch=pf, ctx=ctx)
            res = tr.run(g.particles(), 40, output_freq=4)
            out[pf] = (res.final[0], res.records[0])
        finally:
            ctx.close()
    (fa, ra), (fb, rb) = out[False], out[True]
    for name in ("status", "nearest_node", "failure_reason", "lon", "lat", "u", "v"):
        np.testing.assert_array_equal(getattr(fa, name), getattr(fb, name), err_msg=name)
    assert len(ra.times) == len(rb.times) == 10
    np.testing.assert_array_equal(ra.times, rb.times)
    for name in ("lons", "lats", "us", "vs", "status", "failure_reason"):
        for a, b in zip(getattr(ra, name), getattr(rb, name)):
            np.testing.assert_array_equal(a, b, err_msg=name)
