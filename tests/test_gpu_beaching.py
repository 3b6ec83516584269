"""Beaching on the GPU against the reference's recorded runs.

Each golden case runs RK2 (+ split kick) steps, each followed by the beaching
hook.  Statuses, anchors, failure reasons and wet-step counters must match the
reference bit for bit; positions within the step kernels' tolerance (the
device's trig differs from the C library's in the last bits).  Two routes:
the public per-call API (``integrators.rk2_step`` +
``beaching.apply_beaching_hook``, host arrays in and out every step) and the
device-resident loop (``kc_step`` + ``kc_beach`` with periodic re-sorts).
Two of the cases read the payload's free surface (``use_eta``) and dry mask
(``dry_mask_var``), which move between the records.
"""
import numpy as np
import pytest

from kelp_b200 import beaching as KB
from kelp_b200 import integrators as KI
from kelp_b200.diffusion import DiffusionStepArgs

from test_oracle_golden import BEACH_CASES, beach_kwargs

pytestmark = pytest.mark.gpu

POS_TOL_DEG = 1e-9 / 0.017453292519943295


def _run_cfg(g, c):
    kw = beach_kwargs(c)
    _, _, _, _, _, _, seed, real_id, pid_off = c["params"]
    cfg = KB.BeachingConfig(enabled=True, criteria=kw["criteria"], depth_min=kw["depth_min"],
                            zone_depth=kw["zone_depth"], t_beach=kw["t_beach"] or None,
                            resuspension=kw["resuspension"], rewet_hysteresis=kw["rewet_hysteresis"],
                            min_wet_steps=kw["min_wet_steps"], t_resuspend=kw["t_resuspend"] or None,
                            seed=kw["seed"], use_eta=kw["use_eta"], dry_mask_var=kw["dry_mask_var"])
    return KB.make_run_config(cfg, g.mesh, diffusion_seed=int(seed), particle_offset=int(pid_off))


def _check(got, c, k, cname, route):
    for name in ("status", "nearest_node", "failure_reason", "wet"):
        np.testing.assert_array_equal(got[name], c[f"s{k}_{name}"], err_msg=f"{route} {cname} step {k} {name}")
    for name in ("lon", "lat"):
        np.testing.assert_allclose(got[name], c[f"s{k}_{name}"], rtol=0, atol=POS_TOL_DEG,
                                   err_msg=f"{route} {cname} step {k} {name}")


@pytest.mark.parametrize("cname", BEACH_CASES)
def test_cuda_beaching_public_api(golden, cname):
    g = golden("golden_beach")
    c = g.case(cname)
    dt, T, n_steps, td, khx, khy, seed, real_id, pid_off = c["params"]
    run_cfg = _run_cfg(g, c)
    st = g.particles()
    wet = None
    seen = 0
    for k in range(int(n_steps)):
        vel, vnext, dtn = g.payload(c["schedule"][k], T)
        kw = dict(uv_interp="barycentric", vel_next=vnext, dt_to_next=dtn)
        if khx >= 0:
            kw["diffusion"] = DiffusionStepArgs("uniform", khx, khy, int(seed), int(real_id), k,
                                                pid_offset=int(pid_off))
        prev = st.status
        st = KI.rk2_step(st, vel, g.mesh, dt, td, **kw)
        st, wet = KB.apply_beaching_hook(st, prev, g.mesh, vel, run_cfg, wet, int(real_id), k, dt)
        if f"s{k + 1}_status" in c:
            _check({"status": st.status, "nearest_node": st.nearest_node, "failure_reason": st.failure_reason,
                    "wet": wet, "lon": st.lon, "lat": st.lat}, c, k + 1, cname, "public API")
            seen += 1
    assert seen >= 2


@pytest.mark.parametrize("cname", BEACH_CASES)
def test_cuda_beaching_resident_loop(golden, cname):
    """kc_step + kc_beach on resident particles, re-sorted every 5 steps; the
    step kernels record each particle's entry status for the hook."""
    from kelp_b200.device import DeviceContext
    g = golden("golden_beach")
    c = g.case(cname)
    dt, T, n_steps, td, khx, khy, seed, real_id, pid_off = c["params"]
    run_cfg = _run_cfg(g, c)
    ctx = DeviceContext(0)
    st = g.particles()
    P = st.n_particles
    ctx.upload_particles(st.lon, st.lat, st.z, st.status, st.nearest_node, fr=st.failure_reason)
    ctx.beach_state_upload()
    if run_cfg.need_topo:
        ctx.ensure_coastal(g.mesh, run_cfg.elem_coastal)
    for k in range(int(n_steps)):
        if k % 5 == 4:
            ctx.sort()
        vel, vnext, dtn = g.payload(c["schedule"][k], T)
        kw = dict(uv_interp="barycentric", vel_next=vnext, dt_to_next=dtn)
        kick = None
        if khx >= 0:
            kick = (khx, khy, int(seed), int(real_id), k, int(pid_off))
        a, _ = KI.prepare_step(vel, g.mesh, dt, td, "rk2", kw, ctx, kick=kick)
        ctx.step(a)
        ctx.beach_surface(*KB.payload_surfaces(vel, run_cfg.cfg))
        ctx.beach(KB.beach_args(run_cfg, int(real_id), k, dt))
        if f"s{k + 1}_status" in c:
            out = ctx.download_particles()
            out["wet"] = ctx.beach_state_download()
            assert out["status"].shape == (P,)
            _check(out, c, k + 1, cname, "resident")
    assert ctx.device_errors() == 0
    ctx.close()
