"""The batching entry points against the plain per-step calls, bit for bit.

* kc_run_fused (n steps in one launch, optionally with the beaching hook after
  each, optionally as a replayed CUDA graph) equals n kc_step (+ kc_beach)
  calls, across a re-sort between fused calls.
* Per-particle realization ids let several ensemble members share one array:
  the result equals separate runs with kc_step_args.real_id.
* kc_step_range on consecutive ranges equals one kc_step.
"""
import numpy as np
import pytest

from kelp_b200 import _native as N

pytestmark = pytest.mark.gpu

FIELDS = ("lon", "lat", "z", "status", "nearest_node", "failure_reason", "u", "v", "w")


def _workload(P=20000):
    from kelp_b200 import workloads as W
    return W.c3(P=P, nside=32)


def _beach_args(k):
    b = N.BeachArgs()
    b.use_depth, b.use_coastal, b.use_stochastic, b.on_failure = 1, 1, 1, 1
    b.resuspension, b.min_wet_steps = 3, 2
    b.depth_min, b.zone_depth, b.rewet_hysteresis = 400.0, 900.0, 150.0
    b.p_beach, b.p_resusp = 0.2, 0.3
    b.seed, b.real_id, b.step_i, b.pid_offset = 5, 0, k, 0
    return b


def _start(ctx, w, beach):
    from kelp_b200.mesh import build_boundary_info
    P = w.P
    ctx.upload_particles(w.lon, w.lat, w.z, np.ones(P, np.int32), np.full(P, -1, np.int32), np.zeros(P, np.int8))
    if beach:
        build_boundary_info(w.mesh)
        ctx.ensure_coastal(w.mesh, w.mesh._elem_is_coastal)
        ctx.beach_state_upload()


@pytest.mark.parametrize("graph", [False, True])
@pytest.mark.parametrize("beach", [False, True])
def test_fused_equals_sequential(graph, beach):
    from kelp_b200.device import DeviceContext
    w = _workload()
    ctx = DeviceContext(0)
    ctx.ensure_mesh(w.mesh)
    slots = ctx.slots_for(w.snaps)
    args = [w.step_args(k, slots) for k in range(12)]
    bargs = [_beach_args(k) for k in range(12)] if beach else None

    _start(ctx, w, beach)
    for k in range(12):
        if k == 6:
            ctx.sort()
        ctx.step(args[k])
        if beach:
            ctx.beach(bargs[k])
    ref = ctx.download_particles()
    ref_wet = ctx.beach_state_download() if beach else None
    assert ctx.device_errors() == 0

    _start(ctx, w, beach)
    ctx.run_fused(args[:6], None if bargs is None else bargs[:6], graph=graph)
    ctx.sort()
    ctx.run_fused(args[6:], None if bargs is None else bargs[6:], graph=graph)   # a replay when graph
    got = ctx.download_particles()
    assert ctx.device_errors() == 0
    for n in FIELDS:
        np.testing.assert_array_equal(got[n], ref[n], err_msg=f"{n} graph={graph} beach={beach}")
    if beach:
        np.testing.assert_array_equal(ctx.beach_state_download(), ref_wet)
        assert (ref["status"] == 2).any(), "the case should beach some particles"
    ctx.close()


def test_realizations_share_one_array():
    from kelp_b200.device import DeviceContext
    w = _workload(6000)
    P, members = w.P, 3
    ctx = DeviceContext(0)
    ctx.ensure_mesh(w.mesh)
    slots = ctx.slots_for(w.snaps)
    sep = []
    for r in range(members):
        ctx.upload_particles(w.lon, w.lat, w.z, np.ones(P, np.int32), np.full(P, -1, np.int32),
                             np.zeros(P, np.int8))
        for k in range(6):
            a = w.step_args(k, slots)
            a.real_id = r
            ctx.step(a)
        sep.append(ctx.download_particles())
    rep = lambda x: np.concatenate([x] * members)
    ctx.upload_particles(rep(w.lon), rep(w.lat), rep(w.z), np.ones(P * members, np.int32),
                         np.full(P * members, -1, np.int32), np.zeros(P * members, np.int8),
                         rep(np.arange(P, dtype=np.int64)))
    ctx.set_realization(np.repeat(np.arange(members, dtype=np.int32), P))
    ctx.sort()
    steps = []
    for k in range(6):
        a = w.step_args(k, slots)
        a.real_id = 99   # ignored: every particle carries its own
        steps.append(a)
    ctx.run_fused(steps, graph=True)
    got = ctx.download_particles()
    for n in FIELDS:
        np.testing.assert_array_equal(got[n], np.concatenate([s[n] for s in sep]), err_msg=n)
    ctx.close()


def test_step_range_equals_step():
    from kelp_b200.device import DeviceContext
    w = _workload(9000)
    P = w.P
    ctx = DeviceContext(0)
    ctx.ensure_mesh(w.mesh)
    slots = ctx.slots_for(w.snaps)
    a = w.step_args(0, slots)
    a.pid_offset = 123
    ctx.upload_particles(w.lon, w.lat, w.z, np.ones(P, np.int32), np.full(P, -1, np.int32), np.zeros(P, np.int8))
    ctx.step(a)
    ref = ctx.download_particles()
    ctx.upload_particles(w.lon, w.lat, w.z, np.ones(P, np.int32), np.full(P, -1, np.int32), np.zeros(P, np.int8))
    for b, e in ((0, 1000), (1000, 4321), (4321, P)):
        ctx.step_range(a, b, e - b)
    got = ctx.download_particles()
    for n in FIELDS:
        np.testing.assert_array_equal(got[n], ref[n], err_msg=n)
    with pytest.raises(N.KcError):
        ctx.step_range(a, P - 10, 20)
    ctx.close()


def test_autotune_picks_a_candidate_and_results_do_not_depend_on_it(tmp_path, monkeypatch):
    from kelp_b200 import autotune
    from kelp_b200.device import DeviceContext
    monkeypatch.setenv("KELP_B200_TUNE_CACHE", str(tmp_path / "tune.json"))
    w = _workload(8000)
    P = w.P
    ctx = DeviceContext(0)
    ctx.ensure_mesh(w.mesh)
    slots = ctx.slots_for(w.snaps)

    def reset():
        ctx.upload_particles(w.lon, w.lat, w.z, np.ones(P, np.int32), np.full(P, -1, np.int32),
                             np.zeros(P, np.int8))

    def make_steps(k, n):
        return [w.step_args(kk, slots) for kk in range(k, k + n)]

    key = autotune.mesh_signature(w.mesh, 3, "rk2", "plain", P)
    t = autotune.tune(ctx, key, reset, make_steps, 0, window=4, blocks=(128, 256), steps_per_launch=(1, 2),
                      sort_every=(2, 4))
    assert t["block"] in (128, 256) and t["steps_per_launch"] in (1, 2) and t["sort_every"] in (2, 4)
    assert len(t["trials"]) == 8 and not t["cached"]
    again = autotune.tune(ctx, key, reset, make_steps, 0, window=4)
    assert again["cached"] and again["block"] == t["block"]
    outs = []
    for blk, spl, se in ((128, 1, 2), (256, 2, 4)):
        ctx.set_fused_block(blk)
        reset()
        autotune.run_window(ctx, make_steps, 0, 8, spl, se)
        outs.append(ctx.download_particles())
    for n in FIELDS:
        np.testing.assert_array_equal(outs[0][n], outs[1][n], err_msg=n)
    ctx.close()


def test_fused_refuses_per_step_beaching_surfaces():
    """A beaching surface (kc_beach_surface) belongs to one step: a fused
    launch over several steps refuses the hook while one is set, and runs
    again once it is cleared."""
    from kelp_b200.device import DeviceContext
    w = _workload(4000)
    ctx = DeviceContext(0)
    ctx.ensure_mesh(w.mesh)
    slots = ctx.slots_for(w.snaps)
    args = [w.step_args(k, slots) for k in range(4)]
    _start(ctx, w, True)
    ctx.beach_surface(np.zeros(np.asarray(w.mesh.nodes_lon).size))
    with pytest.raises(N.KcError, match="per step"):
        ctx.run_fused(args, beach=[_beach_args(k) for k in range(4)])
    ctx.beach_surface(None, None)
    ctx.run_fused(args, beach=[_beach_args(k) for k in range(4)])
    ctx.synchronize()
    assert ctx.device_errors() == 0
    ctx.close()
