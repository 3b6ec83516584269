"""kc_step_host (chunked upload / step / download on three streams) returns
exactly what the resident path (kc_particles_upload + kc_step +
kc_particles_download) returns, for any chunk size: each chunk keeps its
particles' global RNG keys."""
import numpy as np
import pytest

from kelp_b200 import _native as N

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("chunk", [0, 1000, 4096, 10 ** 9])
def test_host_step_matches_resident_step(chunk):
    from kelp_b200 import workloads as W
    from kelp_b200.device import DeviceContext, pinned_empty
    w = W.c3(P=20000, nside=32)
    ctx = DeviceContext(0)
    ctx.ensure_mesh(w.mesh)
    slots = ctx.slots_for(w.snaps)
    P = w.P
    st = {"lon": w.lon.copy(), "lat": w.lat.copy(), "z": w.z.copy(), "status": np.ones(P, np.int32),
          "nearest_node": np.full(P, -1, np.int32), "failure_reason": np.zeros(P, np.int8)}
    res = dict(st)
    for k in range(4):
        a = w.step_args(k, slots)
        a.pid_offset = 777
        # resident path
        ctx.upload_particles(res["lon"], res["lat"], res["z"], res["status"], res["nearest_node"],
                             res["failure_reason"], np.arange(P, dtype=np.int64) + 777 - 777)
        ctx.step(a)
        got = ctx.download_particles()
        res = {n: got[n] for n in ("lon", "lat", "z", "status", "nearest_node", "failure_reason")}
        res_uvw = (got["u"], got["v"], got["w"])
        # host path, page-locked output
        out = {n: pinned_empty((P,), v.dtype) for n, v in st.items()}
        for n in ("u", "v", "w"):
            out[n] = pinned_empty((P,), np.float64)
        ctx.step_host(a, st, out, chunk=chunk)
        st = {n: np.array(out[n]) for n in st}
        for n in st:
            np.testing.assert_array_equal(st[n], res[n], err_msg=f"step {k} {n} chunk {chunk}")
        for n, r in zip(("u", "v", "w"), res_uvw):
            np.testing.assert_array_equal(out[n], r, err_msg=f"step {k} {n} chunk {chunk}")
    assert ctx.device_errors() == 0
    ctx.close()


def test_host_step_with_ids_and_release_matches_resident():
    """Particle keys, per-particle realizations and delayed release through
    the host-buffer step equal the resident path's."""
    from kelp_b200 import workloads as W
    from kelp_b200.device import DeviceContext
    w = W.c3(P=12000, nside=32)
    ctx = DeviceContext(0)
    ctx.ensure_mesh(w.mesh)
    slots = ctx.slots_for(w.snaps)
    P = w.P
    rng = np.random.default_rng(1)
    pid = rng.permutation(P).astype(np.int64)
    rid = rng.integers(0, 4, P).astype(np.int32)
    rs = rng.integers(0, 6, P).astype(np.int32)
    st0 = {"lon": w.lon.copy(), "lat": w.lat.copy(), "z": w.z.copy(), "status": np.full(P, 4, np.int32),
           "nearest_node": np.full(P, -1, np.int32), "failure_reason": np.zeros(P, np.int8)}
    res = dict(st0)
    st = dict(st0)
    for k in range(5):
        a = w.step_args(k, slots)
        a.global_step = k
        ctx.upload_particles(res["lon"], res["lat"], res["z"], res["status"], res["nearest_node"],
                             res["failure_reason"], pid, rs)
        ctx.set_realization(rid)
        ctx.step(a)
        got = ctx.download_particles()
        res = {n: got[n] for n in st0}
        out = {n: np.empty_like(v) for n, v in st0.items()}
        ctx.step_host(a, dict(st, pid=pid, real_id=rid, release_step=rs), out, chunk=2048)
        st = out
        for n in st0:
            np.testing.assert_array_equal(st[n], res[n], err_msg=f"step {k} {n}")
    assert (res["status"] == 1).any() and (rs > 0).any()
    assert ctx.device_errors() == 0
    ctx.close()
