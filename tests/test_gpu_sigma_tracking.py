"""Sigma meshes in the device-resident loop (kelp_b200.tracking.Tracker).

The reference's loop hands every sigma step the free surface at the step's
start and end time from one function of time (src/kelp/tracking.py:2562-2596,
_eta_at_time :3097-3133).  The Tracker evaluates those surfaces on the device
from its resident records (kc_sigma_surface_slots); the per-call step
functions take them as sigma_eta_start / sigma_eta_end.  Here the Tracker's
run must equal, bit for bit, a per-call loop that hands each step the
reference's own surfaces (tests/golden/golden_eta_time.npz, recorded from
_eta_at_time), linear and PCHIP, forward and backward, on the sigma shelf of
golden_sigma_surf.
"""
import os

import numpy as np
import pytest

from conftest import GOLDEN
from kelp_b200 import tracking as T

pytestmark = pytest.mark.gpu

TSNAP = 21600.0
DT = 3600.0


def _surfaces(tag, mode):
    d = np.load(os.path.join(GOLDEN, "golden_eta_time.npz"))
    return d[f"{tag}_times"], d[f"{tag}_{mode}"], d["etas"]


@pytest.mark.parametrize("scheme,mode,direction", [("rk2", "linear", 1), ("rk4", "pchip", 1), ("euler", "linear", 1),
                                                   ("rk4", "linear", -1), ("rk2", "pchip", -1)])
def test_tracker_sigma_equals_per_call_with_reference_surfaces(golden, scheme, mode, direction):
    from kelp_b200 import integrators as KI
    g = golden("golden_sigma_surf")
    tag = "fwd" if direction > 0 else "bwd"
    times, surf, etas = _surfaces(tag, mode)
    for k, sn in enumerate(g.snaps):
        np.testing.assert_array_equal(np.asarray(sn.eta, dtype=np.float64), etas[k].astype(np.float64))
    ft = np.arange(len(g.snaps)) * TSNAP
    n = 20
    fn = KI.get_integrator(scheme)
    tr = T.Tracker(g.mesh, g.snaps, ft, integrator=scheme, dt=DT, time_dir=float(direction), w_interp="barycentric",
                   sort_every=7, temporal_reconstruction=mode)
    st0 = g.particles()
    fin = tr.run(st0, n, start_time=float(times[0])).final[0]
    st = st0
    band = T.snapshot_band(DT)
    for k in range(n):
        t = float(times[k])
        br = T.resolve_time_bracket(t, ft, "stop", direction, band)
        vel, vnext, dtn = T.vel_payload(br, g.snaps, direction)
        kw = {}
        if mode == "pchip" and scheme != "euler":
            sten = T.resolve_recon_stencil(br, ft.size)
            if sten is not None:
                kw["recon"] = ([g.snaps[i] for i in sten[0]], [float(ft[i]) for i in sten[0]], sten[1],
                               float(direction))
        assert np.all(np.isfinite(surf[k])) and np.all(np.isfinite(surf[k + 1]))
        st = fn(st, vel, g.mesh, DT, float(direction), uv_interp="barycentric", w_interp="barycentric",
                vel_next=vnext, dt_to_next=dtn, sigma_eta_start=surf[k], sigma_eta_end=surf[k + 1], **kw)
    moved = np.count_nonzero(st.lon != st0.lon)
    assert moved > 0.5 * st0.lon.size
    for name in ("status", "nearest_node", "failure_reason", "lon", "lat", "z"):
        np.testing.assert_array_equal(getattr(fin, name), getattr(st, name), err_msg=name)


def test_supplied_surfaces_change_the_step(golden):
    """A sigma step given surfaces other than the payload's own ends
    elsewhere in depth (the surfaces are read), and passing the payload's own
    surfaces changes nothing."""
    from kelp_b200 import integrators as KI
    g = golden("golden_sigma_surf")
    st0 = g.particles()
    a, b = g.snaps[0], g.snaps[1]
    base = KI.rk2_step(st0, a, g.mesh, DT, 1.0, uv_interp="barycentric", w_interp="barycentric", vel_next=b,
                       dt_to_next=TSNAP)
    own_end = (1.0 - DT / TSNAP) * np.asarray(a.eta, dtype=np.float64) + DT / TSNAP * np.asarray(b.eta,
                                                                                                dtype=np.float64)
    same = KI.rk2_step(st0, a, g.mesh, DT, 1.0, uv_interp="barycentric", w_interp="barycentric", vel_next=b,
                       dt_to_next=TSNAP, sigma_eta_start=np.asarray(a.eta, dtype=np.float64), sigma_eta_end=own_end)
    np.testing.assert_array_equal(base.z, same.z)
    other = KI.rk2_step(st0, a, g.mesh, DT, 1.0, uv_interp="barycentric", w_interp="barycentric", vel_next=b,
                        dt_to_next=TSNAP, sigma_eta_end=own_end + 0.5)
    assert np.count_nonzero(other.z != base.z) > 0.5 * st0.lon.size
    with pytest.raises(ValueError, match="supplied surface"):
        KI.rk2_step(st0, a, g.mesh, DT, 1.0, uv_interp="barycentric", w_interp="barycentric", vel_next=b,
                    dt_to_next=TSNAP, sigma_eta_start=own_end[:-1])
