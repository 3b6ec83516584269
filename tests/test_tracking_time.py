"""The tracking loop's time axis against the reference's bracket resolution
(tracking._resolve_time_bracket, recorded in tests/golden/golden_time.npz)."""
import os

import numpy as np

from kelp_b200.tracking import resolve_time_bracket, vel_payload

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "golden_time.npz")


def test_time_bracket_matches_reference():
    d = np.load(GOLDEN)
    axes = [d["axis_uniform"], d["axis_ragged"]]
    modes = ["stop", "cycle"]
    n_none = 0
    for row in d["rows"]:
        ai, mi, direction, snap, q = int(row[0]), int(row[1]), int(row[2]), float(row[3]), float(row[4])
        got = resolve_time_bracket(q, axes[ai], modes[mi], direction, snap)
        want = row[5:]
        if np.isnan(want[0]):
            assert got is None, (row, got)
            n_none += 1
            continue
        assert got is not None, row
        assert (got[0], got[1]) == (int(want[0]), int(want[1])), (row, got)
        np.testing.assert_array_equal(np.array(got[2:], dtype=np.float64), want[2:], err_msg=str(row))
    assert n_none > 0


def test_payload_directions():
    class F:
        def __init__(self, k):
            self.u = np.full(3, float(k))
            self.v = self.u
            self.w = None
            self.eta = np.zeros(3)
            self.uv_layout = "node"
            self.uv_vertical = "layer"
    fields = [F(k) for k in range(3)]
    ft = np.array([0.0, 100.0, 200.0])
    vel, vnext, dtn = vel_payload(resolve_time_bracket(25.0, ft), fields, 1)
    assert vel.alpha == 0.25 and vnext is fields[1] and dtn == 75.0
    vel, vnext, dtn = vel_payload(resolve_time_bracket(25.0, ft, direction=-1), fields, -1)
    assert vnext is fields[0] and dtn == 25.0
    vel, vnext, dtn = vel_payload(resolve_time_bracket(200.0, ft), fields, 1)
    assert vel is fields[2] and vnext is None and dtn is None


def test_recon_stencil_and_record_clock_match_reference():
    """The PCHIP stencil of each bracket (tracking._resolve_recon_stencil) and
    the clock after a step that ends on the record ahead
    (tracking._step_end_on_record), including clocks a cycle period away."""
    from kelp_b200.tracking import resolve_recon_stencil, step_end_on_record
    d = np.load(os.path.join(os.path.dirname(__file__), "golden", "golden_clock.npz"))
    axes = [d["axis_uniform"], d["axis_ragged"]]
    modes = ["stop", "cycle"]
    n_stencil = 0
    for row in d["rows"]:
        ai, mi, direction, t = int(row[0]), int(row[1]), int(row[2]), float(row[3])
        b = (int(row[4]), int(row[5]), row[6], row[7], row[8])
        st = resolve_recon_stencil(b, axes[ai].size)
        want = [int(x) for x in row[9:13]]
        if want[0] < 0:
            assert st is None, row
        else:
            n_stencil += 1
            assert list(st[0]) == want and st[1] == b[4], row
        end = step_end_on_record(t, b[4], float(row[13]), direction, axes[ai], modes[mi])
        assert end == float(row[14]), (row, end)
    assert n_stencil > 0
