"""The trajectory store and restart checkpoints (kelp_b200.writers), on the
host: records round-trip, a checkpoint carries every optional array and
replaces the previous one whole, a store without one refuses to load."""
import os

import numpy as np
import pytest

from kelp_b200.particles import ParticleState
from kelp_b200.writers import TrajectoryWriter, load_restart, read_trajectory


def _state(P, k):
    rng = np.random.default_rng(k)
    return ParticleState(lon=rng.uniform(-10, 10, P), lat=rng.uniform(-5, 5, P), z=rng.uniform(0, 50, P),
                         status=np.full(P, 1, np.int32), nearest_node=np.arange(P, dtype=np.int32),
                         u=rng.normal(size=P), v=rng.normal(size=P), failure_reason=np.zeros(P, np.int8),
                         elem=np.arange(P, dtype=np.int32) * 2)


def test_records_round_trip(tmp_path):
    P = 7
    w = TrajectoryWriter(str(tmp_path / "t"), P, metadata={"note": "x"}).open()
    states = [_state(P, k) for k in range(3)]
    for k, s in enumerate(states):
        w.append(s, 3600.0 * (k + 1))
    w.write_release(states[0].lon, states[0].lat, states[0].z, np.zeros(P))
    assert w.n_obs == 3
    tr = read_trajectory(str(tmp_path / "t"))
    np.testing.assert_array_equal(tr["time"], [3600.0, 7200.0, 10800.0])
    np.testing.assert_array_equal(tr["lon"], np.stack([s.lon for s in states]))
    np.testing.assert_array_equal(tr["vel_u"], np.stack([s.u for s in states]))
    np.testing.assert_array_equal(tr["release_lat"], states[0].lat)
    with pytest.raises(ValueError):
        w.append(_state(P + 1, 0), 1.0)
    with pytest.raises(ValueError):
        w.append(states[0], float("nan"))


def test_checkpoint_round_trip_and_replace(tmp_path):
    P = 5
    path = str(tmp_path / "c")
    w = TrajectoryWriter(path, P).open()
    with pytest.raises(ValueError):
        load_restart(path)
    s1, s2 = _state(P, 1), _state(P, 2)
    w.write_checkpoint(s1, 9, 2, wet_streak=np.arange(P), release_step=np.full(P, 3), particle_offset=100,
                       uv_vertical="level")
    w.write_checkpoint(s2, 19, 4, wet_streak=np.arange(P) + 1)
    r = load_restart(path)
    assert r["step_i"] == 19 and r["file_idx"] == 4 and r["particle_offset"] is None
    np.testing.assert_array_equal(r["state"].lon, s2.lon)
    np.testing.assert_array_equal(r["state"].elem, s2.elem)
    np.testing.assert_array_equal(r["wet_streak"], np.arange(P) + 1)
    assert r["release_step"] is None and r["state"].release_step is None
    assert not any(f.endswith(".tmp.npz") for f in os.listdir(path))


def test_resume_after_a_crash_drops_the_records_past_the_checkpoint(tmp_path):
    """A run checkpoints after 3 records, writes 2 more and stops; the resumed
    run reopens the store: numbering continues at 3, the 2 records written
    after the checkpoint are gone (the resumed run writes them again), so no
    observation is duplicated."""
    P = 5
    path = str(tmp_path / "t")
    w = TrajectoryWriter(path, P).open()
    for k in range(3):
        w.append(_state(P, k), 3600.0 * (k + 1))
    w.write_checkpoint(_state(P, 2), step_i=3, file_idx=3)
    for k in range(3, 5):
        w.append(_state(P, k), 3600.0 * (k + 1))
    assert w.n_obs == 5
    w2 = TrajectoryWriter(path, P).open()   # the resumed run
    assert w2.n_obs == 3
    for k in range(3, 6):
        w2.append(_state(P, 10 + k), 3600.0 * (k + 1))
    tr = read_trajectory(path)
    np.testing.assert_array_equal(tr["time"], 3600.0 * np.arange(1, 7))
    np.testing.assert_array_equal(tr["lon"][3], _state(P, 13).lon)
