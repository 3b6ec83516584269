"""The oracle's restatement of sampling.py:727 sample_field against the
reference's own outputs (tests/golden/golden_sample_*.npz, made by
make_golden.py from the reference): 2-D node fields and z-level mid-layer
fields, every horizontal method, fill NaNs, points on nodes, dead particles
and nearest = -1.  Bar: bit-identical (NaN where the reference gives NaN)."""
import numpy as np
import pytest

METHODS = ("nearest", "leastsq", "barycentric", "idw")


def _same(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return int(np.count_nonzero(~((a == b) | (np.isnan(a) & np.isnan(b)))))


@pytest.mark.parametrize("name", ["band", "quad", "3d"])
@pytest.mark.parametrize("method", METHODS)
def test_oracle_sample_matches_reference(golden, name, method):
    from oracle import oracle as O
    g = golden(f"golden_sample_{name}")
    d = g.d
    got = O.sample_field(d["v2"], g.mesh, d["lon"], d["lat"], nearest=d["nearest"], alive=d["alive"], method=method)
    assert _same(got, d[f"o2_{method}"]) == 0
    if "v3" in d:
        got3 = O.sample_field(d["v3"], g.mesh, d["lon"], d["lat"], d["z"], nearest=d["nearest"], alive=d["alive"],
                              method=method)
        assert _same(got3, d[f"o3_{method}"]) == 0


def test_sample_fixtures_exercise_the_edge_cases(golden):
    """The fixtures hold what the rules are about: fill NaNs among the
    values, dead particles and nearest = -1 (NaN out), and finite results
    that differ between methods."""
    d = golden("golden_sample_3d").d
    assert np.isnan(d["v2"]).any() and np.isnan(d["v3"]).any()
    assert (~d["alive"]).any() and (d["nearest"] < 0).any()
    dead = ~d["alive"] | (d["nearest"] < 0)
    for m in METHODS:
        assert np.isnan(d[f"o2_{m}"][dead]).all()
    fin = np.isfinite(d["o2_leastsq"]) & np.isfinite(d["o2_idw"])
    assert np.count_nonzero(d["o2_leastsq"][fin] != d["o2_idw"][fin]) > 100


def test_sample_field_host_validation(golden):
    """The reference's argument errors, raised before any device work."""
    from kelp_b200.sampling import sample_field
    g = golden("golden_sample_3d")
    d = g.d
    with pytest.raises(ValueError, match="method"):
        sample_field(d["v2"], g.mesh, d["lon"], d["lat"], method="cubic")
    with pytest.raises(ValueError, match="node"):
        sample_field(d["v2"][:-1], g.mesh, d["lon"], d["lat"])
    with pytest.raises(ValueError, match="zs"):
        sample_field(d["v3"], g.mesh, d["lon"], d["lat"])
    K = np.asarray(g.mesh.sigma).size
    with pytest.raises(ValueError, match="K-1"):
        sample_field(np.zeros((K + 3, d["v2"].size)), g.mesh, d["lon"], d["lat"], d["z"])


@pytest.mark.parametrize("method", METHODS)
def test_oracle_interface_field_matches_reference(golden, method):
    """An interface-shaped (K, N) field: sample_field hands it to the W
    interpolation of the method (sampling.py:876-890)."""
    from oracle import oracle as O
    g = golden("golden_sample_iface")
    d = g.d
    got = O.sample_field(d["vk"], g.mesh, d["lon"], d["lat"], d["z"], nearest=d["nearest"], alive=d["alive"],
                         method=method)
    assert _same(got, d[f"ok_{method}"]) == 0
    assert np.isfinite(d[f"ok_{method}"][d["alive"] & (d["nearest"] >= 0)]).all()


@pytest.mark.parametrize("method", METHODS)
def test_oracle_sigma_fields_match_reference(golden, method):
    """Sigma-mesh sampling (sampling.py:620-723): an interface field through
    the sigma W interpolation, a mid-layer field in the node columns
    max(depth + eta, Dmin)."""
    from oracle import oracle as O
    g = golden("golden_sample_sigma")
    d = g.d
    for key, out in (("vk", "ok"), ("vm", "om")):
        got = O.sample_field(d[key], g.mesh, d["lon"], d["lat"], d["z"], nearest=d["nearest"], alive=d["alive"],
                             method=method, eta=d["eta"], Dmin=0.5)
        assert _same(got, d[f"{out}_{method}"]) == 0, key
