"""The grid-hash occupancy cell rule (core.mesh.choose_grid_hash_cell,
src/kelp/core/mesh.py:464-706) against the reference's own reports and its
per-sample kernel _gh_sample_stats (:384-461), recorded by
tests/golden/make_golden.py on three meshes: a seam-wrapping global band
(sampled), a sinh-stretched regional mesh (exact mode shrinks the cell), a
near-polar mesh whose caps reach the pole.

CPU: the oracle's restatement of the per-sample kernel equals the recorded
arrays, and the host's ladder and decisions, fed by the oracle through a
stand-in context, reproduce both recorded reports.  GPU: kc_grid_cell_stats
equals the recorded arrays and the chooser on the device reproduces the
reports; the rule's pin / reuse / reset behaviour.
"""
import json
import os

import numpy as np
import pytest

from conftest import GOLDEN

MESHES = ("band", "stretched", "polar")


def _load(name):
    d = dict(np.load(os.path.join(GOLDEN, f"golden_cellrule_{name}.npz")))
    return d


def _mesh(d):
    from kelp_b200.mesh import Mesh, build_grid_hash, build_node_to_elems
    en = d["mesh_elem_nodes"]
    n2e, cnt = build_node_to_elems(d["mesh_nodes_lon"].size, en)
    m = Mesh(name="cellrule", nodes_lon=d["mesh_nodes_lon"], nodes_lat=d["mesh_nodes_lat"], depth=d["mesh_depth"],
             elem_nodes=en, elem_center_lon=d["mesh_elem_center_lon"], elem_center_lat=d["mesh_elem_center_lat"],
             node_to_elems=n2e, node_to_elems_count=cnt)
    m.metadata["exact_nearest"] = True
    build_grid_hash(m)
    g = d["mesh_gh_geom"]
    assert m._gh_cell_size == g[0] and np.array_equal(m._gh_offsets, d["mesh_gh_offsets"])
    return m


def _cum(m, cell, lon_min, lat_min, nx, ny, wrap):
    from kelp_b200.mesh import _gh_cell_index, _gh_lon_branch
    lon_b, _ = _gh_lon_branch(np.asarray(m.nodes_lon, dtype=np.float64))
    idx = _gh_cell_index(lon_b, np.asarray(m.nodes_lat), cell, lon_min, lat_min, nx, ny, wrap)
    cum = np.zeros((ny + 1, nx + 1), dtype=np.int64)
    cum[1:, 1:] = np.bincount(idx, minlength=nx * ny).reshape(ny, nx).cumsum(axis=0).cumsum(axis=1)
    return cum.astype(np.int32)


class OracleContext:
    """A stand-in device context whose per-sample statistics come from the
    oracle (the exact nearest node and the restated _gh_sample_stats)."""

    def __init__(self):
        self.mesh = None

    def ensure_mesh(self, mesh):
        self.mesh = mesh

    def grid_cell_stats(self, lon_branch, cell, lon_min, lat_min, nx, ny, wrap, lon, lat):
        from oracle import oracle as O
        nn = O.find_nearest(self.mesh, lon, lat)
        occ, cost, unprov, approx = O.cell_stats(self.mesh, _cum(self.mesh, cell, lon_min, lat_min, nx, ny, wrap),
                                                 cell, lon_min, lat_min, nx, ny, wrap, lon, lat, nn)
        return nn, occ, cost, unprov, approx


@pytest.mark.parametrize("name", MESHES)
def test_oracle_sample_stats_equal_reference(name):
    from oracle import oracle as O
    d = _load(name)
    m = _mesh(d)
    assert np.array_equal(O.find_nearest(m, d["qlon"], d["qlat"]), d["nn"])
    for k in (0, 2, 5):
        cell, lon_min, lat_min, nx, ny, wrap = d[f"k{k}_geom"]
        nx, ny, wrap = int(nx), int(ny), bool(wrap)
        got = O.cell_stats(m, _cum(m, cell, lon_min, lat_min, nx, ny, wrap), cell, lon_min, lat_min, nx, ny, wrap,
                           d["qlon"], d["qlat"], d["nn"])
        for key, g in zip(("occ", "cost", "unprov", "approx"), got):
            assert np.array_equal(g, d[f"k{k}_{key}"]), (name, k, key)


@pytest.mark.parametrize("name", MESHES)
def test_host_chooser_reproduces_reports(name):
    from kelp_b200.gridcell import choose_grid_hash_cell
    d = _load(name)
    m = _mesh(d)
    for mode in ("exact", "approx"):
        want = json.loads(str(d[f"report_{mode}"]))
        cell, rep = choose_grid_hash_cell(m, ctx=OracleContext(), exact=(mode == "exact"), sample=int(d["sample"]))
        assert cell == want["chosen"]
        assert rep == want, (name, mode)


@pytest.mark.gpu
@pytest.mark.parametrize("name", MESHES)
def test_device_sample_stats_equal_reference(name):
    from kelp_b200.device import default_context
    from kelp_b200.mesh import _gh_lon_branch
    d = _load(name)
    m = _mesh(d)
    ctx = default_context()
    ctx.ensure_mesh(m)
    lon_b, wrap = _gh_lon_branch(np.asarray(m.nodes_lon, dtype=np.float64))
    for k in (0, 2, 5):
        cell, lon_min, lat_min, nx, ny, _ = d[f"k{k}_geom"]
        nn, occ, cost, unprov, approx = ctx.grid_cell_stats(lon_b, cell, lon_min, lat_min, int(nx), int(ny), wrap,
                                                            d["qlon"], d["qlat"])
        assert np.array_equal(nn, d["nn"])
        assert np.array_equal(occ, d[f"k{k}_occ"]) and np.array_equal(approx, d[f"k{k}_approx"])
        # the certificate's verdict and the widened rectangle come from
        # acos / asin of the cap: the device's functions, which may round a
        # boundary case differently from the C library's, so mismatches are
        # counted (none were seen on these meshes) rather than assumed away
        bad = int(np.count_nonzero((unprov != d[f"k{k}_unprov"]) | (cost != d[f"k{k}_cost"])))
        print(f"{name} k={k}: {bad} of {nn.size} samples differ")
        assert bad == 0


@pytest.mark.gpu
@pytest.mark.parametrize("name", MESHES)
def test_device_chooser_reproduces_reports(name):
    from kelp_b200.device import default_context
    from kelp_b200.gridcell import choose_grid_hash_cell
    d = _load(name)
    m = _mesh(d)
    for mode in ("exact", "approx"):
        want = json.loads(str(d[f"report_{mode}"]))
        cell, rep = choose_grid_hash_cell(m, ctx=default_context(), exact=(mode == "exact"), sample=int(d["sample"]))
        assert rep == want, (name, mode)


@pytest.mark.gpu
def test_apply_rule_pins_reuses_and_resets():
    from kelp_b200.device import default_context
    from kelp_b200.gridcell import apply_grid_hash_cell_rule, describe_grid_hash
    d = _load("stretched")
    m = _mesh(d)
    ctx = default_context()
    legacy = m._gh_cell_size
    rep = apply_grid_hash_cell_rule(m, "occupancy", ctx=ctx)
    want = json.loads(str(d["report_exact"]))
    assert rep == want and m._gh_cell_size == want["chosen"] != legacy
    assert m.metadata["grid_hash_cell"] == want["chosen"] and m.metadata["grid_hash_cell_rule"] == "occupancy"
    assert "by occupancy/exact" in describe_grid_hash(m)
    assert apply_grid_hash_cell_rule(m, "occupancy", ctx=ctx) is rep          # the same decision, not re-run
    back = apply_grid_hash_cell_rule(m, "legacy", ctx=ctx)
    assert back["rule"] == "legacy" and m._gh_cell_size == legacy and "grid_hash_cell" not in m.metadata


def test_rule_name_and_explicit_pin():
    from kelp_b200.gridcell import apply_grid_hash_cell_rule, describe_grid_hash
    from kelp_b200.mesh import set_grid_hash_cell
    d = _load("band")
    m = _mesh(d)
    with pytest.raises(ValueError):
        apply_grid_hash_cell_rule(m, "smallest", ctx=OracleContext())
    set_grid_hash_cell(m, 3.0)
    rep = apply_grid_hash_cell_rule(m, "occupancy", ctx=OracleContext())
    assert rep["rule"] == "explicit" and m._gh_cell_size == 3.0
    assert "explicit" in describe_grid_hash(m)
