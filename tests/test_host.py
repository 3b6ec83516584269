"""Host-side logic on CPU: the C-ABI library loads and exports every symbol
its header declares; the host mirror of the mesh set-up reproduces the
reference's arrays; the step functions reject unsupported input in Python,
before any device work."""
import os
import re

import numpy as np
import pytest

from kelp_b200 import _native as N
from kelp_b200 import mesh as M

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_library_exports_every_declared_symbol():
    hdr = open(os.path.join(ROOT, "include", "kelp_cuda.h")).read()
    declared = set(re.findall(r"\b(kc_[a-z0-9_]+)\s*\(", hdr))
    L = N.lib()
    missing = [s for s in declared if not hasattr(L, s)]
    assert not missing, missing
    assert declared == set(N.EXPORTS)
    assert L.kc_abi_version() == N.ABI_VERSION == 14


def test_node_xyz_host_routine_matches_reference_table(golden):
    g = golden("golden_band")
    got = M.node_xyz_table(g.mesh.nodes_lon, g.mesh.nodes_lat)
    np.testing.assert_array_equal(got, g.mesh._node_xyz)


@pytest.mark.parametrize("fixture", ["golden_band", "golden_quad", "golden_3d"])
def test_grid_hash_mirror_matches_reference(golden, fixture):
    g = golden(fixture)
    m = M.Mesh(name="x", nodes_lon=g.mesh.nodes_lon, nodes_lat=g.mesh.nodes_lat, depth=g.mesh.depth,
               elem_nodes=g.mesh.elem_nodes, elem_center_lon=np.zeros(1), elem_center_lat=np.zeros(1),
               node_to_elems=g.mesh.node_to_elems, node_to_elems_count=g.mesh.node_to_elems_count)
    M.build_grid_hash(m)
    np.testing.assert_array_equal(m._gh_offsets, g.mesh._gh_offsets)
    np.testing.assert_array_equal(m._gh_node_ids, g.mesh._gh_node_ids)
    np.testing.assert_array_equal(M.ensure_node_xyz(m), g.mesh._node_xyz)
    assert (m._gh_cell_size, m._gh_lon_min, m._gh_lat_min, m._gh_nx, m._gh_ny, m._gh_wrap_lon, m._gh_far_rows) == \
        (g.mesh._gh_cell_size, g.mesh._gh_lon_min, g.mesh._gh_lat_min, g.mesh._gh_nx, g.mesh._gh_ny,
         g.mesh._gh_wrap_lon, g.mesh._gh_far_rows)


def test_pinned_cell_matches_reference(golden):
    g = golden("golden_polar")
    m = M.Mesh(name="x", nodes_lon=g.mesh.nodes_lon, nodes_lat=g.mesh.nodes_lat, depth=g.mesh.depth,
               elem_nodes=g.mesh.elem_nodes, elem_center_lon=np.zeros(1), elem_center_lat=np.zeros(1),
               node_to_elems=g.mesh.node_to_elems, node_to_elems_count=g.mesh.node_to_elems_count)
    M.set_grid_hash_cell(m, g.mesh._gh_cell_size)
    np.testing.assert_array_equal(m._gh_offsets, g.mesh._gh_offsets)
    np.testing.assert_array_equal(m._gh_node_ids, g.mesh._gh_node_ids)
    assert m._gh_far_rows == g.mesh._gh_far_rows


@pytest.mark.parametrize("fixture", ["golden_band", "golden_quad"])
def test_node_to_elems_matches_reference(golden, fixture):
    g = golden(fixture)
    n2e, cnt = M.build_node_to_elems(g.mesh.nodes_lon.size, g.mesh.elem_nodes)
    np.testing.assert_array_equal(cnt, g.mesh.node_to_elems_count)
    np.testing.assert_array_equal(n2e, g.mesh.node_to_elems)


def test_tri_as_quad_dedup():
    en = np.array([[0, 1, 2, 0], [1, 3, 2, -1]], np.int32)
    n2e, cnt = M.build_node_to_elems(4, en)
    assert list(cnt) == [1, 2, 2, 1]
    assert list(n2e[0]) == [0, -1]


def _tiny(golden):
    g = golden("golden_band")
    return g, g.particles(), g.snaps


def test_unsupported_paths_raise_before_device_work(golden):
    from kelp_b200 import integrators as KI
    from kelp_b200.diffusion import DiffusionStepArgs
    g, st, sn = _tiny(golden)
    kw = dict(uv_interp="barycentric", vel_next=sn[1], dt_to_next=86400.0)
    with pytest.raises(ValueError):   # least squares reads element-layout u/v; these are on nodes
        KI.rk2_step(st, sn[0], g.mesh, 3600.0, 1.0, **{**kw, "uv_interp": "leastsq"})
    with pytest.raises(ValueError):   # the edge-neighbour fit reads element-layout u/v too
        KI.rk2_step(st, sn[0], g.mesh, 3600.0, 1.0, **{**kw, "uv_interp": "edge_leastsq"})
    with pytest.raises(ValueError, match="edge_leastsq_bc"):
        KI.rk2_step(st, sn[0], g.mesh, 3600.0, 1.0, **{**kw, "uv_interp": "edge_leastsq", "edge_leastsq_bc": "slip"})
    with pytest.raises(NotImplementedError):
        KI.rk2_step(st, sn[0], g.mesh, 3600.0, 1.0, **{**kw, "uv_interp": "spline"})
    with pytest.raises(NotImplementedError):
        KI.rk2_step(st, sn[0], g.mesh, 3600.0, 1.0, **kw,
                    diffusion=DiffusionStepArgs("em", 1.0, 1.0, 0, 0, 0, composition="split_rk"))
    # malformed PCHIP bundles are refused as reconstruct_pchip refuses them
    with pytest.raises(ValueError):
        KI.rk2_step(st, sn[0], g.mesh, 3600.0, 1.0, **kw, recon=object())
    with pytest.raises(ValueError):   # times not increasing
        KI.rk2_step(st, sn[0], g.mesh, 3600.0, 1.0, **kw, recon=(sn[:4], [0.0, 2.0, 1.0, 3.0], 0.5, 1.0))
    with pytest.raises(ValueError):   # a stage outside the central interval
        KI.rk2_step(st, sn[0], g.mesh, 3600.0, 1.0, **kw,
                    recon=(sn[:4], [0.0, 86400.0, 172800.0, 259200.0], 172000.0, 1.0))
    with pytest.raises(ValueError):   # direction against time_dir
        KI.rk2_step(st, sn[0], g.mesh, 3600.0, 1.0, **kw,
                    recon=(sn[:4], [0.0, 86400.0, 172800.0, 259200.0], 90000.0, -1.0))
    with pytest.raises(NotImplementedError):   # PCHIP runs in the plain form
        KI.rk2_step(st, sn[0], g.mesh, 3600.0, 1.0, **kw, cuda_precision="mixed",
                    recon=(sn[:4], [0.0, 86400.0, 172800.0, 259200.0], 90000.0, 1.0))
    with pytest.raises(NotImplementedError):
        KI.get_integrator("rk45")(st, sn[0], g.mesh, 3600.0, 1.0)
    with pytest.raises(ValueError):
        KI.rk2_step(st, sn[0], g.mesh, -1.0, 1.0, **kw)
    with pytest.raises(ValueError):
        KI.rk2_step(st, sn[0], g.mesh, 3600.0, 0.5, **kw)
    with pytest.raises(ValueError):
        KI.rk2_step(st, sn[0], g.mesh, 3600.0, 1.0, uv_interp="barycentric", vel_next=sn[1])
    with pytest.raises(ValueError):
        KI.get_integrator("nope")


def test_all_dead_returns_without_device(golden):
    from kelp_b200 import integrators as KI
    g, st, sn = _tiny(golden)
    st = st.replace(status=np.full(st.n_particles, 3, np.int32))
    out = KI.rk2_step(st, sn[0], g.mesh, 3600.0, 1.0, uv_interp="barycentric", vel_next=sn[1], dt_to_next=86400.0)
    assert out is st
    st2 = st.replace(u=np.ones(st.n_particles), v=np.ones(st.n_particles))
    out2 = KI.rk2_step(st2, sn[0], g.mesh, 3600.0, 1.0, uv_interp="barycentric", vel_next=sn[1],
                       dt_to_next=86400.0)
    assert not out2.u.any() and not out2.v.any()


def test_registry_mirrors_reference():
    from kelp_b200 import integrators as KI
    assert set(KI.INTEGRATORS) == {"euler", "rk2", "rk4", "rk45"}
    assert KI.get_integrator("RK2") is KI.rk2_step


def test_autotune_cache_roundtrip(tmp_path, monkeypatch, golden):
    from kelp_b200 import autotune
    monkeypatch.setenv("KELP_B200_TUNE_CACHE", str(tmp_path / "t.json"))
    g = golden("golden_quad")
    key = autotune.mesh_signature(g.mesh, 2, "rk2", "plain", 1000)
    assert key.startswith("N") and "-d2-rk2-plain-P512" in key
    autotune._store({key: {"block": 256, "steps_per_launch": 6, "sort_every": 12}})
    assert autotune._load()[key]["block"] == 256


def test_shared_stride_of_3d_element_fields():
    """3-D element-layout u/v (K-1, E) and node w (K, N) upload with one row
    stride, max(E, N); node-layout fields pass through unchanged."""
    from kelp_b200.device import _shared_stride
    u, w = np.arange(30.0).reshape(3, 10), np.arange(24.0).reshape(4, 6)
    u2, v2, w2 = _shared_stride(u, u + 1.0, w)
    assert u2.shape == (3, 10) and v2.shape == (3, 10) and w2.shape == (4, 10)
    assert np.array_equal(w2[:, :6], w) and not w2[:, 6:].any() and np.array_equal(u2, u)
    u3, _, w3 = _shared_stride(np.ones((3, 4)), np.ones((3, 4)), np.ones((4, 9)))
    assert u3.shape == (3, 9) and w3.shape == (4, 9)
    n = np.ones((3, 5))
    assert _shared_stride(n, n, np.ones((4, 5)))[0] is n
