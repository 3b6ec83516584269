"""The grid hash built on the device (kc_grid_hash_build) equals the host
build -- itself pinned to the reference's tables by test_host.py -- bit for
bit: offsets and the stable node order, on a global lattice (wrapped
longitudes), a regional mesh, a HEALPix dual mesh and a 1 M-node tripolar
C-grid mesh."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _meshes(golden):
    from kelp_b200 import healpix as H
    from kelp_b200 import synthetic as S
    from kelp_b200 import workloads as W
    yield "lattice", S.lattice_mesh(0.75, 80.0, jitter=0.2, land_frac=0.3)
    yield "golden_quad", golden("golden_quad").mesh
    nside = 64
    pix = np.arange(12 * nside * nside)
    plon, plat = H.pix2lonlat(nside, pix)
    wet = S._sphere_noise(plon, plat, seed=2) > -0.3
    yield "healpix64", H.dual_mesh(nside, wet, np.full(pix.size, 1000.0))
    yield "c5_tripolar", W.c5(P=1000).mesh


def test_device_grid_hash_equals_host(golden):
    from kelp_b200 import mesh as M
    from kelp_b200.device import default_context
    ctx = default_context()
    for name, m in _meshes(golden):
        host = M.Mesh(name="h", nodes_lon=np.asarray(m.nodes_lon), nodes_lat=np.asarray(m.nodes_lat),
                      depth=np.zeros(len(m.nodes_lon)), elem_nodes=np.asarray(m.elem_nodes),
                      elem_center_lon=np.zeros(1), elem_center_lat=np.zeros(1),
                      node_to_elems=np.asarray(m.node_to_elems), node_to_elems_count=np.asarray(m.node_to_elems_count))
        dev = M.Mesh(**{f: getattr(host, f) for f in ("name", "nodes_lon", "nodes_lat", "depth", "elem_nodes",
                                                      "elem_center_lon", "elem_center_lat", "node_to_elems",
                                                      "node_to_elems_count")})
        M.build_grid_hash(host)
        M.build_grid_hash(dev, ctx=ctx)
        np.testing.assert_array_equal(dev._gh_offsets, host._gh_offsets, err_msg=name)
        np.testing.assert_array_equal(dev._gh_node_ids, host._gh_node_ids, err_msg=name)
        assert (dev._gh_nx, dev._gh_ny, dev._gh_far_rows) == (host._gh_nx, host._gh_ny, host._gh_far_rows)
