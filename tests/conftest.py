"""Shared fixtures of the test suite.

``gpu``-marked tests need a CUDA device and the built native library; every
other test runs on CPU.  Golden fixtures (``tests/golden/*.npz``) hold inputs
and the reference's own outputs, produced by ``tests/golden/make_golden.py``.
"""
import os
import sys
import types

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built native library")
    config.addinivalue_line("markers", "slow: long-running")


class Golden:
    """One golden fixture: the mesh (reference-built grid hash and node table),
    snapshots, particles, and the recorded runs."""

    def __init__(self, name):
        self.name = name
        self.d = dict(np.load(os.path.join(GOLDEN, f"{name}.npz")))
        g = self.d["mesh_gh_geom"]
        m = types.SimpleNamespace()
        for k in ("nodes_lon", "nodes_lat", "depth", "elem_nodes", "node_to_elems", "node_to_elems_count",
                  "sigma"):
            setattr(m, k, self.d[f"mesh_{k}"])
        m._gh_offsets = self.d["mesh_gh_offsets"]
        m._gh_node_ids = self.d["mesh_gh_node_ids"]
        m._node_xyz = self.d["mesh_node_xyz"]
        m._gh_cell_size, m._gh_lon_min, m._gh_lat_min = float(g[0]), float(g[1]), float(g[2])
        m._gh_nx, m._gh_ny, m._gh_wrap_lon, m._gh_far_rows = int(g[3]), int(g[4]), bool(g[5]), int(g[6])
        m.r_earth = float(g[7])
        m.vertical_coord = str(self.d["mesh_vertical_coord"]) if "mesh_vertical_coord" in self.d else "zlevel"
        m.metadata = {"exact_nearest": True}
        m._elem_neighbors = self.d.get("mesh_elem_neighbors")
        if "mesh_elem_center_lon" in self.d:   # element centres (least-squares u/v)
            m.elem_center_lon = self.d["mesh_elem_center_lon"]
            m.elem_center_lat = self.d["mesh_elem_center_lat"]
        self.uv_element = "mesh_uv_element" in self.d
        self.uv_edge = "mesh_uv_edge" in self.d   # element-layout u/v by the edge-neighbour fit
        if "mesh_cgrid_corners" in self.d:   # a NEMO C-grid mesh (build_nemo_cgrid_mesh)
            m._nemo_cgrid = True
            for k in ("corners", "elem_ji", "nlev", "nlev_raster", "zw", "area", "e3b", "kbu", "e3u", "kbv", "e3v",
                      "e2u", "e1v"):
                setattr(m, "_nemo_cgrid_" + k, self.d["mesh_cgrid_" + k])
            m._structured_shape = tuple(int(x) for x in self.d["mesh_cgrid_shape"])
            m._nemo_cgrid_partial = str(self.d["mesh_cgrid_partial"])
        self.mesh = m
        from kelp_b200.fields import VelocityField
        placement = {"golden_dl_lev": "level", "golden_dl_llin": "layer_linear",
                     "golden_sigma_llin": "layer_linear"}.get(name, "layer")
        self.snaps = []
        i = 0
        while f"snap{i}_u" in self.d:
            w = self.d.get(f"snap{i}_w")
            eta = self.d.get(f"snap{i}_eta")
            self.snaps.append(VelocityField(u=self.d[f"snap{i}_u"], v=self.d[f"snap{i}_v"], w=w,
                                            eta=np.zeros(self.d[f"snap{i}_u"].shape[-1]) if eta is None else eta,
                                            uv_layout=("nemo_cgrid" if "mesh_cgrid_corners" in self.d else
                                                       "element" if self.uv_element else "node"),
                                            uv_vertical=placement if w is not None else "layer",
                                            az=self.d.get(f"snap{i}_az"),
                                            scalars={k[len(f"snap{i}_scalar_"):]: self.d[k] for k in self.d
                                                     if k.startswith(f"snap{i}_scalar_")} or None))
            i += 1

    def cases(self):
        return sorted({k.split("__")[0] for k in self.d if "__" in k})

    def case(self, name):
        pre = name + "__"
        return {k[len(pre):]: v for k, v in self.d.items() if k.startswith(pre)}

    def particles(self):
        from kelp_b200.particles import ParticleState
        P = self.d["p_lon"].size
        return ParticleState(lon=self.d["p_lon"].copy(), lat=self.d["p_lat"].copy(), z=self.d["p_z"].copy(),
                             status=self.d["p_status"].copy(), nearest_node=np.full(P, -1, np.int32),
                             failure_reason=np.zeros(P, np.int8))

    def payload(self, sched_row, T):
        """(vel, vel_next, dt_to_next) of one recorded step (a steady step,
        recorded with dt_to_next -1, reads the first record alone)."""
        from kelp_b200.fields import LazyLerpField
        ia, alpha, dtn = int(sched_row[0]), float(sched_row[1]), float(sched_row[2])
        if dtn < 0:
            return self.snaps[ia], None, None
        a, b = self.snaps[ia], self.snaps[ia + 1]
        if abs(alpha) < 1e-12:
            vel = a
        elif abs(alpha - 1.0) < 1e-12:
            vel = b
        else:
            vel = LazyLerpField(a, b, alpha)
        return vel, b, dtn


@pytest.fixture(scope="session")
def golden():
    cache = {}

    def get(name):
        if name not in cache:
            cache[name] = Golden(name)
        return cache[name]

    return get
