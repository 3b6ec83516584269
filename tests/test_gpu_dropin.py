"""The drop-in contract with objects shaped exactly like KELP's own.

``tests/golden/reference_types.json`` records (from the reference itself)
the field lists of ``kelp.core.mesh.Mesh``, ``kelp.core.io.VelocityField``,
``kelp.core.particles.ParticleState``, ``kelp.core.io.LazyLerpField`` and
``kelp.numerics.diffusion.DiffusionStepArgs`` (a NamedTuple, with its
defaults), and the read-only properties the classes define.  Here classes with
those fields and properties and nothing else (dataclasses with a ``replace``,
a NamedTuple) carry a golden case's mesh, payload and
particles through ``kelp_b200.integrators.get_integrator`` -- the
registry KELP's tracking loop calls -- and the result must be the reference's
recorded one, returned as the caller's own state type.
"""
import collections
import dataclasses
import json
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
TYPES = json.load(open(os.path.join(HERE, "golden", "reference_types.json")))


# What each recorded property returns in KELP (kelp/core/mesh.py:167-190,
# kelp/core/particles.py:224-231); z_levels, the zlevel column boundaries,
# is |sigma| on a zlevel mesh and an error on a sigma mesh.
PROPERTIES = {
    "n_nodes": lambda m: m.nodes_lon.shape[0],
    "n_elements": lambda m: m.elem_nodes.shape[0],
    "n_sigma": lambda m: m.sigma.shape[0],
    "z_levels": lambda m: np.abs(m.sigma) if m.vertical_coord == "zlevel" else (_ for _ in ()).throw(
        NotImplementedError("mesh.z_levels is only valid for z-level meshes")),
    "n_particles": lambda s: s.lon.shape[0],
    "alive_mask": lambda s: s.status == 1,
}


def _dataclass(name, fields):
    ns = {"replace": lambda self, **kw: dataclasses.replace(self, **kw)}
    ns.update({p: property(PROPERTIES[p]) for p in TYPES["properties"].get(name, [])})
    return dataclasses.make_dataclass(name, [(f, object, dataclasses.field(default=None)) for f in fields],
                                      namespace=ns)


Mesh = _dataclass("Mesh", TYPES["Mesh"])
VelocityField = _dataclass("VelocityField", TYPES["VelocityField"])
ParticleState = _dataclass("ParticleState", TYPES["ParticleState"])
LazyLerpField = _dataclass("LazyLerpField", TYPES["LazyLerpField"])
DiffusionStepArgs = collections.namedtuple("DiffusionStepArgs", TYPES["DiffusionStepArgs"],
                                           defaults=[TYPES["DiffusionStepArgs_defaults"].get(f)
                                                     for f in TYPES["DiffusionStepArgs"]])


def _mesh(g):
    d, src = g.d, g.mesh
    m = Mesh(name=g.name, nodes_lon=src.nodes_lon, nodes_lat=src.nodes_lat, depth=src.depth,
             elem_nodes=src.elem_nodes, elem_center_lon=np.zeros(src.elem_nodes.shape[0]),
             elem_center_lat=np.zeros(src.elem_nodes.shape[0]), node_to_elems=src.node_to_elems,
             node_to_elems_count=src.node_to_elems_count, sigma=src.sigma, vertical_coord=src.vertical_coord,
             r_earth=src.r_earth, metadata={"exact_nearest": True})
    for k in ("_gh_offsets", "_gh_node_ids", "_gh_cell_size", "_gh_lon_min", "_gh_lat_min", "_gh_nx", "_gh_ny",
              "_gh_wrap_lon", "_gh_far_rows", "_node_xyz", "_elem_neighbors"):
        setattr(m, k, getattr(src, k))
    return m


def _snaps(g):
    return [VelocityField(u=s.u, v=s.v, eta=s.eta, w=s.w, uv_layout="node", uv_vertical=s.uv_vertical)
            for s in g.snaps]


@pytest.mark.parametrize("fixture,cname", [("golden_band", "rk2"), ("golden_3d", "rk2_wbary_kick"),
                                           ("golden_3d", "rk4_wnear")])
def test_reference_shaped_objects_through_the_registry(golden, fixture, cname):
    from kelp_b200 import integrators as KI
    g = golden(fixture)
    c = g.case(cname)
    dt, T, n_steps, td, khx, khy, seed, real_id, pid_off = c["params"]
    mesh, snaps = _mesh(g), _snaps(g)
    P = g.d["p_lon"].size
    st = ParticleState(lon=g.d["p_lon"].copy(), lat=g.d["p_lat"].copy(), z=g.d["p_z"].copy(),
                       status=g.d["p_status"].copy(), nearest_node=np.full(P, -1, np.int32),
                       failure_reason=np.zeros(P, np.int8))
    step = KI.get_integrator(cname.split("_")[0])
    for k in range(int(n_steps)):
        ia, alpha, dtn = int(c["schedule"][k][0]), float(c["schedule"][k][1]), float(c["schedule"][k][2])
        a, b = snaps[ia], snaps[ia + 1]
        vel = a if abs(alpha) < 1e-12 else (b if abs(alpha - 1.0) < 1e-12 else LazyLerpField(a, b, alpha))
        diff = None
        if khx >= 0:
            diff = DiffusionStepArgs(scheme="uniform", kh_x=khx, kh_y=khy, seed=int(seed), real_id=int(real_id),
                                     step_i=k, pid_offset=int(pid_off))
        st = step(st, vel, mesh, dt, td, uv_interp="barycentric",
                  w_interp="barycentric" if "wbary" in cname else "nearest", vel_next=b, dt_to_next=dtn,
                  diffusion=diff)
    assert type(st) is ParticleState   # the caller's own type, built by its replace
    tag = f"s{int(n_steps)}_"
    for name in ("status", "nearest_node", "failure_reason"):
        np.testing.assert_array_equal(np.asarray(getattr(st, name)), c[tag + name], err_msg=name)
    for name in ("lon", "lat"):
        np.testing.assert_allclose(np.asarray(getattr(st, name)), c[tag + name], rtol=0, atol=1e-9 / 0.0174533)
    np.testing.assert_allclose(np.asarray(st.z), c[tag + "z"], rtol=0, atol=1e-6)
