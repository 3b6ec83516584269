"""The CPU oracle against the reference's own outputs (golden fixtures).

Pins ``oracle/kelp_oracle.c`` before it is trusted as the checker of the CUDA
kernels.  Integer outputs (status, nearest node, failure reason) must match
bit for bit.  Positions and velocities of the fused reference kernels (2-D
RK2/RK4, 3-D RK2) match bit for bit too: both sides evaluate the same
expressions with the C library's math and no contraction.  The unfused
reference paths (Euler) evaluate their displacement metric with numpy's SIMD
``cos``, so there the tolerance is 1e-12 degrees.
"""
import numpy as np
import pytest

from oracle import oracle as O
from kelp_b200.diffusion import DiffusionStepArgs

CASES = [("golden_band", c) for c in ("rk2", "rk4", "euler", "rk2_bwd", "rk2_kick", "rk4_kick_aniso", "rk2_dt4800",
                                      "rk2_walk", "rk4_walk_kick", "euler_walk")]
CASES += [("golden_quad", c) for c in ("rk2", "rk4", "euler", "rk2_kick")]
CASES += [("golden_polar", "rk2")]
CASES += [("golden_3d", c) for c in ("rk2_wnear", "rk2_wbary", "rk2_wbary_kick", "rk4_wnear", "rk4_wbary_kick", "euler_wbary",
                                     "rk2_wbary_kick_azf", "rk4_wnear_azf_nokh", "rk2_wbary_walk",
                                     "rk4_wnear_walk_kick")]
CASES += [("golden_dl_lev", c) for c in ("rk2_lev_wbary", "rk4_lev_wnear_kick", "euler_lev_wnear", "rk2_lev_wbary_azc")]
CASES += [("golden_dl_llin", c) for c in ("rk2_llin_wbary", "rk4_llin_wnear_kick", "euler_llin_wnear")]
# W by least squares and by inverse distance (unfused reference steps)
CASES += [("golden_wring", c) for c in ("rk2_wlsq", "rk4_wlsq_kick", "euler_wlsq", "rk2_wlsq_bwd", "rk2_widw",
                                        "rk4_widw_kick")]
# sigma meshes (mesh.vertical_coord "sigma", free surface eta, s = z / H_p)
SIGMA_CASES = [("golden_sigma", c) for c in ("rk2_wnear", "rk2_wbary", "rk4_wbary", "euler_wbary", "euler_wnear",
                                             "rk2_wbary_kick", "rk4_wnear_kick", "rk2_wnear_bwd",
                                             "rk2_wbary_steady", "rk4_wnear_steady", "rk2_wbary_walk")]
SIGMA_CASES += [("golden_sigma_llin", c) for c in ("rk2_llin_wbary", "rk4_llin_wnear_kick", "euler_llin_wnear")]
# the tracking layer's surfaces supplied to sigma steps (sigma_eta_start / sigma_eta_end)
SIGMA_CASES += [("golden_sigma_surf", c) for c in ("rk2_wbary_surf", "rk4_wnear_surf", "euler_wbary_surf",
                                                  "rk2_wbary_steady_surf", "rk4_wnear_steady_surf_kick",
                                                  "rk4_wbary_steady_endonly", "rk2_wnear_startonly_kick")]
# W and the particle's column by least squares / inverse distance on sigma meshes
SIGMA_CASES += [("golden_sigma_wring", c) for c in ("rk2_wlsq", "rk4_widw_kick", "euler_wlsq", "rk2_widw_bwd",
                                                   "rk4_wlsq_surf_kick")]
# the vertical Az kick on sigma meshes (constant source, end-of-step column)
SIGMA_CASES += [("golden_sigma_az", c) for c in ("rk2_wbary_azc", "rk4_wnear_kick_azc", "euler_wbary_azc",
                                                "rk2_wnear_bwd_kick_azc", "rk2_wbary_surf_kick_azc")]
CASES += SIGMA_CASES
# NEMO C-grid meshes (uv_interp nemo_cgrid): the 2-D unfused steps and the 3-D fractional-level step
CGRID_CASES = [("golden_cgrid2d", c) for c in ("rk2", "rk4", "euler", "rk2_bwd", "rk4_steady", "rk2_kick", "rk2_walk")]
CGRID_CASES += [("golden_cgrid3d", c) for c in ("rk2", "rk4", "euler", "rk2_bwd", "rk4_steady")]
# a global tripolar raster (T-pivot north fold, E-W halo) built by the reference's own builder
CGRID_CASES += [(f"golden_cgrid_tripolar{d}", c) for d in ("2d", "3d") for c in ("rk2", "rk4")]
CASES += CGRID_CASES
# PCHIP temporal reconstruction (4-snapshot stencil; the last interval falls back to linear)
PCHIP_CASES = [("golden_pchip2d", c) for c in ("rk2", "rk4_kick")]
PCHIP_CASES += [("golden_pchip3d", c) for c in ("rk2_wbary", "rk4_wnear")]
PCHIP_CASES += [("golden_pchip_sigma", c) for c in ("rk4_wbary", "rk2_wnear")]
CASES += PCHIP_CASES
# element-layout u/v by element-centre least squares (uv_interp leastsq, 2-D)
LSQ_CASES = [(f, c) for f in ("golden_lsq_band", "golden_lsq_quad")
             for c in ("rk2", "rk4", "euler", "rk2_bwd", "rk2_kick", "rk4_steady", "rk2_pchip")]
CASES += LSQ_CASES
# 3-D element-layout u/v by least squares per layer, node W (the unfused reference steps)
LSQ_CASES += [("golden_lsq3d", c) for c in ("rk2_wbary", "rk4_wnear_kick", "euler_wlsq", "rk2_wlsq_bwd",
                                            "rk4_wbary_pchip")]
CASES += LSQ_CASES[-5:]
# element-layout u/v by the edge-neighbour least squares (freeslip / noslip ghosts)
EDGE_CASES = [(f, c) for f in ("golden_edge_band", "golden_edge_quad")
              for c in ("rk2", "rk4_noslip", "euler", "rk2_kick_noslip")]
EDGE_CASES += [("golden_edge3d", c) for c in ("rk2_wbary", "rk4_wlsq_noslip", "euler_wnear")]
CASES += EDGE_CASES


def w_interp_of(cname):
    """The recorded case's W method, from its name."""
    for tag, method in (("wlsq", "leastsq"), ("widw", "idw"), ("wbary", "barycentric")):
        if tag in cname:
            return method
    return "nearest"


def uv_interp_of(g):
    """The recorded fixture's u/v interpolator."""
    if getattr(g.mesh, "_nemo_cgrid", False):
        return "nemo_cgrid"
    if getattr(g, "uv_edge", False):
        return "edge_leastsq"
    return "leastsq" if g.uv_element else "barycentric"


def edge_kw(g, cname):
    """The edge_leastsq boundary rule of a recorded case (from its name)."""
    if not getattr(g, "uv_edge", False):
        return {}
    return {"edge_leastsq_bc": "noslip" if "noslip" in cname else "freeslip"}


def recon_of(g, c, k):
    """The recorded step's PCHIP bundle (tracking.py:2415-2436), or None."""
    row = c["schedule"][k]
    if row.shape[0] < 5 or row[3] != 1:
        return None
    T, td = float(c["params"][1]), float(c["params"][3])
    ia = int(row[0])
    idx = (ia - 1, ia, ia + 1, ia + 2)
    return ([g.snaps[i] for i in idx], [float(i * T) for i in idx], float(row[4]), td)


def diffusion_args(c, k):
    """The recorded case's DiffusionStepArgs of step k (None without diffusion)."""
    dt, T, n_steps, td, khx, khy, seed, real_id, pid_off = c["params"]
    if khx < 0:
        return None
    az = {}
    if "az" in c:
        az = dict(az_enabled=True, az_const=float(c["az"][0]), az_requires_field=bool(c["az"][1]))
    return DiffusionStepArgs("uniform", khx, khy, int(seed), int(real_id), k, pid_offset=int(pid_off), **az)


def surfaces_of(c, k):
    """The recorded step's sigma surfaces (start, end), None where not supplied."""
    return tuple(c[key][k] if key in c else None for key in ("sigma_eta_start", "sigma_eta_end"))


def replay_oracle(g, cname):
    c = g.case(cname)
    dt, T, n_steps, td, khx, khy, seed, real_id, pid_off = c["params"]
    scheme = cname.split("_")[0]
    w_interp = w_interp_of(cname)
    st = g.particles()
    if "elem0" in c:   # elem_search: walk
        st = st.replace(elem=c["elem0"].copy())
    view = O.MeshView(g.mesh)
    snaps = {}
    for k in range(int(n_steps)):
        vel, vnext, dtn = g.payload(c["schedule"][k], T)
        diff = diffusion_args(c, k)
        es, ee = surfaces_of(c, k)
        out = O.step(st, vel, g.mesh, dt, td, scheme, vel_next=vnext, dt_to_next=dtn, w_interp=w_interp,
                     diffusion=diff, view=view, recon=recon_of(g, c, k),
                     uv_interp={"nemo_cgrid": "barycentric"}.get(uv_interp_of(g), uv_interp_of(g)),
                     eta_start=es, eta_end=ee, **edge_kw(g, cname))
        st = st.replace(lon=out["lon"], lat=out["lat"], z=out["z"], status=out["status"],
                        nearest_node=out["nearest_node"], failure_reason=out["failure_reason"],
                        u=out["u"], v=out["v"], w=out["w"], elem=out.get("elem"))
        if f"s{k + 1}_lon" in c:
            snaps[k + 1] = out
    return c, snaps


@pytest.mark.parametrize("fixture,cname", CASES)
def test_oracle_matches_reference(golden, fixture, cname):
    g = golden(fixture)
    c, snaps = replay_oracle(g, cname)
    exact_float = not cname.startswith("euler")
    for k, out in snaps.items():
        tag = f"s{k}_"
        for name in ("status", "nearest_node", "failure_reason", "elem"):
            if tag + name in c:
                np.testing.assert_array_equal(out[name], c[tag + name], err_msg=f"{cname} step {k} {name}")
        for name in ("lon", "lat", "z", "u", "v", "w"):
            if tag + name not in c:
                continue
            if exact_float:
                np.testing.assert_array_equal(out[name], c[tag + name], err_msg=f"{cname} step {k} {name}")
            else:
                np.testing.assert_allclose(out[name], c[tag + name], rtol=0, atol=1e-12,
                                           err_msg=f"{cname} step {k} {name}")


@pytest.mark.parametrize("fixture", ["golden_quad", "golden_polar"])
def test_oracle_exact_nearest(golden, fixture):
    g = golden(fixture)
    got = O.find_nearest(g.mesh, g.d["p_q_lon"], g.d["p_q_lat"])
    np.testing.assert_array_equal(got, g.d["p_q_nearest"])


def test_oracle_rng_normals():
    import os
    d = np.load(os.path.join(os.path.dirname(__file__), "golden", "golden_rng.npz"))
    keys, want = d["keys"], d["normals"]
    got = np.empty_like(want)
    for i, k in enumerate(keys):
        g = np.empty(2)
        O.lib().orc_normal_pair(*(int(x) for x in k), g.ctypes.data)
        got[i] = g
    np.testing.assert_array_equal(got, want)


def test_oracle_node_xyz(golden):
    g = golden("golden_band")
    np.testing.assert_array_equal(O.node_xyz(g.mesh.nodes_lon, g.mesh.nodes_lat), g.mesh._node_xyz)


BEACH_CASES = ("dco_auto", "sto_both", "cd_sresusp", "depth_never", "eta_dry_auto", "eta_sto_both")
_RESUSP_NAMES = {0: "never", 1: "auto", 2: "stochastic", 3: "auto_or_stochastic"}


def beach_kwargs(c):
    """The hook's parameters recorded with a beaching case."""
    b = c["beach"]
    crit = [n for n, on in zip(("depth", "coastal_element", "stochastic", "on_failure"), b[:4]) if on]
    return dict(criteria=crit, resuspension=_RESUSP_NAMES[int(b[4])], min_wet_steps=int(b[5]),
                depth_min=float(b[6]), zone_depth=float(b[7]), rewet_hysteresis=float(b[8]),
                t_beach=float(b[9]), t_resuspend=float(b[10]), seed=int(b[11]),
                use_eta=bool(b[12]) if b.size > 12 else False,
                dry_mask_var="dry" if b.size > 13 and b[13] else None)


def beach_surfaces(vel, kw):
    """The payload's eta and dry mask the hook reads (tracking.py:236-327)."""
    from kelp_b200.beaching import BeachingConfig, payload_surfaces
    return payload_surfaces(vel, BeachingConfig(use_eta=kw["use_eta"], dry_mask_var=kw["dry_mask_var"]))


def replay_oracle_beach(g, cname):
    """RK2 (+ kick) steps, each followed by the beaching hook, on the oracle."""
    c = g.case(cname)
    dt, T, n_steps, td, khx, khy, seed, real_id, pid_off = c["params"]
    kw = beach_kwargs(c)
    st = g.particles()
    wet = np.zeros(st.n_particles, np.int32)
    view = O.MeshView(g.mesh)
    snaps = {}
    for k in range(int(n_steps)):
        vel, vnext, dtn = g.payload(c["schedule"][k], T)
        diff = None
        if khx >= 0:
            diff = DiffusionStepArgs("uniform", khx, khy, int(seed), int(real_id), k, pid_offset=int(pid_off))
        prev = st.status
        out = O.step(st, vel, g.mesh, dt, td, "rk2", vel_next=vnext, dt_to_next=dtn, diffusion=diff, view=view)
        st = st.replace(lon=out["lon"], lat=out["lat"], status=out["status"], nearest_node=out["nearest_node"],
                        failure_reason=out["failure_reason"])
        eta, dry = beach_surfaces(vel, kw)
        okw = {k: v for k, v in kw.items() if k not in ("use_eta", "dry_mask_var")}
        res, wet = O.beach(st, prev, g.mesh, g.d["p_coastal"], wet, real_id=int(real_id), step_i=k, dt=dt,
                           pid_offset=int(pid_off), view=view, eta=eta, dry_mask=dry, **okw)
        st = st.replace(**res)
        if f"s{k + 1}_status" in c:
            snaps[k + 1] = {"lon": st.lon, "lat": st.lat, "status": st.status, "nearest_node": st.nearest_node,
                            "failure_reason": st.failure_reason, "wet": wet}
    return c, snaps


@pytest.mark.parametrize("cname", BEACH_CASES)
def test_oracle_beaching_matches_reference(golden, cname):
    g = golden("golden_beach")
    c, snaps = replay_oracle_beach(g, cname)
    assert snaps
    for k, out in snaps.items():
        for name in ("status", "nearest_node", "failure_reason", "wet", "lon", "lat"):
            np.testing.assert_array_equal(out[name], c[f"s{k}_{name}"], err_msg=f"{cname} step {k} {name}")


def test_oracle_coastal_flags(golden):
    from kelp_b200.mesh import build_boundary_info
    g = golden("golden_beach")
    import types
    m = types.SimpleNamespace(elem_nodes=g.mesh.elem_nodes, nodes_lon=g.mesh.nodes_lon, _elem_is_coastal=None)
    build_boundary_info(m)
    np.testing.assert_array_equal(m._elem_is_coastal.astype(np.uint8), g.d["p_coastal"])


@pytest.mark.parametrize("fixture", ["golden_band", "golden_3d"])
def test_elem_neighbors_match_reference(golden, fixture):
    import types
    from kelp_b200.mesh import build_elem_neighbors
    g = golden(fixture)
    m = types.SimpleNamespace(elem_nodes=g.mesh.elem_nodes, nodes_lon=g.mesh.nodes_lon, _elem_neighbors=None)
    np.testing.assert_array_equal(build_elem_neighbors(m), g.d["mesh_elem_neighbors"])


@pytest.mark.parametrize("fixture", ["golden_cgrid2d", "golden_cgrid3d", "golden_cgrid_tripolar2d",
                                     "golden_cgrid_tripolar3d"])
def test_cgrid_mesh_builder_matches_reference(golden, fixture):
    """kelp_b200.nemo.build_cgrid_mesh on the recorded raster equals the
    reference's own build_nemo_cgrid_mesh: nodes, cells, ring, tables, grid
    hash; on the tripolar raster through the seam and the fold."""
    from kelp_b200.nemo import CgridLayout, build_cgrid_mesh
    g = golden(fixture)
    d = g.d
    kw = {}
    if "mesh_cgin_zw" in d:
        kw = dict(e2u=d["mesh_cgin_e2u"], e1v=d["mesh_cgin_e1v"], nlev2d=d["mesh_cgin_nlev"],
                  zw=d["mesh_cgin_zw"], area=d["mesh_cgin_area"], e3b=d["mesh_cgin_e3b"])
        if "mesh_cgin_e3u0" in d:
            kw["e3u0"] = d["mesh_cgin_e3u0"]
    if "mesh_cgin_fold" in d:
        kw["layout"] = CgridLayout(d["mesh_cgin_glamf"].shape, periodic=True, fold=str(d["mesh_cgin_fold"]))
    m = build_cgrid_mesh(d["mesh_cgin_glamf"], d["mesh_cgin_gphif"], d["mesh_cgin_wet"], **kw)
    for k in ("nodes_lon", "nodes_lat", "depth", "elem_nodes", "node_to_elems", "node_to_elems_count"):
        np.testing.assert_array_equal(np.asarray(getattr(m, k)), d[f"mesh_{k}"], err_msg=k)
    np.testing.assert_array_equal(m._gh_offsets, d["mesh_gh_offsets"])
    np.testing.assert_array_equal(m._gh_node_ids, d["mesh_gh_node_ids"])
    for k in ("corners", "elem_ji", "nlev", "nlev_raster", "zw", "area", "e3b", "kbu", "e3u", "kbv", "e3v",
              "e2u", "e1v"):
        np.testing.assert_array_equal(np.asarray(getattr(m, "_nemo_cgrid_" + k)).reshape(-1),
                                      d["mesh_cgrid_" + k].reshape(-1), err_msg=k)


def test_tripolar_raster_canonical_form_matches_reference(golden):
    """kelp_b200.nemo.to_canonical of face-velocity rasters equals the
    reference's nemo_cgrid_to_canonical (halo columns, the fold's half turn,
    the vector sign)."""
    from kelp_b200.nemo import CgridLayout, to_canonical
    d = golden("golden_cgrid_tripolar2d").d
    lay = CgridLayout(d["mesh_cgin_glamf"].shape, periodic=True, fold=str(d["mesh_cgin_fold"]))
    np.testing.assert_array_equal(to_canonical(d["mesh_cgin_raw_u"], lay, "U", vector=True), d["mesh_cgin_canon_u"])
    np.testing.assert_array_equal(to_canonical(d["mesh_cgin_raw_v"], lay, "V", vector=True), d["mesh_cgin_canon_v"])
