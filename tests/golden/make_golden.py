"""Generate the golden fixtures of tests/golden/ by running the REFERENCE.

This script imports KELP itself (its ``src`` tree, path given by
``KELP_REFERENCE_SRC``) and runs its own Numba step functions
(``kelp.numerics.integrators.rk2_step`` / ``rk4_step`` / ``euler_step``), its
``find_nearest_nodes`` and its counter RNG on small seeded synthetic inputs.
The inputs (mesh arrays, the reference-built grid hash and unit-sphere node
table, snapshots, particles) and the reference's outputs are written to
``tests/golden/*.npz``.  The fixtures pin the CPU oracle and, through it, the
CUDA kernels; nothing at test time imports the reference.

    KELP_REFERENCE_SRC=<kelp checkout>/src python tests/golden/make_golden.py
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
if "KELP_REFERENCE_SRC" not in os.environ:
    sys.exit("set KELP_REFERENCE_SRC to the src/ directory of a KELP checkout")
sys.path.insert(0, os.environ["KELP_REFERENCE_SRC"])

os.environ.setdefault("NUMBA_NUM_THREADS", "8")

from kelp.core.io import LazyLerpField as RLazy, VelocityField as RVel  # noqa: E402
from kelp.core.mesh import (Mesh as RMesh, build_node_to_elems as r_n2e, build_search,  # noqa: E402
                            find_containing_elements, find_nearest_nodes, set_exact_nearest, set_grid_hash_cell)
from kelp.core.particles import ParticleState as RState, ParticleStatus  # noqa: E402
from kelp.numerics import integrators as RI  # noqa: E402
from kelp.numerics.diffusion import DiffusionStepArgs as RDiff, _normal_pair  # noqa: E402
from kelp.core.config import BeachingConfig as RBeachCfg  # noqa: E402
from kelp.core.mesh import build_boundary_info as r_boundary  # noqa: E402
from kelp.numerics.beaching import BeachRunConfig as RBeachRun, _RESUSP_CODES  # noqa: E402
from kelp.tracking import _apply_beaching_hook  # noqa: E402

from kelp_b200 import synthetic as S  # noqa: E402  (input generators only)


def ref_mesh(m, cell=0.0, sigma=None):
    en = np.ascontiguousarray(m.elem_nodes, dtype=np.int32)
    n2e, cnt = r_n2e(m.n_nodes, en)
    rm = RMesh(name="golden", nodes_lon=np.array(m.nodes_lon), nodes_lat=np.array(m.nodes_lat),
               depth=np.array(m.depth), elem_nodes=en,
               elem_center_lon=np.array(m.elem_center_lon), elem_center_lat=np.array(m.elem_center_lat),
               node_to_elems=n2e, node_to_elems_count=cnt,
               sigma=np.zeros(0) if sigma is None else np.asarray(sigma, dtype=np.float64))
    build_search(rm)
    if cell > 0:
        set_grid_hash_cell(rm, cell)
    set_exact_nearest(rm, True)
    return rm


def mesh_record(rm):
    extra = {} if rm._elem_neighbors is None else {"elem_neighbors": rm._elem_neighbors}
    if rm.vertical_coord != "zlevel":
        extra["vertical_coord"] = np.array(rm.vertical_coord)
    return {**extra,"nodes_lon": rm.nodes_lon, "nodes_lat": rm.nodes_lat, "depth": rm.depth,
            "elem_nodes": rm.elem_nodes, "node_to_elems": rm.node_to_elems,
            "node_to_elems_count": rm.node_to_elems_count, "sigma": rm.sigma,
            "gh_offsets": rm._gh_offsets, "gh_node_ids": rm._gh_node_ids, "node_xyz": rm._node_xyz,
            "gh_geom": np.array([rm._gh_cell_size, rm._gh_lon_min, rm._gh_lat_min, rm._gh_nx, rm._gh_ny,
                                 int(rm._gh_wrap_lon), rm._gh_far_rows, rm.r_earth], dtype=np.float64)}


def ref_fields(snaps, placement="layer"):
    return [RVel(u=s.u, v=s.v, w=s.w, eta=np.asarray(s.eta), uv_layout="node",
                 uv_vertical=placement, az=getattr(s, "az", None), scalars=getattr(s, "scalars", None))
            for s in snaps]


def payload(fields, t, T):
    """_build_vel_payload (tracking.py:3136-3206), forward, snapshots T apart."""
    ia = int(np.floor(t / T + 1e-9))
    ta = ia * T
    a, b = fields[ia], fields[ia + 1]
    alpha = (t - ta) / T
    vel = a if abs(alpha) < 1e-12 else (b if abs(alpha - 1.0) < 1e-12 else RLazy(a, b, alpha))
    return vel, b, (ta + T) - t, ia, alpha


def run_case(rm, fields, lon, lat, z, status, scheme, dt, T, n_steps, *, time_dir=1.0, w_interp="nearest",
             kh=None, seed=7, real_id=0, pid_offset=0, record=(1,), az=None, walk=False, steady=False,
             uv_interp="barycentric", pchip=False, t0=0.0, surfaces=None, edge_bc=None):
    fn = {"rk2": RI.rk2_step, "rk4": RI.rk4_step, "euler": RI.euler_step}[scheme]
    P = lon.size
    st = RState(lon=lon.copy(), lat=lat.copy(), z=z.copy(), status=status.copy(),
                nearest_node=np.full(P, -1, np.int32), failure_reason=np.zeros(P, np.int8))
    out = {}
    if walk:
        # elem_search: walk seeds the carried elements with one global
        # search (tracking.py:2243-2250)
        el0, _ = find_containing_elements(rm, st.lon, st.lat, find_nearest_nodes(rm, st.lon, st.lat))
        st = st.replace(elem=el0.astype(np.int32))
        out["elem0"] = np.asarray(st.elem).copy()
    sched = []
    for k in range(n_steps):
        t = t0 + k * dt
        vel, vnext, dtn, ia, alpha = payload(fields, t, T)
        if steady:   # no time-aware payload: every stage reads the first record
            vel, vnext, dtn, ia, alpha = fields[0], None, -1.0, 0, 0.0
        kw = dict(uv_interp=uv_interp, w_interp=w_interp, vel_next=vnext,
                  dt_to_next=None if steady else dtn)
        if edge_bc is not None:
            kw["edge_leastsq_bc"] = edge_bc
        if kh is not None:
            kw["diffusion"] = RDiff(scheme="uniform", kh_x=kh[0], kh_y=kh[1], seed=seed, real_id=real_id,
                                    step_i=k, pid_offset=pid_offset, **(az or {}))
        has_recon = 0
        if pchip and scheme != "euler" and abs(alpha) >= 1e-12 and 1 <= ia and ia + 2 < len(fields):
            # tracking._resolve_recon_stencil: (ia-1, ia, ia+1, ia+2) around the bracket
            idx = (ia - 1, ia, ia + 1, ia + 2)
            kw["recon"] = ([fields[i] for i in idx], [float(i * T) for i in idx], t, float(time_dir))
            has_recon = 1
        sched.append([ia, alpha, dtn, has_recon, t])
        if surfaces is not None:   # the tracking layer's sigma surfaces at the step's start and end
            es, ee = surfaces(t, t + dt * time_dir)
            for key, e in (("sigma_eta_start", es), ("sigma_eta_end", ee)):
                if e is not None:
                    kw[key] = e
                    out.setdefault(key, []).append(e)
        st = fn(st, vel, rm, dt, time_dir, **kw)
        if (k + 1) in record or k + 1 == n_steps:
            tag = f"s{k + 1}"
            for name in ("lon", "lat", "z", "status", "nearest_node", "failure_reason", "u", "v"):
                out[f"{tag}_{name}"] = np.asarray(getattr(st, name))
            if st.w is not None:
                out[f"{tag}_w"] = np.asarray(st.w)
            if st.elem is not None:
                out[f"{tag}_elem"] = np.asarray(st.elem)
    for key in ("sigma_eta_start", "sigma_eta_end"):
        if key in out:
            out[key] = np.array(out[key])
    out["schedule"] = np.array(sched, dtype=np.float64)
    out["params"] = np.array([dt, T, n_steps, time_dir, -1 if kh is None else kh[0], -1 if kh is None else kh[1],
                              seed, real_id, pid_offset], dtype=np.float64)
    if az:
        out["az"] = np.array([float(az.get("az_const", 0.0)), float(az.get("az_requires_field", False))])
    return out


def run_beach_case(rm, fields, lon, lat, z, status, dt, T, n_steps, beach, *, kh=(5.0e4, 5.0e4), seed=7,
                   real_id=0, pid_offset=0, record=(1, 2, 4, 8, 12, 16)):
    """RK2 + split kick steps, each followed by the reference's beaching hook
    (tracking.py:2616-2672): prev_status is the status at the step's entry."""
    P = lon.size
    cfg = RBeachCfg(enabled=True, **beach)
    crit = frozenset(cfg.criteria)
    need_topo = bool({"coastal_element", "stochastic"} & crit)
    coastal = None
    if need_topo:
        r_boundary(rm)
        coastal = rm._elem_is_coastal
    bseed = cfg.seed if cfg.seed is not None else seed
    zone = cfg.zone_depth if cfg.zone_depth is not None else 2.0 * cfg.depth_min
    run_cfg = RBeachRun(cfg=cfg, crit=crit, need_topo=need_topo, elem_coastal=coastal, seed=bseed, zone=zone,
                        pid_offset=pid_offset)
    st = RState(lon=lon.copy(), lat=lat.copy(), z=z.copy(), status=status.copy(),
                nearest_node=np.full(P, -1, np.int32), failure_reason=np.zeros(P, np.int8))
    wet = np.zeros(P, np.int32)
    out = {}
    sched = []
    for k in range(n_steps):
        t = k * dt
        vel, vnext, dtn, ia, alpha = payload(fields, t, T)
        kw = dict(uv_interp="barycentric", vel_next=vnext, dt_to_next=dtn)
        if kh is not None:
            kw["diffusion"] = RDiff(scheme="uniform", kh_x=kh[0], kh_y=kh[1], seed=seed, real_id=real_id,
                                    step_i=k, pid_offset=pid_offset)
        sched.append([ia, alpha, dtn])
        prev = st.status
        st = RI.rk2_step(st, vel, rm, dt, 1.0, **kw)
        st, wet = _apply_beaching_hook(st, prev, rm, vel, run_cfg, wet, real_id, k, dt)
        if (k + 1) in record or k + 1 == n_steps:
            tag = f"s{k + 1}"
            for name in ("lon", "lat", "status", "nearest_node", "failure_reason"):
                out[f"{tag}_{name}"] = np.asarray(getattr(st, name))
            out[f"{tag}_wet"] = np.asarray(wet)
    out["schedule"] = np.array(sched, dtype=np.float64)
    out["params"] = np.array([dt, T, n_steps, 1.0, -1 if kh is None else kh[0], -1 if kh is None else kh[1],
                              seed, real_id, pid_offset], dtype=np.float64)
    c = set(cfg.criteria)
    out["beach"] = np.array([int("depth" in c), int("coastal_element" in c), int("stochastic" in c),
                             int("on_failure" in c), _RESUSP_CODES[cfg.resuspension], cfg.min_wet_steps,
                             cfg.depth_min, zone, cfg.rewet_hysteresis, cfg.t_beach or 0.0,
                             cfg.t_resuspend or 0.0, bseed, int(bool(cfg.use_eta)),
                             int(bool(cfg.dry_mask_var))], dtype=np.float64)
    n_beached = int((st.status == int(ParticleStatus.BEACHED)).sum())
    print(f"  beach case: {n_beached} beached at the end, {int((wet > 0).sum())} wet streaks")
    return out


def beach_fixture():
    """A regional coast with shallow shelves: particles strand, remap on
    failure and resuspend under every criterion."""
    T = 86400.0
    m = S.lattice_mesh(1.0, 20.0, lon_min=-25.0, lon_max=25.0, jitter=0.15, land_frac=0.3, quad_frac=0.25,
                       depth=lambda lo, la: S.smooth_bathymetry(lo, la, 0.0, 6.0, seed=8))
    rm = ref_mesh(m)
    snaps = S.gyre_snapshots(m, 4, amp=1.5, dtype=np.float64)
    # a free surface that floods and drains the shelves (use_eta) and a dry
    # mask scalar (dry_mask_var), both moving between the daily records
    lo, la = np.asarray(m.nodes_lon), np.asarray(m.nodes_lat)
    for i, sn in enumerate(snaps):
        sn.eta = 1.2 * np.sin(np.radians(9.0 * lo + 40.0 * i)) * np.cos(np.radians(7.0 * la - 25.0 * i))
        dry = ((np.asarray(m.depth) + sn.eta) < 0.9) | (np.sin(np.radians(23.0 * lo + 31.0 * la + 50.0 * i)) > 0.93)
        sn.scalars = {"dry": dry.astype(np.float64)}
    rf = ref_fields(snaps)
    lon, lat, z, status = particles(m, 1500, 31, n_dead=20)
    cases = {
        "dco_auto": run_beach_case(rm, rf, lon, lat, z, status, 10800.0, T, 16,
                                   dict(criteria=["depth", "coastal_element", "on_failure"], depth_min=1.0,
                                        resuspension="auto", min_wet_steps=2, rewet_hysteresis=0.5)),
        "sto_both": run_beach_case(rm, rf, lon, lat, z, status, 10800.0, T, 16,
                                   dict(criteria=["stochastic", "on_failure"], depth_min=1.0, zone_depth=3.0,
                                        t_beach=43200.0, resuspension="auto_or_stochastic", t_resuspend=21600.0,
                                        min_wet_steps=3, seed=99),
                                   real_id=2, pid_offset=500),
        "cd_sresusp": run_beach_case(rm, rf, lon, lat, z, status, 10800.0, T, 16,
                                     dict(criteria=["coastal_element", "depth"], depth_min=0.5,
                                          resuspension="stochastic", t_resuspend=10800.0, rewet_hysteresis=0.2),
                                     kh=(2.0e4, 2.0e4)),
        "depth_never": run_beach_case(rm, rf, lon, lat, z, status, 10800.0, T, 12,
                                      dict(criteria=["depth"], depth_min=2.0), kh=None),
        "eta_dry_auto": run_beach_case(rm, rf, lon, lat, z, status, 10800.0, T, 16,
                                       dict(criteria=["depth", "on_failure"], depth_min=1.0, use_eta=True,
                                            dry_mask_var="dry", resuspension="auto", min_wet_steps=2,
                                            rewet_hysteresis=0.3)),
        "eta_sto_both": run_beach_case(rm, rf, lon, lat, z, status, 10800.0, T, 16,
                                       dict(criteria=["stochastic", "depth"], depth_min=0.8, zone_depth=3.0,
                                            t_beach=43200.0, use_eta=True, dry_mask_var="dry",
                                            resuspension="auto_or_stochastic", t_resuspend=21600.0,
                                            min_wet_steps=2, seed=5),
                                       real_id=1, pid_offset=300),
    }
    r_boundary(rm)
    save("golden_beach", mesh_record(rm), snaps, cases,
         {"lon": lon, "lat": lat, "z": z, "status": status, "coastal": rm._elem_is_coastal.astype(np.uint8)})


def particles(m, P, seed, z=False, n_off=0, n_dead=0):
    lon, lat, zz = S.release_uniform(m, P, seed=seed, depth_uniform=z)
    status = np.full(P, int(ParticleStatus.ALIVE), np.int32)
    rng = np.random.default_rng(seed + 100)
    if n_off:
        idx = rng.choice(P, n_off, replace=False)
        lat[idx] = rng.uniform(-89, 89, n_off)          # many land up on land / outside
        lon[idx] = rng.uniform(-180, 180, n_off)
    if n_dead:
        idx = rng.choice(P, n_dead, replace=False)
        status[idx[: n_dead // 2]] = int(ParticleStatus.OUTSIDE)
        status[idx[n_dead // 2:]] = int(ParticleStatus.NOT_RELEASED)
    return lon, lat, zz, status


def save(name, mesh_rec, snaps, cases, parts):
    d = {}
    for k, v in mesh_rec.items():
        d[f"mesh_{k}"] = v
    for i, s in enumerate(snaps):
        d[f"snap{i}_u"] = s.u
        d[f"snap{i}_v"] = s.v
        if s.w is not None:
            d[f"snap{i}_w"] = s.w
        if getattr(s, "az", None) is not None:
            d[f"snap{i}_az"] = s.az
        if np.any(np.asarray(s.eta) != 0):
            d[f"snap{i}_eta"] = s.eta
        for k, v in (getattr(s, "scalars", None) or {}).items():
            d[f"snap{i}_scalar_{k}"] = v
    for k, v in parts.items():
        d[f"p_{k}"] = v
    for cname, c in cases.items():
        for k, v in c.items():
            d[f"{cname}__{k}"] = v
    path = os.path.join(HERE, f"{name}.npz")
    np.savez_compressed(path, **d)
    print(name, os.path.getsize(path) // 1024, "KB", sorted(cases))


def main():
    T = 86400.0
    # --- global band (seam wrap), jitter, land mask, triangles --------------
    m = S.lattice_mesh(3.0, 72.0, jitter=0.2, land_frac=0.3)
    rm = ref_mesh(m)
    snaps = S.gyre_snapshots(m, 4, amp=1.5)
    rf = ref_fields(snaps)
    lon, lat, z, status = particles(m, 1500, 11, n_off=60, n_dead=40)
    cases = {}
    cases["rk2"] = run_case(rm, rf, lon, lat, z, status, "rk2", 21600.0, T, 12)
    cases["rk4"] = run_case(rm, rf, lon, lat, z, status, "rk4", 21600.0, T, 12)
    cases["euler"] = run_case(rm, rf, lon, lat, z, status, "euler", 21600.0, T, 12)
    cases["rk2_bwd"] = run_case(rm, rf, lon, lat, z, status, "rk2", 21600.0, T, 12, time_dir=-1.0)
    cases["rk2_kick"] = run_case(rm, rf, lon, lat, z, status, "rk2", 21600.0, T, 12, kh=(5.0e4, 5.0e4),
                                 seed=7, real_id=3, pid_offset=1000)
    cases["rk4_kick_aniso"] = run_case(rm, rf, lon, lat, z, status, "rk4", 21600.0, T, 8, kh=(8.0e4, 2.0e4),
                                       seed=11, real_id=0)
    cases["rk2_dt4800"] = run_case(rm, rf, lon, lat, z, status, "rk2", 4800.0, T, 20)
    # elem_search: walk (carried elements, edge walk with global fallbacks)
    cases["rk2_walk"] = run_case(rm, rf, lon, lat, z, status, "rk2", 21600.0, T, 12, walk=True, record=(1, 6))
    cases["rk4_walk_kick"] = run_case(rm, rf, lon, lat, z, status, "rk4", 21600.0, T, 8, kh=(5.0e4, 5.0e4),
                                      seed=3, walk=True)
    cases["euler_walk"] = run_case(rm, rf, lon, lat, z, status, "euler", 10800.0, T, 12, walk=True)
    nn_q = find_nearest_nodes(rm, lon, lat)
    save("golden_band", mesh_record(rm), snaps, cases,
         {"lon": lon, "lat": lat, "z": z, "status": status, "nearest_exact": nn_q})

    # --- regional mixed tri/quad mesh (no wrap), float64 fields -------------
    m = S.lattice_mesh(1.0, 15.0, lon_min=-20.0, lon_max=20.0, jitter=0.15, land_frac=0.2, quad_frac=0.3)
    rm = ref_mesh(m)
    snaps = S.gyre_snapshots(m, 4, amp=2.0, dtype=np.float64)
    rf = ref_fields(snaps)
    lon, lat, z, status = particles(m, 1200, 12, n_dead=20)
    cases = {"rk2": run_case(rm, rf, lon, lat, z, status, "rk2", 10800.0, T, 16),
             "rk4": run_case(rm, rf, lon, lat, z, status, "rk4", 10800.0, T, 16),
             "euler": run_case(rm, rf, lon, lat, z, status, "euler", 10800.0, T, 16),
             "rk2_kick": run_case(rm, rf, lon, lat, z, status, "rk2", 10800.0, T, 16, kh=(2.0e4, 2.0e4))}
    q_lon = np.random.default_rng(5).uniform(-60, 60, 3000)
    q_lat = np.random.default_rng(6).uniform(-60, 60, 3000)
    save("golden_quad", mesh_record(rm), snaps, cases,
         {"lon": lon, "lat": lat, "z": z, "status": status, "q_lon": q_lon, "q_lat": q_lat,
          "q_nearest": find_nearest_nodes(rm, q_lon, q_lat)})

    # --- polar cap: anisotropic cells force the widened exact search --------
    m = S.lattice_mesh(2.0, 88.0, jitter=0.1, land_frac=0.0, cell_size=0.5)
    rm = ref_mesh(m, cell=0.5)
    q_lon = np.random.default_rng(7).uniform(-180, 180, 4000)
    q_lat = np.concatenate([np.random.default_rng(8).uniform(70, 89.9, 2000),
                            np.random.default_rng(9).uniform(-89.9, 89.9, 2000)])
    snaps = S.gyre_snapshots(m, 3, amp=1.0)
    rf = ref_fields(snaps)
    lon = np.random.default_rng(10).uniform(-180, 180, 800)
    lat = np.random.default_rng(11).uniform(60, 87.5, 800)
    z = np.zeros(800)
    status = np.full(800, 1, np.int32)
    cases = {"rk2": run_case(rm, rf, lon, lat, z, status, "rk2", 21600.0, T, 6)}
    save("golden_polar", mesh_record(rm), snaps, cases,
         {"lon": lon, "lat": lat, "z": z, "status": status, "q_lon": q_lon, "q_lat": q_lat,
          "q_nearest": find_nearest_nodes(rm, q_lon, q_lat)})

    # --- 3-D z-level band: layer u/v, W nearest / barycentric, kick ---------
    zl = S.stretched_levels(12, 5.0, 4000.0)
    m = S.lattice_mesh(3.0, 60.0, jitter=0.2, land_frac=0.25,
                       depth=lambda lo, la: S.smooth_bathymetry(lo, la, 30.0, 4000.0), sigma=zl)
    rm = ref_mesh(m, sigma=zl)
    snaps = S.gyre_snapshots(m, 4, amp=1.5, z_levels=zl, decay=800.0, w_scale=2e-3)
    for k, sn in enumerate(snaps):   # a vertical diffusivity on the interfaces (K, N) for the Az kick
        sn.az = ((1e-2 * (1.0 + 0.2 * k)) * np.exp(-np.asarray(zl)[:, None] / 300.0)
                 * (1.0 + 0.5 * np.sin(np.radians(3.0 * np.asarray(m.nodes_lon))))[None, :] + 1e-4).astype(np.float32)
    rf = ref_fields(snaps)
    lon, lat, z, status = particles(m, 1200, 13, z=True, n_dead=20)
    cases = {"rk2_wnear": run_case(rm, rf, lon, lat, z, status, "rk2", 21600.0, T, 12, w_interp="nearest"),
             "rk2_wbary": run_case(rm, rf, lon, lat, z, status, "rk2", 21600.0, T, 12, w_interp="barycentric"),
             "rk2_wbary_kick": run_case(rm, rf, lon, lat, z, status, "rk2", 21600.0, T, 12,
                                        w_interp="barycentric", kh=(3.0e4, 3.0e4), seed=5),
             # unfused reference paths: 3-D RK4 and 3-D Euler
             "rk4_wnear": run_case(rm, rf, lon, lat, z, status, "rk4", 21600.0, T, 12, w_interp="nearest"),
             "rk4_wbary_kick": run_case(rm, rf, lon, lat, z, status, "rk4", 21600.0, T, 12,
                                        w_interp="barycentric", kh=(3.0e4, 1.0e4), seed=9),
             "euler_wbary": run_case(rm, rf, lon, lat, z, status, "euler", 10800.0, T, 16, w_interp="barycentric"),
             # the vertical Az kick: the snapshots' Az field with the split
             # horizontal kick, and a constant Az alone (Kh = 0)
             "rk2_wbary_kick_azf": run_case(rm, rf, lon, lat, z, status, "rk2", 21600.0, T, 12,
                                            w_interp="barycentric", kh=(3.0e4, 3.0e4), seed=6,
                                            az=dict(az_enabled=True, az_requires_field=True)),
             "rk4_wnear_azf_nokh": run_case(rm, rf, lon, lat, z, status, "rk4", 21600.0, T, 10,
                                            w_interp="nearest", kh=(0.0, 0.0), seed=8,
                                            az=dict(az_enabled=True, az_const=5e-3)),
             "rk2_wbary_walk": run_case(rm, rf, lon, lat, z, status, "rk2", 21600.0, T, 12,
                                        w_interp="barycentric", walk=True),
             "rk4_wnear_walk_kick": run_case(rm, rf, lon, lat, z, status, "rk4", 21600.0, T, 10,
                                             w_interp="nearest", kh=(3.0e4, 3.0e4), seed=2, walk=True)}
    save("golden_3d", mesh_record(rm), snaps, cases, {"lon": lon, "lat": lat, "z": z, "status": status})

    # --- depth-linear u/v (uv_vertical level / layer_linear) on the same mesh;
    # a fifth of the particles start below their shallowest vertex (walls)
    zdl = z.copy()
    deep = np.random.default_rng(21).uniform(size=zdl.size) < 0.2
    zdl[deep] *= 1.6
    cases = {}
    for placement, tag in (("level", "lev"), ("layer_linear", "llin")):
        sn = S.gyre_snapshots(m, 4, amp=1.5, z_levels=zl, decay=800.0, w_scale=2e-3, placement=placement)
        rfp = [RVel(u=s.u, v=s.v, w=s.w, eta=np.zeros(s.u.shape[-1]), uv_layout="node", uv_vertical=placement)
               for s in sn]
        cases[f"rk2_{tag}_wbary"] = run_case(rm, rfp, lon, lat, zdl, status, "rk2", 21600.0, T, 12,
                                             w_interp="barycentric")
        cases[f"rk4_{tag}_wnear_kick"] = run_case(rm, rfp, lon, lat, zdl, status, "rk4", 21600.0, T, 10,
                                                  w_interp="nearest", kh=(2.0e4, 2.0e4), seed=4)
        cases[f"euler_{tag}_wnear"] = run_case(rm, rfp, lon, lat, zdl, status, "euler", 10800.0, T, 8,
                                               w_interp="nearest")
        if tag == "lev":   # snapshots without Az: the constant source
            cases["rk2_lev_wbary_azc"] = run_case(rm, rfp, lon, lat, zdl, status, "rk2", 21600.0, T, 10,
                                                  w_interp="barycentric", kh=(2.0e4, 2.0e4), seed=3,
                                                  az=dict(az_enabled=True, az_const=2e-3))
        save(f"golden_dl_{tag}", mesh_record(rm), sn, {k: v for k, v in cases.items() if f"_{tag}_" in k},
             {"lon": lon, "lat": lat, "z": zdl, "status": status})

    # --- counter RNG: normal pairs of the reference for a key grid ----------
    keys = []
    vals = []
    rng = np.random.default_rng(0)
    for _ in range(4000):
        k = (int(rng.integers(0, 2**63)), int(rng.integers(0, 64)), int(rng.integers(0, 2**40)),
             int(rng.integers(0, 100000)), int(rng.integers(0, 2)))
        keys.append(k)
        vals.append(_normal_pair(*(np.uint64(x) for x in k)))
    np.savez_compressed(os.path.join(HERE, "golden_rng.npz"), keys=np.array(keys, dtype=np.uint64),
                        normals=np.array(vals, dtype=np.float64))
    print("golden_rng")


def sigma_fixture():
    """FESOM-C-style sigma meshes (mesh.vertical_coord "sigma"): a regional
    mixed tri/quad shelf, 0.2-120 m deep, 11 sigma interfaces, a free surface
    eta that changes from record to record (some columns fall below Dmin),
    layer and layer_linear u/v, the dia-sigma W on the interfaces."""
    T = 21600.0
    sig = np.array([1.0, 0.95, 0.88, 0.8, 0.7, 0.58, 0.45, 0.32, 0.2, 0.1, 0.0])
    m = S.lattice_mesh(1.0, 15.0, lon_min=-20.0, lon_max=20.0, jitter=0.15, land_frac=0.2, quad_frac=0.3,
                       depth=lambda lo, la: S.smooth_bathymetry(lo, la, 0.2, 120.0), sigma=sig)
    rm = ref_mesh(m, sigma=sig)
    rm.vertical_coord = "sigma"
    lon_n, lat_n = np.radians(np.asarray(m.nodes_lon)), np.radians(np.asarray(m.nodes_lat))
    pseudo = (1.0 - sig) * 100.0   # depth scale of the synthetic vertical structure
    lon, lat, z, status = particles(m, 1200, 31, z=True, n_dead=20)
    for placement, tag in (("layer", "sigma"), ("layer_linear", "sigma_llin")):
        snaps = S.gyre_snapshots(m, 6, amp=1.0, z_levels=pseudo, decay=60.0, w_scale=4e-4, placement=placement)
        for k, sn in enumerate(snaps):
            sn.eta = (0.6 * np.sin(2.0 * lon_n + 0.9 * k) * np.cos(3.0 * lat_n) - 0.15).astype(np.float32)
        rf = ref_fields(snaps, placement)
        if placement == "layer":
            cases = {"rk2_wnear": run_case(rm, rf, lon, lat, z, status, "rk2", 3600.0, T, 12, w_interp="nearest"),
                     "rk2_wbary": run_case(rm, rf, lon, lat, z, status, "rk2", 3600.0, T, 12,
                                           w_interp="barycentric"),
                     "rk4_wbary": run_case(rm, rf, lon, lat, z, status, "rk4", 3600.0, T, 12,
                                           w_interp="barycentric"),
                     "euler_wbary": run_case(rm, rf, lon, lat, z, status, "euler", 1800.0, T, 16,
                                             w_interp="barycentric"),
                     "euler_wnear": run_case(rm, rf, lon, lat, z, status, "euler", 1800.0, T, 16,
                                             w_interp="nearest"),
                     "rk2_wbary_kick": run_case(rm, rf, lon, lat, z, status, "rk2", 3600.0, T, 12,
                                                w_interp="barycentric", kh=(20.0, 20.0), seed=5),
                     "rk4_wnear_kick": run_case(rm, rf, lon, lat, z, status, "rk4", 3600.0, T, 10,
                                                w_interp="nearest", kh=(30.0, 10.0), seed=9),
                     "rk2_wnear_bwd": run_case(rm, rf, lon, lat, z, status, "rk2", 3600.0, T, 12,
                                               w_interp="nearest", time_dir=-1.0),
                     "rk2_wbary_steady": run_case(rm, rf, lon, lat, z, status, "rk2", 3600.0, T, 8,
                                                  w_interp="barycentric", steady=True),
                     "rk4_wnear_steady": run_case(rm, rf, lon, lat, z, status, "rk4", 3600.0, T, 8,
                                                  w_interp="nearest", steady=True),
                     "rk2_wbary_walk": run_case(rm, rf, lon, lat, z, status, "rk2", 3600.0, T, 12,
                                                w_interp="barycentric", walk=True)}
        else:
            cases = {"rk2_llin_wbary": run_case(rm, rf, lon, lat, z, status, "rk2", 3600.0, T, 12,
                                                w_interp="barycentric"),
                     "rk4_llin_wnear_kick": run_case(rm, rf, lon, lat, z, status, "rk4", 3600.0, T, 10,
                                                     w_interp="nearest", kh=(20.0, 20.0), seed=4),
                     "euler_llin_wnear": run_case(rm, rf, lon, lat, z, status, "euler", 1800.0, T, 12,
                                                  w_interp="nearest")}
        save(f"golden_{tag}", mesh_record(rm), snaps, cases, {"lon": lon, "lat": lat, "z": z, "status": status})


def sigma_surf_fixture():
    """The tracking layer's surfaces on sigma steps (sigma_eta_start /
    sigma_eta_end of the step functions, integrators.py:1358-1441, supplied
    per step by tracking.py:2562-2596): on the sigma shelf of golden_sigma,
    each step gets the surfaces of a smooth function of time (not the
    payload's own) at its start and end -- time-aware RK2 / RK4 / Euler, steady
    steps whose stages blend from the start to the end surface, the end
    surface alone (the discrete mode), the start alone, and the split kick.
    tests/golden/golden_sigma_surf.npz."""
    T = 21600.0
    sig = np.array([1.0, 0.95, 0.88, 0.8, 0.7, 0.58, 0.45, 0.32, 0.2, 0.1, 0.0])
    m = S.lattice_mesh(1.0, 15.0, lon_min=-20.0, lon_max=20.0, jitter=0.15, land_frac=0.2, quad_frac=0.3,
                       depth=lambda lo, la: S.smooth_bathymetry(lo, la, 0.2, 120.0), sigma=sig)
    rm = ref_mesh(m, sigma=sig)
    rm.vertical_coord = "sigma"
    lon_n, lat_n = np.radians(np.asarray(m.nodes_lon)), np.radians(np.asarray(m.nodes_lat))
    pseudo = (1.0 - sig) * 100.0
    lon, lat, z, status = particles(m, 1200, 37, z=True, n_dead=20)
    snaps = S.gyre_snapshots(m, 6, amp=1.0, z_levels=pseudo, decay=60.0, w_scale=4e-4, placement="layer")
    for k, sn in enumerate(snaps):
        sn.eta = (0.6 * np.sin(2.0 * lon_n + 0.9 * k) * np.cos(3.0 * lat_n) - 0.15).astype(np.float32)
    rf = ref_fields(snaps)

    def surf(t):
        return 0.5 * np.sin(2.0 * lon_n + 2.0e-4 * t) * np.cos(3.0 * lat_n) - 0.1 + 0.3 * np.cos(lat_n + 1.0e-4 * t)

    both = lambda t0, t1: (surf(t0), surf(t1))
    cases = {"rk2_wbary_surf": run_case(rm, rf, lon, lat, z, status, "rk2", 3600.0, T, 10, w_interp="barycentric",
                                        surfaces=both),
             "rk4_wnear_surf": run_case(rm, rf, lon, lat, z, status, "rk4", 3600.0, T, 10, w_interp="nearest",
                                        surfaces=both),
             "euler_wbary_surf": run_case(rm, rf, lon, lat, z, status, "euler", 1800.0, T, 12,
                                          w_interp="barycentric", surfaces=both),
             "rk2_wbary_steady_surf": run_case(rm, rf, lon, lat, z, status, "rk2", 3600.0, T, 8,
                                               w_interp="barycentric", steady=True, surfaces=both),
             "rk4_wnear_steady_surf_kick": run_case(rm, rf, lon, lat, z, status, "rk4", 3600.0, T, 8,
                                                    w_interp="nearest", steady=True, kh=(20.0, 20.0), seed=3,
                                                    surfaces=both),
             "rk4_wbary_steady_endonly": run_case(rm, rf, lon, lat, z, status, "rk4", 3600.0, T, 8,
                                                  w_interp="barycentric", steady=True,
                                                  surfaces=lambda t0, t1: (None, surf(t1))),
             "rk2_wnear_startonly_kick": run_case(rm, rf, lon, lat, z, status, "rk2", 3600.0, T, 10,
                                                  w_interp="nearest", kh=(30.0, 10.0), seed=8,
                                                  surfaces=lambda t0, t1: (surf(t0), None))}
    save("golden_sigma_surf", mesh_record(rm), snaps, cases, {"lon": lon, "lat": lat, "z": z, "status": status})


def sigma_az_fixture():
    """The vertical Az kick on sigma meshes (integrators.py:917-930,
    diffusion.py:458-482 _loop_az_kick_sigma: the constant source, folded
    into the particle's end-of-step column): on the sigma shelf of
    golden_sigma_surf, Az alone and with the horizontal split kick, RK2 / RK4
    / Euler, forward and backward, with and without the tracking layer's
    surfaces.  tests/golden/golden_sigma_az.npz."""
    T = 21600.0
    sig = np.array([1.0, 0.95, 0.88, 0.8, 0.7, 0.58, 0.45, 0.32, 0.2, 0.1, 0.0])
    m = S.lattice_mesh(1.0, 15.0, lon_min=-20.0, lon_max=20.0, jitter=0.15, land_frac=0.2, quad_frac=0.3,
                       depth=lambda lo, la: S.smooth_bathymetry(lo, la, 0.2, 120.0), sigma=sig)
    rm = ref_mesh(m, sigma=sig)
    rm.vertical_coord = "sigma"
    lon_n, lat_n = np.radians(np.asarray(m.nodes_lon)), np.radians(np.asarray(m.nodes_lat))
    pseudo = (1.0 - sig) * 100.0
    lon, lat, z, status = particles(m, 1200, 39, z=True, n_dead=20)
    snaps = S.gyre_snapshots(m, 6, amp=1.0, z_levels=pseudo, decay=60.0, w_scale=4e-4, placement="layer")
    for k, sn in enumerate(snaps):
        sn.eta = (0.6 * np.sin(2.0 * lon_n + 0.9 * k) * np.cos(3.0 * lat_n) - 0.15).astype(np.float32)
    rf = ref_fields(snaps)

    def surf(t):
        return 0.5 * np.sin(2.0 * lon_n + 2.0e-4 * t) * np.cos(3.0 * lat_n) - 0.1 + 0.3 * np.cos(lat_n + 1.0e-4 * t)

    azc = dict(az_enabled=True, az_const=2e-3)
    cases = {"rk2_wbary_azc": run_case(rm, rf, lon, lat, z, status, "rk2", 3600.0, T, 10, w_interp="barycentric",
                                       kh=(0.0, 0.0), seed=4, az=azc),
             "rk4_wnear_kick_azc": run_case(rm, rf, lon, lat, z, status, "rk4", 3600.0, T, 10, w_interp="nearest",
                                            kh=(20.0, 20.0), seed=6, az=azc),
             "euler_wbary_azc": run_case(rm, rf, lon, lat, z, status, "euler", 1800.0, T, 12,
                                         w_interp="barycentric", kh=(0.0, 0.0), seed=2, az=azc),
             "rk2_wnear_bwd_kick_azc": run_case(rm, rf, lon, lat, z, status, "rk2", 3600.0, T, 10,
                                                w_interp="nearest", kh=(30.0, 10.0), seed=7, az=azc,
                                                time_dir=-1.0),
             "rk2_wbary_surf_kick_azc": run_case(rm, rf, lon, lat, z, status, "rk2", 3600.0, T, 10,
                                                 w_interp="barycentric", kh=(20.0, 20.0), seed=9, az=azc,
                                                 surfaces=lambda t0, t1: (surf(t0), surf(t1)))}
    save("golden_sigma_az", mesh_record(rm), snaps, cases, {"lon": lon, "lat": lat, "z": z, "status": status})


def wring_fixture():
    """W by least squares (the reference's default w_interp,
    vertical.py:493-601) and by inverse distance (:1148-1229) on the 3-D
    z-level mesh of golden_3d, through the reference's unfused steps: RK2,
    RK4, Euler, the split kick, backward time, depth-linear u/v.
    tests/golden/golden_wring.npz."""
    T = 86400.0
    zl = S.stretched_levels(12, 5.0, 4000.0)
    m = S.lattice_mesh(3.0, 60.0, jitter=0.2, land_frac=0.25,
                       depth=lambda lo, la: S.smooth_bathymetry(lo, la, 30.0, 4000.0), sigma=zl)
    rm = ref_mesh(m, sigma=zl)
    snaps = S.gyre_snapshots(m, 4, amp=1.5, z_levels=zl, decay=800.0, w_scale=2e-3)
    rf = ref_fields(snaps)
    lon, lat, z, status = particles(m, 1200, 47, z=True, n_dead=20)
    cases = {"rk2_wlsq": run_case(rm, rf, lon, lat, z, status, "rk2", 21600.0, T, 10, w_interp="leastsq"),
             "rk4_wlsq_kick": run_case(rm, rf, lon, lat, z, status, "rk4", 21600.0, T, 10, w_interp="leastsq",
                                       kh=(3.0e4, 3.0e4), seed=5),
             "euler_wlsq": run_case(rm, rf, lon, lat, z, status, "euler", 10800.0, T, 12, w_interp="leastsq"),
             "rk2_wlsq_bwd": run_case(rm, rf, lon, lat, z, status, "rk2", 21600.0, T, 10, w_interp="leastsq",
                                      time_dir=-1.0),
             "rk2_widw": run_case(rm, rf, lon, lat, z, status, "rk2", 21600.0, T, 10, w_interp="idw"),
             "rk4_widw_kick": run_case(rm, rf, lon, lat, z, status, "rk4", 21600.0, T, 10, w_interp="idw",
                                       kh=(3.0e4, 1.0e4), seed=9)}
    save("golden_wring", mesh_record(rm), snaps, cases, {"lon": lon, "lat": lat, "z": z, "status": status})


def sigma_wring_fixture():
    """W (and the particle's column height) by least squares and by inverse
    distance on sigma meshes (vertical_sigma.py:493-563, :656-905): on the
    sigma shelf of golden_sigma_surf, RK2 / RK4 / Euler, the split kick,
    backward time, the tracking layer's surfaces, depth-linear u/v.
    tests/golden/golden_sigma_wring.npz."""
    T = 21600.0
    sig = np.array([1.0, 0.95, 0.88, 0.8, 0.7, 0.58, 0.45, 0.32, 0.2, 0.1, 0.0])
    m = S.lattice_mesh(1.0, 15.0, lon_min=-20.0, lon_max=20.0, jitter=0.15, land_frac=0.2, quad_frac=0.3,
                       depth=lambda lo, la: S.smooth_bathymetry(lo, la, 0.2, 120.0), sigma=sig)
    rm = ref_mesh(m, sigma=sig)
    rm.vertical_coord = "sigma"
    lon_n, lat_n = np.radians(np.asarray(m.nodes_lon)), np.radians(np.asarray(m.nodes_lat))
    pseudo = (1.0 - sig) * 100.0
    lon, lat, z, status = particles(m, 1200, 59, z=True, n_dead=20)
    snaps = S.gyre_snapshots(m, 6, amp=1.0, z_levels=pseudo, decay=60.0, w_scale=4e-4, placement="layer")
    for k, sn in enumerate(snaps):
        sn.eta = (0.6 * np.sin(2.0 * lon_n + 0.9 * k) * np.cos(3.0 * lat_n) - 0.15).astype(np.float32)
    rf = ref_fields(snaps)

    def surf(t):
        return 0.5 * np.sin(2.0 * lon_n + 2.0e-4 * t) * np.cos(3.0 * lat_n) - 0.1 + 0.3 * np.cos(lat_n + 1.0e-4 * t)

    cases = {"rk2_wlsq": run_case(rm, rf, lon, lat, z, status, "rk2", 3600.0, T, 10, w_interp="leastsq"),
             "rk4_widw_kick": run_case(rm, rf, lon, lat, z, status, "rk4", 3600.0, T, 10, w_interp="idw",
                                       kh=(20.0, 20.0), seed=3),
             "euler_wlsq": run_case(rm, rf, lon, lat, z, status, "euler", 1800.0, T, 12, w_interp="leastsq"),
             "rk2_widw_bwd": run_case(rm, rf, lon, lat, z, status, "rk2", 3600.0, T, 10, w_interp="idw",
                                      time_dir=-1.0),
             "rk4_wlsq_surf_kick": run_case(rm, rf, lon, lat, z, status, "rk4", 3600.0, T, 8, w_interp="leastsq",
                                            kh=(30.0, 10.0), seed=6, surfaces=lambda t0, t1: (surf(t0), surf(t1)))}
    save("golden_sigma_wring", mesh_record(rm), snaps, cases, {"lon": lon, "lat": lat, "z": z, "status": status})


def eta_time_fixture():
    """tracking.py:3097-3133 _eta_at_time, the surface a sigma step sees at
    the start and end times of its step, on the records of golden_sigma_surf
    (6 records 6 h apart): linear blends and the PCHIP stencil (multistage
    steps with temporal_reconstruction pchip), every step start and end of a
    forward run with dt = 1 h (and of a backward one), computed by the
    reference with a record cache standing in for its reader.
    tests/golden/golden_eta_time.npz."""
    import types
    from kelp.tracking import _eta_at_time, _snapshot_band
    T = 21600.0
    sig = np.array([1.0, 0.95, 0.88, 0.8, 0.7, 0.58, 0.45, 0.32, 0.2, 0.1, 0.0])
    m = S.lattice_mesh(1.0, 15.0, lon_min=-20.0, lon_max=20.0, jitter=0.15, land_frac=0.2, quad_frac=0.3,
                       depth=lambda lo, la: S.smooth_bathymetry(lo, la, 0.2, 120.0), sigma=sig)
    lon_n, lat_n = np.radians(np.asarray(m.nodes_lon)), np.radians(np.asarray(m.nodes_lat))
    etas = [(0.6 * np.sin(2.0 * lon_n + 0.9 * k) * np.cos(3.0 * lat_n) - 0.15).astype(np.float32) for k in range(6)]
    ft = np.arange(6) * T
    cache = types.SimpleNamespace(get=lambda i, *a, **k: types.SimpleNamespace(eta=etas[i]))
    d = {"file_times": ft, "etas": np.array(etas)}
    dt = 3600.0
    for tag, direction, t0 in (("fwd", 1, 0.0), ("bwd", -1, ft[-1])):
        times = t0 + direction * dt * np.arange(int(ft[-1] / dt) + 1)
        d[f"{tag}_times"] = times
        for pch in (False, True):
            out = [_eta_at_time(float(t), ft, ft.size, "stop", direction, cache, None, None, None, "tinterp",
                                None, None, pchip=pch, cycle=None, snap=_snapshot_band(dt)) for t in times]
            d[f"{tag}_{'pchip' if pch else 'linear'}"] = np.array([np.full(lon_n.size, np.nan) if e is None
                                                                   else np.asarray(e, dtype=np.float64) for e in out])
    np.savez_compressed(os.path.join(HERE, "golden_eta_time.npz"), **d)
    print("golden_eta_time", os.path.getsize(os.path.join(HERE, "golden_eta_time.npz")) // 1024, "KB")


CGRID_KEYS = ("corners", "elem_ji", "nlev", "nlev_raster", "zw", "area", "e3b", "kbu", "e3u", "kbv", "e3v",
              "e2u", "e1v")


def cgrid_fixture():
    """NEMO C-grid meshes built by the reference's own builder
    (readers/nemo/_mesh.py build_nemo_cgrid_mesh, imported without the
    reader package, which needs xarray): a regional curvilinear raster with
    islands, model face widths, and in 3-D z-levels with partial bottom cells
    and partial u faces; face-raster u/v (and interface w) records."""
    import types
    src = os.environ["KELP_REFERENCE_SRC"]
    for name in ("kelp.readers", "kelp.readers.nemo"):
        if name not in sys.modules:
            pkg = types.ModuleType(name)
            pkg.__path__ = [os.path.join(src, *name.split("."))]
            sys.modules[name] = pkg
    from kelp.readers.nemo._mesh import build_nemo_cgrid_mesh
    T = 86400.0
    ny, nx = 36, 48
    jj, ii = np.mgrid[0:ny, 0:nx].astype(np.float64)
    glamf = -10.0 + 0.5 * ii + 0.06 * np.sin(0.2 * jj)
    gphif = 30.0 + 0.4 * jj + 0.04 * np.cos(0.15 * ii)
    # T-point geometry (cell centres) for the masks and metrics
    glat_t = gphif - 0.2
    noise = (np.sin(0.31 * ii + 0.7) * np.cos(0.27 * jj - 0.4) + 0.6 * np.sin(0.13 * ii * jj / 9.0 + 1.1))
    wet = noise > -0.55
    wet[:, :2] = False
    wet[:2, :] = False
    e1t = 0.5 * 111120.0 * np.cos(np.radians(glat_t))
    e2t = np.full((ny, nx), 0.4 * 111120.0)
    e2u = e2t * (1.0 + 0.01 * np.sin(0.3 * jj))
    e1v = 0.5 * 111120.0 * np.cos(np.radians(gphif))
    zw = np.concatenate([[0.0], np.cumsum(10.0 * 1.35 ** np.arange(12))])   # 13 interfaces
    K = zw.size - 1
    depth = 60.0 + (zw[-1] - 80.0) * 0.5 * (1.0 + np.sin(0.11 * ii + 0.3) * np.cos(0.09 * jj))
    nlev = np.where(wet, np.clip(np.searchsorted(zw, depth, side="left"), 1, K), 0).astype(np.int32)
    lay = np.diff(zw)
    bot_ref = lay[np.maximum(nlev - 1, 0)]
    e3b = np.where(nlev > 0, np.clip(depth - zw[np.maximum(nlev - 1, 0)], 0.3 * bot_ref, bot_ref), 0.0)
    e3u0 = np.broadcast_to(lay[:, None, None], (K, ny, nx)).copy()
    for j in range(ny):
        for i in range(nx - 1):
            kb = min(nlev[j, i], nlev[j, i + 1]) - 1
            if kb >= 0:
                e3u0[kb, j, i] = min(e3b[j, i] if nlev[j, i] - 1 == kb else lay[kb],
                                     e3b[j, i + 1] if nlev[j, i + 1] - 1 == kb else lay[kb])
    area = e1t * e2t
    rng = np.random.default_rng(41)
    m3 = build_nemo_cgrid_mesh(glamf, gphif, wet, e2u=e2u, e1v=e1v, nlev2d=nlev, zw=zw, area=area, e3b=e3b,
                               e3u0=e3u0, name="cgrid3d")
    set_exact_nearest(m3, True)
    m2 = build_nemo_cgrid_mesh(glamf, gphif, wet, name="cgrid2d")
    set_exact_nearest(m2, True)

    def fields(three_d, n_snap=4):
        out = []
        lev = np.arange(K)[:, None, None]
        for k in range(n_snap):
            ph = 0.8 * k
            u = 0.4 * np.sin(0.25 * jj + ph) * np.cos(0.18 * ii) + 0.1
            v = 0.3 * np.cos(0.2 * ii - ph) * np.sin(0.15 * jj) - 0.05
            if not three_d:
                uu = np.where(wet, u, 0.0).astype(np.float32).reshape(-1)
                vv = np.where(wet, v, 0.0).astype(np.float32).reshape(-1)
                out.append(RVel(u=uu, v=vv, w=None, eta=np.zeros(ny * nx), uv_layout="nemo_cgrid"))
                continue
            dec = np.exp(-zw[:-1] / 600.0)[:, None, None]
            uu = (u[None] * dec * (lev < nlev[None])).astype(np.float32).reshape(K, -1)
            vv = (v[None] * dec * (lev < nlev[None])).astype(np.float32).reshape(K, -1)
            ww = (2e-4 * np.sin(0.3 * ii + 0.2 * jj + ph)[None] * np.sin(np.pi * zw / zw[-1])[:, None, None]
                  ).astype(np.float32).reshape(K + 1, -1)
            out.append(RVel(u=uu, v=vv, w=ww, eta=np.zeros(ny * nx), uv_layout="nemo_cgrid"))
        return out

    P = 1500
    lon = rng.uniform(glamf.min(), glamf.max(), P)
    lat = rng.uniform(gphif.min(), gphif.max(), P)
    z = rng.uniform(0.0, 1800.0, P)
    status = np.full(P, int(ParticleStatus.ALIVE), np.int32)
    status[rng.choice(P, 30, replace=False)] = int(ParticleStatus.OUTSIDE)
    for rm, tag, three_d in ((m2, "cgrid2d", False), (m3, "cgrid3d", True)):
        rf = fields(three_d)
        run = dict(uv_interp="nemo_cgrid")
        cases = {"rk2": run_case(rm, rf, lon, lat, z, status, "rk2", 7200.0, T, 12, **run),
                 "rk4": run_case(rm, rf, lon, lat, z, status, "rk4", 7200.0, T, 12, **run),
                 "euler": run_case(rm, rf, lon, lat, z, status, "euler", 3600.0, T, 12, **run),
                 "rk2_bwd": run_case(rm, rf, lon, lat, z, status, "rk2", 7200.0, T, 12, time_dir=-1.0, **run),
                 "rk4_steady": run_case(rm, rf, lon, lat, z, status, "rk4", 7200.0, T, 8, steady=True, **run)}
        if not three_d:
            cases["rk2_kick"] = run_case(rm, rf, lon, lat, z, status, "rk2", 7200.0, T, 12, kh=(50.0, 50.0),
                                         seed=13, **run)
            cases["rk2_walk"] = run_case(rm, rf, lon, lat, z, status, "rk2", 7200.0, T, 12, walk=True, **run)
        rec = mesh_record(rm)
        for k in CGRID_KEYS:
            rec["cgrid_" + k] = np.asarray(getattr(rm, "_nemo_cgrid_" + k))
        rec["cgrid_shape"] = np.array(rm._structured_shape)
        rec["cgrid_partial"] = np.array(rm._nemo_cgrid_partial)
        # the builder's inputs, for checking a restated builder against the reference's
        rec.update({"cgin_glamf": glamf, "cgin_gphif": gphif, "cgin_wet": wet})
        if three_d:
            rec.update({"cgin_e2u": e2u, "cgin_e1v": e1v, "cgin_nlev": nlev, "cgin_zw": zw, "cgin_area": area,
                        "cgin_e3b": e3b, "cgin_e3u0": e3u0})
        save(f"golden_{tag}", rec, rf, cases, {"lon": lon, "lat": lat, "z": z, "status": status})


def cgrid_tripolar_fixture():
    """A global tripolar C-grid (T-pivot north fold, E-W halo columns; the
    synthetic ORCA-like raster of kelp_b200.synthetic.tripolar_grid) through
    the reference's own NemoCgridLayout, build_nemo_cgrid_mesh and
    nemo_cgrid_to_canonical, and its C-grid steps (2-D RK2, 3-D RK4 with
    partial bottom cells) of particles seeded next to the seam and the fold:
    tests/golden/golden_cgrid_tripolar2d.npz / _tripolar3d.npz."""
    import types
    src = os.environ["KELP_REFERENCE_SRC"]
    for name in ("kelp.readers", "kelp.readers.nemo"):
        if name not in sys.modules:
            pkg = types.ModuleType(name)
            pkg.__path__ = [os.path.join(src, *name.split("."))]
            sys.modules[name] = pkg
    from kelp.readers.nemo._mesh import build_nemo_cgrid_mesh
    from kelp.readers.nemo._layout import NemoCgridLayout, nemo_cgrid_to_canonical
    T = 86400.0
    ny, nx = 48, 66
    lay, glamf, gphif, glamt, gphit = S.tripolar_grid(ny, nx, fold="T")
    rlay = NemoCgridLayout((ny, nx), halo_cols=True, halo_row=True, periodic=True, fold="T")

    def sep(lo1, la1, lo2, la2):
        r = np.radians
        c = np.sin(r(la1)) * np.sin(r(la2)) + np.cos(r(la1)) * np.cos(r(la2)) * np.cos(r(lo1 - lo2))
        return np.degrees(np.arccos(np.clip(c, -1.0, 1.0)))

    jj, ii = np.indices((ny, nx))
    noise = np.sin(0.43 * ii + 0.2) * np.cos(0.37 * jj - 0.5) + 0.5 * np.sin(0.11 * ii * jj / 7.0)
    wet = ((sep(glamt, gphit, 73.0, 65.0) > 14.0) & (sep(glamt, gphit, -107.0, 65.0) > 14.0) & (gphit > -70.0)
           & (noise > -0.9))
    wet = nemo_cgrid_to_canonical(wet.astype(np.float64), rlay, "T") > 0.5
    zw = np.concatenate([[0.0], np.cumsum(10.0 * 1.35 ** np.arange(12))])
    K = zw.size - 1
    lay_d = np.diff(zw)
    depth = 60.0 + (zw[-1] - 80.0) * 0.5 * (1.0 + np.sin(np.radians(3.0 * glamt)) * np.cos(np.radians(2.0 * gphit)))
    nlev = np.where(wet, np.clip(np.searchsorted(zw, depth, side="left"), 1, K), 0).astype(np.int32)
    bot_ref = lay_d[np.maximum(nlev - 1, 0)]
    e3b = np.where(nlev > 0, np.clip(depth - zw[np.maximum(nlev - 1, 0)], 0.3 * bot_ref, bot_ref), 0.0)
    nlev = nemo_cgrid_to_canonical(nlev.astype(np.float64), rlay, "T").astype(np.int32)
    e3b = nemo_cgrid_to_canonical(e3b, rlay, "T")
    u2, v2, e2u, e1v = S.cgrid_stream_flow(glamf, gphif, amp=3e7)
    e2u = nemo_cgrid_to_canonical(e2u, rlay, "U")
    e1v = nemo_cgrid_to_canonical(e1v, rlay, "V")
    area = nemo_cgrid_to_canonical(np.maximum(e2u * e1v, 1.0), rlay, "T")
    m3 = build_nemo_cgrid_mesh(glamf, gphif, wet, layout=rlay, e2u=e2u, e1v=e1v, nlev2d=nlev, zw=zw, area=area,
                               e3b=e3b, name="tripolar3d")
    set_exact_nearest(m3, True)
    m2 = build_nemo_cgrid_mesh(glamf, gphif, wet, layout=rlay, name="tripolar2d")
    set_exact_nearest(m2, True)

    def fields(three_d, n_snap=3):
        out = []
        for k in range(n_snap):
            ph = 1.0 + 0.25 * k
            u = nemo_cgrid_to_canonical(u2 * ph, rlay, "U", vector=True)
            v = nemo_cgrid_to_canonical(v2 * (2.0 - ph * 0.5), rlay, "V", vector=True)
            if not three_d:
                out.append(RVel(u=u.astype(np.float32).reshape(-1), v=v.astype(np.float32).reshape(-1), w=None,
                                eta=np.zeros(ny * nx), uv_layout="nemo_cgrid"))
                continue
            lev = np.arange(K)[:, None, None]
            dec = np.exp(-zw[:-1] / 400.0)[:, None, None]
            uu = (u[None] * dec * (lev < nlev[None])).astype(np.float32).reshape(K, -1)
            vv = (v[None] * dec * (lev < nlev[None])).astype(np.float32).reshape(K, -1)
            wt = nemo_cgrid_to_canonical(3e-4 * np.sin(np.radians(5.0 * glamt + 40.0 * k)) * np.cos(np.radians(gphit)),
                                         rlay, "T")
            ww = (wt[None] * np.sin(np.pi * zw / zw[-1])[:, None, None]).astype(np.float32).reshape(K + 1, -1)
            out.append(RVel(u=uu, v=vv, w=ww, eta=np.zeros(ny * nx), uv_layout="nemo_cgrid"))
        return out

    # particles: uniform over the wet cells, plus clusters across the seam
    # (+-180) and along the fold line (the poles' meridian plane, high north)
    rng = np.random.default_rng(77)
    P = 1500
    lon = np.concatenate([rng.uniform(-180, 180, 700), rng.uniform(176.0, 184.0, 400),
                          np.where(rng.random(400) < 0.5, 73.0, -107.0) + rng.uniform(-30, 30, 400)])
    lat = np.concatenate([rng.uniform(-60, 85, 700), rng.uniform(-50, 70, 400), rng.uniform(76.0, 89.0, 400)])
    lon = ((lon + 180.0) % 360.0) - 180.0
    z = rng.uniform(0.0, 1500.0, P)
    status = np.full(P, int(ParticleStatus.ALIVE), np.int32)
    for rm, tag, three_d in ((m2, "tripolar2d", False), (m3, "tripolar3d", True)):
        rf = fields(three_d)
        run = dict(uv_interp="nemo_cgrid")
        if three_d:
            cases = {"rk4": run_case(rm, rf, lon, lat, z, status, "rk4", 10800.0, T, 12, **run),
                     "rk2": run_case(rm, rf, lon, lat, z, status, "rk2", 10800.0, T, 12, **run)}
        else:
            cases = {"rk2": run_case(rm, rf, lon, lat, z, status, "rk2", 10800.0, T, 12, **run),
                     "rk4": run_case(rm, rf, lon, lat, z, status, "rk4", 10800.0, T, 12, **run)}
        rec = mesh_record(rm)
        for k in CGRID_KEYS:
            rec["cgrid_" + k] = np.asarray(getattr(rm, "_nemo_cgrid_" + k))
        rec["cgrid_shape"] = np.array(rm._structured_shape)
        rec["cgrid_partial"] = np.array(rm._nemo_cgrid_partial)
        rec.update({"cgin_glamf": glamf, "cgin_gphif": gphif, "cgin_wet": wet, "cgin_fold": np.array("T"),
                    "cgin_raw_u": u2, "cgin_raw_v": v2,
                    "cgin_canon_u": nemo_cgrid_to_canonical(u2, rlay, "U", vector=True),
                    "cgin_canon_v": nemo_cgrid_to_canonical(v2, rlay, "V", vector=True)})
        if three_d:
            rec.update({"cgin_e2u": e2u, "cgin_e1v": e1v, "cgin_nlev": nlev, "cgin_zw": zw, "cgin_area": area,
                        "cgin_e3b": e3b})
        save(f"golden_cgrid_{tag}", rec, rf, cases, {"lon": lon, "lat": lat, "z": z, "status": status})


def pchip_fixture():
    """Monotone-cubic (PCHIP) temporal reconstruction over a 4-snapshot
    stencil (numerics/temporal_reconstruct.py; the tracking layer's bundle,
    tracking.py:2415-2436): 2-D band, 3-D z-level (the fused RK2 PCHIP
    kernel and the unfused RK4), a sigma mesh.  Steps start one record in, so
    the stencil exists; the last interval falls back to the linear blend."""
    T = 86400.0
    m = S.lattice_mesh(3.0, 72.0, jitter=0.2, land_frac=0.3)
    rm = ref_mesh(m)
    snaps = S.gyre_snapshots(m, 6, amp=1.5)
    for k, sn in enumerate(snaps):   # an uneven record sequence: the cubic differs from the lerp
        sn.u = (sn.u * (1.0 + 0.6 * np.sin(1.3 * k))).astype(np.float32)
        sn.v = (sn.v * (1.0 - 0.4 * np.cos(0.9 * k))).astype(np.float32)
    rf = ref_fields(snaps)
    lon, lat, z, status = particles(m, 1200, 51, n_off=40, n_dead=20)
    cases = {"rk2": run_case(rm, rf, lon, lat, z, status, "rk2", 21600.0, T, 14, pchip=True, t0=T),
             "rk4_kick": run_case(rm, rf, lon, lat, z, status, "rk4", 21600.0, T, 14, pchip=True, t0=T,
                                  kh=(5.0e4, 5.0e4), seed=21)}
    save("golden_pchip2d", mesh_record(rm), snaps, cases, {"lon": lon, "lat": lat, "z": z, "status": status})

    zl = S.stretched_levels(12, 5.0, 4000.0)
    m = S.lattice_mesh(3.0, 60.0, jitter=0.2, land_frac=0.25,
                       depth=lambda lo, la: S.smooth_bathymetry(lo, la, 30.0, 4000.0), sigma=zl)
    rm = ref_mesh(m, sigma=zl)
    snaps = S.gyre_snapshots(m, 6, amp=1.5, z_levels=zl, decay=800.0, w_scale=2e-3)
    for k, sn in enumerate(snaps):
        f = 1.0 + 0.5 * np.sin(1.1 * k)
        sn.u, sn.v, sn.w = ((x * f).astype(np.float32) for x in (sn.u, sn.v, sn.w))
    rf = ref_fields(snaps)
    lon, lat, z, status = particles(m, 1200, 52, z=True, n_dead=20)
    cases = {"rk2_wbary": run_case(rm, rf, lon, lat, z, status, "rk2", 21600.0, T, 14, w_interp="barycentric",
                                   pchip=True, t0=T),
             "rk4_wnear": run_case(rm, rf, lon, lat, z, status, "rk4", 21600.0, T, 14, w_interp="nearest",
                                   pchip=True, t0=T)}
    save("golden_pchip3d", mesh_record(rm), snaps, cases, {"lon": lon, "lat": lat, "z": z, "status": status})

    sig = np.array([1.0, 0.95, 0.88, 0.8, 0.7, 0.58, 0.45, 0.32, 0.2, 0.1, 0.0])
    m = S.lattice_mesh(1.0, 15.0, lon_min=-20.0, lon_max=20.0, jitter=0.15, land_frac=0.2, quad_frac=0.3,
                       depth=lambda lo, la: S.smooth_bathymetry(lo, la, 0.2, 120.0), sigma=sig)
    rm = ref_mesh(m, sigma=sig)
    rm.vertical_coord = "sigma"
    lon_n, lat_n = np.radians(np.asarray(m.nodes_lon)), np.radians(np.asarray(m.nodes_lat))
    Ts = 21600.0
    snaps = S.gyre_snapshots(m, 6, amp=1.0, z_levels=(1.0 - sig) * 100.0, decay=60.0, w_scale=4e-4)
    for k, sn in enumerate(snaps):
        sn.eta = (0.6 * np.sin(2.0 * lon_n + 0.9 * k) * np.cos(3.0 * lat_n) - 0.15).astype(np.float32)
    rf = ref_fields(snaps)
    lon, lat, z, status = particles(m, 1000, 53, z=True, n_dead=20)
    cases = {"rk4_wbary": run_case(rm, rf, lon, lat, z, status, "rk4", 3600.0, Ts, 16, w_interp="barycentric",
                                   pchip=True, t0=Ts),
             "rk2_wnear": run_case(rm, rf, lon, lat, z, status, "rk2", 3600.0, Ts, 16, w_interp="nearest",
                                   pchip=True, t0=Ts)}
    save("golden_pchip_sigma", mesh_record(rm), snaps, cases, {"lon": lon, "lat": lat, "z": z, "status": status})


def time_fixture():
    """The reference's time-bracket resolution (tracking._resolve_time_bracket)
    on a grid of query times, record axes, modes and directions."""
    from kelp.tracking import _resolve_time_bracket, _snapshot_band
    axes = {"uniform": np.arange(5) * 86400.0, "ragged": np.array([0.0, 3600.0, 90000.0, 100000.0, 180000.0])}
    rows = []
    for ai, (aname, ft) in enumerate(axes.items()):
        qs = np.concatenate([ft, ft + 1e-7, ft - 1e-7, np.linspace(-1e5, ft[-1] + 3e5, 57),
                             ft + 0.2, ft - 0.2])
        for mi, mode in enumerate(("stop", "cycle")):
            for d in (1, -1):
                for snap in (0.0, _snapshot_band(3600.0)):
                    for q in qs:
                        b = _resolve_time_bracket(float(q), ft, ft.size, mode, d, cycle=None, snap=snap)
                        out = [np.nan] * 5 if b is None else [float(x) for x in b]
                        rows.append([ai, mi, d, snap, q] + out)
    np.savez_compressed(os.path.join(HERE, "golden_time.npz"), rows=np.array(rows),
                        axis_uniform=axes["uniform"], axis_ragged=axes["ragged"])
    print("golden_time", len(rows))
    # the PCHIP stencil of every bracket (tracking._resolve_recon_stencil) and
    # the clock after a step that ends on the record ahead
    # (tracking._step_end_on_record), for clocks one pass either side in cycle mode
    from kelp.tracking import _resolve_recon_stencil, _step_end_on_record, _cycle_period
    crow = []
    for row in rows:
        ai, mi, d, snap, q = row[:5]
        if np.isnan(row[5]):
            continue
        ft = list(axes.values())[int(ai)]
        mode = ("stop", "cycle")[int(mi)]
        b = (int(row[5]), int(row[6]), row[7], row[8], row[9])
        st = _resolve_recon_stencil(b, ft.size)
        idx = [-1] * 4 if st is None else list(st[0])
        target = b[3] if d > 0 else b[2]
        dtn = abs(target - b[4])
        shifts = (0.0,) if mode == "stop" else (0.0, _cycle_period(ft, ft.size, None), -_cycle_period(ft, ft.size, None))
        for sh in shifts:
            end = _step_end_on_record(q + sh, b[4], dtn, int(d), ft, ft.size, mode, None)
            crow.append([ai, mi, d, q + sh] + list(b) + idx + [dtn, end])
    np.savez_compressed(os.path.join(HERE, "golden_clock.npz"), rows=np.array(crow, dtype=np.float64),
                        axis_uniform=axes["uniform"], axis_ragged=axes["ragged"])
    print("golden_clock", len(crow))


def lsq_fixture():
    """Element-layout u/v with the element-centre least squares
    (uv_interp "leastsq", interpolate.py:52-474): the seam-wrapping band and
    the regional tri/quad mesh, element velocities the mean of the vertex
    gyre values; steady, time-aware, backward, kicked and PCHIP runs."""
    T = 86400.0

    def elem_fields(m, snaps):
        en = np.asarray(m.elem_nodes)
        valid = en >= 0
        out = []
        for sn in snaps:
            u, v = np.asarray(sn.u), np.asarray(sn.v)
            ue = np.where(valid, u[np.maximum(en, 0)], 0.0).sum(1) / valid.sum(1)
            ve = np.where(valid, v[np.maximum(en, 0)], 0.0).sum(1) / valid.sum(1)
            out.append(RVel(u=ue.astype(u.dtype), v=ve.astype(v.dtype), w=None, eta=np.zeros(m.n_nodes),
                            uv_layout="element"))
        return out

    for name, m, P, dt, dtype in (
            ("golden_lsq_band", S.lattice_mesh(3.0, 72.0, jitter=0.2, land_frac=0.3), 1500, 21600.0, np.float32),
            ("golden_lsq_quad", S.lattice_mesh(1.0, 15.0, lon_min=-20.0, lon_max=20.0, jitter=0.15, land_frac=0.2,
                                               quad_frac=0.3), 1200, 10800.0, np.float64)):
        rm = ref_mesh(m)
        rf = elem_fields(m, S.gyre_snapshots(m, 5, amp=1.5, dtype=dtype))
        lon, lat, z, status = particles(m, P, 21, n_off=40, n_dead=30)
        cases = {"rk2": run_case(rm, rf, lon, lat, z, status, "rk2", dt, T, 12, uv_interp="leastsq"),
                 "rk4": run_case(rm, rf, lon, lat, z, status, "rk4", dt, T, 12, uv_interp="leastsq"),
                 "euler": run_case(rm, rf, lon, lat, z, status, "euler", dt, T, 12, uv_interp="leastsq"),
                 "rk2_bwd": run_case(rm, rf, lon, lat, z, status, "rk2", dt, T, 12, time_dir=-1.0,
                                     uv_interp="leastsq"),
                 "rk2_kick": run_case(rm, rf, lon, lat, z, status, "rk2", dt, T, 12, kh=(5.0e4, 5.0e4), seed=5,
                                      uv_interp="leastsq"),
                 "rk4_steady": run_case(rm, rf, lon, lat, z, status, "rk4", dt, T, 8, steady=True,
                                        uv_interp="leastsq"),
                 "rk2_pchip": run_case(rm, rf, lon, lat, z, status, "rk2", dt, T, 12, uv_interp="leastsq",
                                       pchip=True, t0=T)}
        rec = mesh_record(rm)
        rec.update(elem_center_lon=rm.elem_center_lon, elem_center_lat=rm.elem_center_lat, uv_element=np.array(1))
        save(name, rec, rf, cases, {"lon": lon, "lat": lat, "z": z, "status": status})


def lsq3d_fixture():
    """3-D element-layout u/v with the element-centre least squares per layer
    (uv_interp "leastsq", interpolate.py:644-750 with the layer of
    integrators.py _compute_layers), node W, through the reference's unfused
    3-D steps: the z-level mesh of golden_3d, element velocities the mean of
    the vertex gyre values of each layer; W nearest / barycentric / least
    squares, RK2 / RK4 / Euler, kick, backward, PCHIP.
    tests/golden/golden_lsq3d.npz."""
    T = 86400.0
    zl = S.stretched_levels(12, 5.0, 4000.0)
    m = S.lattice_mesh(3.0, 60.0, jitter=0.2, land_frac=0.25,
                       depth=lambda lo, la: S.smooth_bathymetry(lo, la, 30.0, 4000.0), sigma=zl)
    rm = ref_mesh(m, sigma=zl)
    en = np.asarray(m.elem_nodes)
    valid = en >= 0
    rf = []
    for sn in S.gyre_snapshots(m, 5, amp=1.5, z_levels=zl, decay=800.0, w_scale=2e-3):
        u, v = np.asarray(sn.u), np.asarray(sn.v)
        ue = np.where(valid[None], u[:, np.maximum(en, 0)], 0.0).sum(2) / valid.sum(1)[None]
        ve = np.where(valid[None], v[:, np.maximum(en, 0)], 0.0).sum(2) / valid.sum(1)[None]
        rf.append(RVel(u=ue.astype(u.dtype), v=ve.astype(v.dtype), w=np.asarray(sn.w), eta=np.zeros(m.n_nodes),
                       uv_layout="element"))
    lon, lat, z, status = particles(m, 1200, 53, z=True, n_dead=20)
    cases = {"rk2_wbary": run_case(rm, rf, lon, lat, z, status, "rk2", 21600.0, T, 10, w_interp="barycentric",
                                   uv_interp="leastsq"),
             "rk4_wnear_kick": run_case(rm, rf, lon, lat, z, status, "rk4", 21600.0, T, 10, w_interp="nearest",
                                        kh=(3.0e4, 3.0e4), seed=5, uv_interp="leastsq"),
             "euler_wlsq": run_case(rm, rf, lon, lat, z, status, "euler", 10800.0, T, 12, w_interp="leastsq",
                                    uv_interp="leastsq"),
             "rk2_wlsq_bwd": run_case(rm, rf, lon, lat, z, status, "rk2", 21600.0, T, 10, w_interp="leastsq",
                                      time_dir=-1.0, uv_interp="leastsq"),
             "rk4_wbary_pchip": run_case(rm, rf, lon, lat, z, status, "rk4", 21600.0, T, 8, w_interp="barycentric",
                                         uv_interp="leastsq", pchip=True, t0=T)}
    rec = mesh_record(rm)
    rec.update(elem_center_lon=rm.elem_center_lon, elem_center_lat=rm.elem_center_lat, uv_element=np.array(1))
    save("golden_lsq3d", rec, rf, cases, {"lon": lon, "lat": lat, "z": z, "status": status})


def edge_fixture():
    """Element-layout u/v by the edge-neighbour least squares (uv_interp
    "edge_leastsq", interpolate.py:2588-2747, 3210-3300): the plane through
    the containing element's centre velocity and its edge neighbours', with
    mirrored ghost points on boundary edges (freeslip or noslip), through the
    reference's unfused steps: the seam-wrapping band and the regional
    tri/quad mesh in 2-D, the z-level mesh of golden_3d in 3-D.
    tests/golden/golden_edge_band.npz, golden_edge_quad.npz, golden_edge3d.npz."""
    T = 86400.0

    def elem_fields(m, snaps):
        en = np.asarray(m.elem_nodes)
        valid = en >= 0
        out = []
        for sn in snaps:
            u, v = np.asarray(sn.u), np.asarray(sn.v)
            if u.ndim == 1:
                ue = np.where(valid, u[np.maximum(en, 0)], 0.0).sum(1) / valid.sum(1)
                ve = np.where(valid, v[np.maximum(en, 0)], 0.0).sum(1) / valid.sum(1)
            else:
                ue = np.where(valid[None], u[:, np.maximum(en, 0)], 0.0).sum(2) / valid.sum(1)[None]
                ve = np.where(valid[None], v[:, np.maximum(en, 0)], 0.0).sum(2) / valid.sum(1)[None]
            out.append(RVel(u=ue.astype(u.dtype), v=ve.astype(v.dtype), w=None if sn.w is None else np.asarray(sn.w),
                            eta=np.zeros(m.n_nodes), uv_layout="element"))
        return out

    def saved(name, rm, rf, cases, lon, lat, z, status):
        rec = mesh_record(rm)
        rec.update(elem_center_lon=rm.elem_center_lon, elem_center_lat=rm.elem_center_lat, uv_element=np.array(1),
                   uv_edge=np.array(1))
        save(name, rec, rf, cases, {"lon": lon, "lat": lat, "z": z, "status": status})

    ui = "edge_leastsq"
    for name, m, P, dt, dtype in (
            ("golden_edge_band", S.lattice_mesh(3.0, 72.0, jitter=0.2, land_frac=0.3), 1500, 21600.0, np.float32),
            ("golden_edge_quad", S.lattice_mesh(1.0, 15.0, lon_min=-20.0, lon_max=20.0, jitter=0.15, land_frac=0.2,
                                                quad_frac=0.3), 1200, 10800.0, np.float64)):
        rm = ref_mesh(m)
        rf = elem_fields(m, S.gyre_snapshots(m, 5, amp=1.5, dtype=dtype))
        lon, lat, z, status = particles(m, P, 71, n_off=40, n_dead=30)
        cases = {"rk2": run_case(rm, rf, lon, lat, z, status, "rk2", dt, T, 12, uv_interp=ui),
                 "rk4_noslip": run_case(rm, rf, lon, lat, z, status, "rk4", dt, T, 12, uv_interp=ui,
                                        edge_bc="noslip"),
                 "euler": run_case(rm, rf, lon, lat, z, status, "euler", dt, T, 12, uv_interp=ui),
                 "rk2_kick_noslip": run_case(rm, rf, lon, lat, z, status, "rk2", dt, T, 12, kh=(5.0e4, 5.0e4),
                                             seed=5, uv_interp=ui, edge_bc="noslip")}
        saved(name, rm, rf, cases, lon, lat, z, status)
    zl = S.stretched_levels(12, 5.0, 4000.0)
    m = S.lattice_mesh(3.0, 60.0, jitter=0.2, land_frac=0.25,
                       depth=lambda lo, la: S.smooth_bathymetry(lo, la, 30.0, 4000.0), sigma=zl)
    rm = ref_mesh(m, sigma=zl)
    rf = elem_fields(m, S.gyre_snapshots(m, 5, amp=1.5, z_levels=zl, decay=800.0, w_scale=2e-3))
    lon, lat, z, status = particles(m, 1200, 73, z=True, n_dead=20)
    cases = {"rk2_wbary": run_case(rm, rf, lon, lat, z, status, "rk2", 21600.0, T, 10, w_interp="barycentric",
                                   uv_interp=ui),
             "rk4_wlsq_noslip": run_case(rm, rf, lon, lat, z, status, "rk4", 21600.0, T, 10, w_interp="leastsq",
                                         uv_interp=ui, edge_bc="noslip"),
             "euler_wnear": run_case(rm, rf, lon, lat, z, status, "euler", 10800.0, T, 12, w_interp="nearest",
                                     uv_interp=ui)}
    saved("golden_edge3d", rm, rf, cases, lon, lat, z, status)


RNG_KEY_SETS = (   # (seed, realization, first particle id, step, component), 2^20 particles each
    (0, 0, 0, 0, 0),
    (20240917, 3, 5_000_000, 1459, 0),
    (2**63 - 25, 63, 2**40, 99_999, 1),
    (7, 1, 123_456_789, 42, 0),
)
RNG_SET_SIZE = 1 << 20


def sample_fixture():
    """sampling.py:727 sample_field, the reference's own outputs: 2-D node
    fields on a seam-wrapping triangle band and on a regional tri/quad mesh,
    and a z-level mid-layer (K-1, N) field on a 3-D band, with every method;
    fill NaNs in the fields (isolated nodes, and the levels below each node's
    bottom), query points on nodes (the coincident-node rule), dead particles
    and nearest = -1.  tests/golden/golden_sample_*.npz."""
    from kelp.numerics.sampling import sample_field as r_sample
    methods = ("nearest", "leastsq", "barycentric", "idw")
    zl = S.stretched_levels(12, 5.0, 4000.0)
    meshes = {
        "band": (S.lattice_mesh(3.0, 72.0, jitter=0.2, land_frac=0.3), None),
        "quad": (S.lattice_mesh(1.0, 15.0, lon_min=-20.0, lon_max=20.0, jitter=0.15, land_frac=0.2,
                                quad_frac=0.3), None),
        "3d": (S.lattice_mesh(3.0, 60.0, jitter=0.2, land_frac=0.25,
                              depth=lambda lo, la: S.smooth_bathymetry(lo, la, 30.0, 4000.0), sigma=zl), zl),
    }
    for name, (m, sig) in meshes.items():
        rm = ref_mesh(m, sigma=sig)
        rng = np.random.default_rng({"band": 1, "quad": 2, "3d": 3}[name])
        lo, la = np.asarray(m.nodes_lon), np.asarray(m.nodes_lat)
        N = lo.size
        v2 = 10.0 + 5.0 * np.sin(np.radians(2.0 * lo)) * np.cos(np.radians(3.0 * la)) + 0.01 * la
        v2[rng.choice(N, N // 30, replace=False)] = np.nan
        P = 1500
        lon, lat, z, _ = particles(m, P, 21 + len(name), z=sig is not None)
        on = rng.choice(P, 60, replace=False)                       # exactly on nodes
        pick = rng.choice(N, 60, replace=False)
        lon[on], lat[on] = lo[pick], la[pick]
        alive = np.ones(P, bool)
        alive[rng.choice(P, 40, replace=False)] = False
        nearest = find_nearest_nodes(rm, lon, lat).astype(np.int32)
        nearest[rng.choice(P, 20, replace=False)] = -1
        d = {f"mesh_{k}": v for k, v in mesh_record(rm).items()}
        d.update(lon=lon, lat=lat, alive=alive, nearest=nearest, v2=v2)
        for meth in methods:
            d[f"o2_{meth}"] = r_sample(v2, rm, lon, lat, nearest=nearest, alive=alive, method=meth)
        if sig is not None:
            zmid = 0.5 * (np.abs(zl)[:-1] + np.abs(zl)[1:])
            v3 = (4.0 + 20.0 * np.exp(-zmid[:, None] / 700.0)
                  * (1.0 + 0.3 * np.sin(np.radians(3.0 * lo)))[None, :])
            v3[zmid[:, None] > np.asarray(m.depth)[None, :]] = np.nan     # fill below the bottom
            v3[rng.integers(0, zmid.size, 50), rng.choice(N, 50, replace=False)] = np.nan
            d.update(z=z, v3=v3)
            for meth in methods:
                d[f"o3_{meth}"] = r_sample(v3, rm, lon, lat, z, nearest=nearest, alive=alive, method=meth)
        path = os.path.join(HERE, f"golden_sample_{name}.npz")
        np.savez_compressed(path, **d)
        print(f"golden_sample_{name}", os.path.getsize(path) // 1024, "KB")


def lazy0_fixture():
    """integrators.py:5691-5692 -> :5380-5608: a 3-D RK2 step whose payload is
    an endpoint LazyLerpField (alpha 0) takes the reference's unfused RK2,
    which materialises the payload as 1.0 a + 0.0 b.  On the 3-D z-level
    mesh of golden_3d, each step's payload is LazyLerpField(record ia,
    record ia + 1, 0.0) with record ia + 1 as vel_next: W barycentric, and W
    nearest with the split kick.  (With a non-finite b the reference's
    unfused step raises inside find_nearest_nodes once a NaN position
    reaches it, so only finite records are recorded.)
    tests/golden/golden_lazy0.npz."""
    T = 86400.0
    zl = S.stretched_levels(12, 5.0, 4000.0)
    m = S.lattice_mesh(3.0, 60.0, jitter=0.2, land_frac=0.25,
                       depth=lambda lo, la: S.smooth_bathymetry(lo, la, 30.0, 4000.0), sigma=zl)
    rm = ref_mesh(m, sigma=zl)
    snaps = S.gyre_snapshots(m, 4, amp=1.5, z_levels=zl, decay=800.0, w_scale=2e-3)
    rf = ref_fields(snaps)
    lon, lat, z, status = particles(m, 1200, 43, z=True, n_dead=20)

    def run(w_interp, kh, n_steps=10, dt=21600.0, seed=5):
        P = lon.size
        st = RState(lon=lon.copy(), lat=lat.copy(), z=z.copy(), status=status.copy(),
                    nearest_node=np.full(P, -1, np.int32), failure_reason=np.zeros(P, np.int8))
        out = {}
        for k in range(n_steps):
            t = k * dt
            ia = int(np.floor(t / T + 1e-9))
            kw = dict(uv_interp="barycentric", w_interp=w_interp, vel_next=rf[ia + 1], dt_to_next=(ia + 1) * T - t)
            if kh is not None:
                kw["diffusion"] = RDiff(scheme="uniform", kh_x=kh, kh_y=kh, seed=seed, real_id=0, step_i=k)
            st = RI.rk2_step(st, RLazy(rf[ia], rf[ia + 1], 0.0), rm, dt, 1.0, **kw)
        for name in ("lon", "lat", "z", "status", "nearest_node", "failure_reason", "u", "v", "w"):
            out[f"s{n_steps}_{name}"] = np.asarray(getattr(st, name))
        out["params"] = np.array([dt, T, n_steps, 1.0, -1 if kh is None else kh, -1 if kh is None else kh, seed],
                                 dtype=np.float64)
        return out

    cases = {"rk2_wbary": run("barycentric", None), "rk2_wnear_kick": run("nearest", 3.0e4)}
    save("golden_lazy0", mesh_record(rm), snaps, cases, {"lon": lon, "lat": lat, "z": z, "status": status})
    for c, o in cases.items():
        print(c, "statuses", np.bincount(o["s10_status"]), "failure reasons", np.bincount(o["s10_failure_reason"]))


def cellrule_fixture():
    """mesh.py:464-616 choose_grid_hash_cell, the reference's own reports in
    both modes, and its per-sample kernel _gh_sample_stats (:384-461) at a few
    candidates of the ladder: a seam-wrapping global band, a regional mesh
    whose node density varies by two orders of magnitude (a sinh-stretched
    lattice: exact mode leaves the reader's cell there), and a near-polar
    mesh whose caps reach the pole.  The band and the polar mesh are sampled
    (sample < E: the seeded draw), the stretched mesh uses every element
    centre.
    tests/golden/golden_cellrule_*.npz."""
    import json
    from kelp.core import mesh as RM
    from kelp_b200.mesh import make_mesh

    def stretched():
        b = S.lattice_mesh(0.5, 20.0, lon_min=-30.0, lon_max=30.0, jitter=0.2, land_frac=0.1)
        lon = 30.0 * np.sinh(np.asarray(b.nodes_lon) / 5.0) / np.sinh(6.0)
        lat = 20.0 * np.sinh(np.asarray(b.nodes_lat) / 4.0) / np.sinh(5.0)
        return make_mesh("stretched", lon, lat, np.asarray(b.depth), np.asarray(b.elem_nodes))

    meshes = {"band": (S.lattice_mesh(2.0, 75.0, jitter=0.25, land_frac=0.3), 5000),
              "stretched": (stretched(), 200_000),
              "polar": (S.lattice_mesh(1.5, 88.5, jitter=0.3, land_frac=0.2), 20_000)}
    for name, (m, sample) in meshes.items():
        rm = ref_mesh(m)
        reps = {mode: RM.choose_grid_hash_cell(rm, exact=(mode == "exact"), sample=sample)[1]
                for mode in ("exact", "approx")}
        d = {f"mesh_{k}": v for k, v in mesh_record(rm).items()}
        d["mesh_elem_center_lon"] = np.asarray(rm.elem_center_lon)
        d["mesh_elem_center_lat"] = np.asarray(rm.elem_center_lat)
        d["sample"] = np.array(sample)
        for mode, rep in reps.items():
            d[f"report_{mode}"] = np.array(json.dumps(rep))
        # per-sample statistics of three candidates (the chooser's sample, all finite here)
        E = rm.n_elements
        pick = np.sort(np.random.default_rng(0).choice(E, sample, replace=False)) if E > sample else np.arange(E)
        qlon = np.ascontiguousarray(rm.elem_center_lon[pick], dtype=np.float64)
        qlat = np.ascontiguousarray(rm.elem_center_lat[pick], dtype=np.float64)
        nn = np.empty(qlon.size, dtype=np.int32)
        RM._grid_hash_nearest_batch(qlon.size, qlon, qlat, rm._gh_offsets, rm._gh_node_ids, rm._gh_cell_size,
                                    rm._gh_lon_min, rm._gh_lat_min, rm._gh_nx, rm._gh_ny, rm._gh_wrap_lon,
                                    rm.nodes_lon, rm.nodes_lat, RM._require_node_xyz(rm), nn, True,
                                    int(rm._gh_far_rows))
        d.update(qlon=qlon, qlat=qlat, nn=nn)
        lon_b, wrap = RM._gh_lon_branch(rm.nodes_lon)
        for k in (0, 2, 5):
            cell = float(rm._gh_cell_size) / (np.sqrt(2.0) ** k)
            lon_min, lat_min, nx, ny = RM._gh_grid_geometry(lon_b, rm.nodes_lat, cell, wrap)
            idx = RM._gh_cell_index(lon_b, rm.nodes_lat, cell, lon_min, lat_min, nx, ny, wrap)
            counts = np.bincount(idx, minlength=nx * ny).reshape(ny, nx)
            cum = np.zeros((ny + 1, nx + 1), dtype=np.int32)
            np.cumsum(counts, axis=0, dtype=np.int32, out=cum[1:, 1:])
            np.cumsum(cum[1:, 1:], axis=1, dtype=np.int32, out=cum[1:, 1:])
            occ = np.empty(qlon.size, np.int64)
            cost = np.empty(qlon.size, np.float64)
            unprov = np.empty(qlon.size, np.int8)
            approx = np.empty(qlon.size, np.int8)
            RM._gh_sample_stats(qlon, qlat, nn, np.ascontiguousarray(rm.nodes_lon), np.ascontiguousarray(rm.nodes_lat),
                                cum, cell, float(lon_min), float(lat_min), int(nx), int(ny), bool(wrap),
                                occ, cost, unprov, approx)
            d[f"k{k}_geom"] = np.array([cell, lon_min, lat_min, nx, ny, int(wrap)], dtype=np.float64)
            d.update({f"k{k}_occ": occ, f"k{k}_cost": cost, f"k{k}_unprov": unprov, f"k{k}_approx": approx})
        path = os.path.join(HERE, f"golden_cellrule_{name}.npz")
        np.savez_compressed(path, **d)
        print(f"golden_cellrule_{name}", os.path.getsize(path) // 1024, "KB",
              {m_: (r["chosen"], r["legacy"], len(r["candidates"])) for m_, r in reps.items()})


def sample_iface_fixture():
    """sampling.py:876-890: an interface-shaped (K, N) node field on a
    z-level mesh, which sample_field hands to the W interpolation of each
    method (vertical.py:1330-1420, time_dir +1): the 3-D band of
    golden_sample_3d, points at every depth (the surface, below the bottom),
    dead particles and nearest = -1.  tests/golden/golden_sample_iface.npz."""
    from kelp.numerics.sampling import sample_field as r_sample
    zl = S.stretched_levels(12, 5.0, 4000.0)
    m = S.lattice_mesh(3.0, 60.0, jitter=0.2, land_frac=0.25,
                       depth=lambda lo, la: S.smooth_bathymetry(lo, la, 30.0, 4000.0), sigma=zl)
    rm = ref_mesh(m, sigma=zl)
    rng = np.random.default_rng(61)
    lo = np.asarray(m.nodes_lon)
    zi = np.abs(np.asarray(zl))
    vk = (2.0 + 10.0 * np.exp(-zi[:, None] / 500.0) * (1.0 + 0.4 * np.cos(np.radians(2.0 * lo)))[None, :]
          + 1e-3 * np.arange(lo.size)[None, :] / lo.size)
    P = 1500
    lon, lat, z, _ = particles(m, P, 67, z=True)
    z[:40] = 0.0
    z[40:80] = 1e4          # below every bottom
    alive = np.ones(P, bool)
    alive[rng.choice(P, 40, replace=False)] = False
    nearest = find_nearest_nodes(rm, lon, lat).astype(np.int32)
    nearest[rng.choice(P, 20, replace=False)] = -1
    d = {f"mesh_{k}": v for k, v in mesh_record(rm).items()}
    d.update(lon=lon, lat=lat, z=z, alive=alive, nearest=nearest, vk=vk)
    for meth in ("nearest", "leastsq", "barycentric", "idw"):
        d[f"ok_{meth}"] = r_sample(vk, rm, lon, lat, z, nearest=nearest, alive=alive, method=meth)
    path = os.path.join(HERE, "golden_sample_iface.npz")
    np.savez_compressed(path, **d)
    print("golden_sample_iface", os.path.getsize(path) // 1024, "KB")


def sample_sigma_fixture():
    """sampling.py:620-723 _sample_sigma_3d: an interface (K, N) and a
    mid-layer (K-1, N) field on the sigma shelf of golden_sigma_surf with a
    free surface eta, every method; points at the surface and below every
    bottom, dead particles and nearest = -1.  tests/golden/golden_sample_sigma.npz."""
    from kelp.numerics.sampling import sample_field as r_sample
    sig = np.array([1.0, 0.95, 0.88, 0.8, 0.7, 0.58, 0.45, 0.32, 0.2, 0.1, 0.0])
    m = S.lattice_mesh(1.0, 15.0, lon_min=-20.0, lon_max=20.0, jitter=0.15, land_frac=0.2, quad_frac=0.3,
                       depth=lambda lo, la: S.smooth_bathymetry(lo, la, 0.2, 120.0), sigma=sig)
    rm = ref_mesh(m, sigma=sig)
    rm.vertical_coord = "sigma"
    rng = np.random.default_rng(79)
    lo, la = np.asarray(m.nodes_lon), np.asarray(m.nodes_lat)
    eta = 0.6 * np.sin(np.radians(2.0 * lo) * 20.0) * np.cos(np.radians(3.0 * la) * 10.0) - 0.15
    K = sig.size
    vk = 3.0 + 2.0 * sig[:, None] + 0.5 * np.cos(np.radians(4.0 * lo))[None, :] + 1e-3 * np.arange(K)[:, None]
    sm = 0.5 * (sig[:-1] + sig[1:])
    vm = 10.0 + 4.0 * sm[:, None] * (1.0 + 0.3 * np.sin(np.radians(5.0 * la)))[None, :]
    P = 1500
    lon, lat, z, _ = particles(m, P, 83, z=True)
    z[:40] = 0.0
    z[40:80] = 500.0     # below every column
    alive = np.ones(P, bool)
    alive[rng.choice(P, 40, replace=False)] = False
    nearest = find_nearest_nodes(rm, lon, lat).astype(np.int32)
    nearest[rng.choice(P, 20, replace=False)] = -1
    d = {f"mesh_{k}": v for k, v in mesh_record(rm).items()}
    d.update(lon=lon, lat=lat, z=z, alive=alive, nearest=nearest, vk=vk, vm=vm, eta=eta)
    for meth in ("nearest", "leastsq", "barycentric", "idw"):
        d[f"ok_{meth}"] = r_sample(vk, rm, lon, lat, z, nearest=nearest, alive=alive, eta=eta, method=meth, Dmin=0.5)
        d[f"om_{meth}"] = r_sample(vm, rm, lon, lat, z, nearest=nearest, alive=alive, eta=eta, method=meth, Dmin=0.5)
    path = os.path.join(HERE, "golden_sample_sigma.npz")
    np.savez_compressed(path, **d)
    print("golden_sample_sigma", os.path.getsize(path) // 1024, "KB")


def rng1m_fixture():
    """The reference's own _normal_pair on 4 x 2^20 keys (contiguous particle
    ids under 4 key tuples), stored as per-chunk digests (tests/golden/
    rng_digest.py; the 64 MB of pairs stay out of the repository):
    tests/golden/golden_rng_1m.json."""
    import json
    from numba import njit
    sys.path.insert(0, HERE)
    from rng_digest import CHUNK, digest

    @njit(cache=False)
    def pairs(seed, real_id, pid0, step, comp, n):
        out = np.empty((n, 2))
        for i in range(n):
            g1, g2 = _normal_pair(np.uint64(seed), np.uint64(real_id), np.uint64(pid0 + i), np.uint64(step),
                                  np.uint64(comp))
            out[i, 0] = g1
            out[i, 1] = g2
        return out

    sets = []
    for seed, rid, pid0, step, comp in RNG_KEY_SETS:
        g = pairs(seed, rid, pid0, step, comp, RNG_SET_SIZE)
        sets.append({"seed": str(seed), "real_id": rid, "pid0": str(pid0), "step": step, "comp": comp,
                     "n": RNG_SET_SIZE, "chunk": CHUNK,
                     "digests": [format(d, "016x") for d in digest(g)],
                     "first": [float.hex(float(v)) for v in g[0]]})
    with open(os.path.join(HERE, "golden_rng_1m.json"), "w") as fh:
        json.dump({"generator": "kelp.numerics.diffusion._normal_pair", "sets": sets}, fh, indent=1)
    print("golden_rng_1m")


def reftypes_fixture():
    """The attribute layout of the reference's own types (field names in
    order, the read-only properties each class defines, and the defaults of
    DiffusionStepArgs), for the drop-in test that passes objects shaped
    exactly like KELP's to kelp_b200's step functions:
    tests/golden/reference_types.json."""
    import dataclasses
    import inspect
    import json
    from kelp.core.particles import ParticleState as RPS
    out = {"Mesh": [f.name for f in dataclasses.fields(RMesh)],
           "VelocityField": [f.name for f in dataclasses.fields(RVel)],
           "ParticleState": [f.name for f in dataclasses.fields(RPS)],
           "LazyLerpField": ["vel_a", "vel_b", "alpha"],
           "DiffusionStepArgs": list(RDiff._fields),
           "DiffusionStepArgs_defaults": {k: v for k, v in RDiff._field_defaults.items()},
           "properties": {c.__name__: [n for n, v in inspect.getmembers(c) if isinstance(v, property)]
                          for c in (RMesh, RVel, RPS)}}
    with open(os.path.join(HERE, "reference_types.json"), "w") as fh:
        json.dump(out, fh, indent=1)
    print("reference_types")


if __name__ == "__main__":
    # no argument: every fixture; otherwise the named ones ("steps", "beach", ...)
    which = set(sys.argv[1:]) or {"steps", "beach", "time", "sigma", "cgrid", "pchip", "lsq", "rng1m", "tripolar", "reftypes", "sample", "cellrule", "lazy0", "sigma_surf", "eta_time", "sigma_az", "wring", "lsq3d", "sigma_wring", "sample_iface", "edge", "sample_sigma"}
    if "rng1m" in which:
        rng1m_fixture()
    if "reftypes" in which:
        reftypes_fixture()
    if "sample" in which:
        sample_fixture()
    if "cellrule" in which:
        cellrule_fixture()
    if "lazy0" in which:
        lazy0_fixture()
    if "sigma_surf" in which:
        sigma_surf_fixture()
    if "eta_time" in which:
        eta_time_fixture()
    if "sigma_az" in which:
        sigma_az_fixture()
    if "wring" in which:
        wring_fixture()
    if "lsq3d" in which:
        lsq3d_fixture()
    if "sigma_wring" in which:
        sigma_wring_fixture()
    if "sample_iface" in which:
        sample_iface_fixture()
    if "edge" in which:
        edge_fixture()
    if "sample_sigma" in which:
        sample_sigma_fixture()
    if "lsq" in which:
        lsq_fixture()
    if "steps" in which:
        main()
    if "beach" in which:
        beach_fixture()
    if "time" in which:
        time_fixture()
    if "sigma" in which:
        sigma_fixture()
    if "cgrid" in which:
        cgrid_fixture()
    if "tripolar" in which:
        cgrid_tripolar_fixture()
    if "pchip" in which:
        pchip_fixture()
