"""TEST INFRASTRUCTURE, NOT THE PRODUCT: ctypes driver of the CPU oracle
(``oracle/kelp_oracle.c``), a C restatement of KELP's step path.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline
leg use this module, and only as the checker / the timed CPU baseline.  The
functions mirror the reference's step API over its own array layout:
``step(state, vel, mesh, dt, time_dir, scheme, ...)`` returns new arrays like
KELP's ``rk2_step`` (``src/kelp/numerics/integrators.py:5611``).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")


class OMesh(C.Structure):
    _fields_ = [("N", C.c_int64), ("E", C.c_int64), ("max_v", C.c_int), ("max_conn", C.c_int),
                ("lon", C.c_void_p), ("lat", C.c_void_p), ("depth", C.c_void_p), ("xyz", C.c_void_p),
                ("zlev", C.c_void_p), ("en", C.c_void_p), ("n2e", C.c_void_p), ("n2e_cnt", C.c_void_p),
                ("gh_off", C.c_void_p), ("gh_ids", C.c_void_p),
                ("cell", C.c_double), ("lon_min", C.c_double), ("lat_min", C.c_double), ("r_earth", C.c_double),
                ("nx", C.c_int), ("ny", C.c_int), ("wrap", C.c_int), ("far_rows", C.c_int),
                ("exact", C.c_int), ("K", C.c_int),
                ("dl_p", C.c_void_p), ("dl_bed", C.c_void_p), ("dl_last", C.c_void_p), ("dl_M", C.c_int),
                ("enb", C.c_void_p), ("sigma", C.c_void_p), ("sig", C.c_int),
                ("cg", C.c_int), ("cg_corners", C.c_void_p), ("cg_ji", C.c_void_p), ("cg_nlev", C.c_void_p),
                ("cg_nlev_r", C.c_void_p), ("cg_nx", C.c_int), ("cg_K", C.c_int), ("cg_shrunk", C.c_int),
                ("cg_has_e", C.c_int), ("cg_nynx", C.c_int64),
                ("cg_e2u", C.c_void_p), ("cg_e1v", C.c_void_p), ("cg_area", C.c_void_p), ("cg_zw", C.c_void_p),
                ("cg_e3b", C.c_void_p), ("cg_e3u", C.c_void_p), ("cg_e3v", C.c_void_p),
                ("cg_kbu", C.c_void_p), ("cg_kbv", C.c_void_p), ("ec_lon", C.c_void_p), ("ec_lat", C.c_void_p)]


class OField(C.Structure):
    _fields_ = [("ua", C.c_void_p), ("va", C.c_void_p), ("wa", C.c_void_p),
                ("ub", C.c_void_p), ("vb", C.c_void_p), ("wb", C.c_void_p),
                ("ut", C.c_void_p), ("vt", C.c_void_p), ("wt", C.c_void_p),
                ("f32", C.c_int), ("alpha0", C.c_double), ("n", C.c_int64),
                ("aza", C.c_void_p), ("azb", C.c_void_p),
                ("etaa", C.c_void_p), ("etab", C.c_void_p), ("etat", C.c_void_p),
                ("pchip", C.c_int), ("ud", C.c_void_p), ("vd", C.c_void_p), ("wd", C.c_void_p),
                ("etad", C.c_void_p), ("pt", C.c_double * 4), ("lsq", C.c_int)]


class OStep(C.Structure):
    _fields_ = [("scheme", C.c_int), ("dims", C.c_int), ("w_code", C.c_int), ("kick", C.c_int),
                ("dt", C.c_double), ("td", C.c_double), ("ak", C.c_double * 4),
                ("kh_x", C.c_double), ("kh_y", C.c_double),
                ("seed", C.c_uint64), ("real_id", C.c_uint64), ("step_i", C.c_uint64),
                ("pid_offset", C.c_uint64), ("uv_dl", C.c_int),
                ("az_on", C.c_int), ("az_field", C.c_int), ("az_const", C.c_double),
                ("Dmin", C.c_double), ("z0b_min", C.c_double), ("alpha_end", C.c_double),
                ("eta_s", C.c_void_p), ("eta_e", C.c_void_p), ("sig_steady", C.c_int)]


_lib = None


def build() -> str:
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        L = C.CDLL(LIB)
        vp, i64 = C.c_void_p, C.c_int64
        L.orc_step.argtypes = [C.POINTER(OMesh), C.POINTER(OField), C.POINTER(OStep), i64,
                               vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, i64, vp]
        L.orc_walk.argtypes = [C.POINTER(OMesh), i64, vp, vp, vp, vp, vp]
        L.orc_find_nearest.argtypes = [C.POINTER(OMesh), i64, vp, vp, vp]
        L.orc_contain.argtypes = [C.POINTER(OMesh), i64, vp, vp, vp, vp]
        L.orc_sample_sigma.argtypes = [C.POINTER(OMesh), vp, C.c_int, vp, C.c_double, i64, vp, vp, vp, vp, vp,
                                       C.c_int, vp]
        L.orc_cell_stats.argtypes = [C.POINTER(OMesh), vp, C.c_double, C.c_double, C.c_double, C.c_int, C.c_int,
                                     C.c_int, i64, vp, vp, vp, vp, vp, vp, vp]
        L.orc_normals.argtypes = [i64, C.c_uint64, C.c_uint64, C.c_uint64, C.c_uint64, C.c_uint64, vp]
        L.orc_node_xyz.argtypes = [i64, vp, vp, vp]
        L.orc_sample.argtypes = [C.POINTER(OMesh), vp, C.c_int, vp, i64, vp, vp, vp, vp, vp, C.c_int, vp]
        L.orc_normal_pair.argtypes = [C.c_uint64] * 5 + [vp]
        L.orc_beach.argtypes = [C.POINTER(OMesh), C.c_void_p, vp, i64, vp, vp, vp, vp, vp, vp, vp, vp, vp]
        L.orc_set_threads.argtypes = [C.c_int]
        L.orc_get_threads.restype = C.c_int
        _lib = L
    return _lib


def set_threads(n: int) -> None:
    lib().orc_set_threads(int(n))


def threads() -> int:
    return int(lib().orc_get_threads())


def _p(a):
    return None if a is None else a.ctypes.data


class MeshView:
    """The oracle's view of a mesh (keeps the converted arrays alive)."""

    def __init__(self, mesh):
        c = lambda a, t: np.ascontiguousarray(a, dtype=t)
        self.lon = c(mesh.nodes_lon, np.float64)
        self.lat = c(mesh.nodes_lat, np.float64)
        self.depth = c(mesh.depth, np.float64)
        xyz = getattr(mesh, "_node_xyz", None)
        if xyz is None:   # a mesh whose node table is filled on first use: the C library's values, here
            xyz = node_xyz(mesh.nodes_lon, mesh.nodes_lat)
            mesh._node_xyz = xyz
        self.xyz = c(xyz, np.float64)
        self.en = c(mesh.elem_nodes, np.int32)
        self.n2e = c(mesh.node_to_elems, np.int32)
        self.cnt = c(mesh.node_to_elems_count, np.int32)
        self.off = c(mesh._gh_offsets, np.int32)
        self.ids = c(mesh._gh_node_ids, np.int32)
        sig = np.asarray(getattr(mesh, "sigma", np.zeros(0)))
        self.is_sigma = getattr(mesh, "vertical_coord", "zlevel") == "sigma"
        self.sig = c(sig, np.float64) if (self.is_sigma and sig.size) else None
        self.zl = c(np.abs(sig), np.float64) if (sig.size and not self.is_sigma) else None
        s = OMesh()
        s.N, s.E = self.lon.size, self.en.shape[0]
        s.max_v, s.max_conn = self.en.shape[1], self.n2e.shape[1]
        s.lon, s.lat, s.depth, s.xyz = _p(self.lon), _p(self.lat), _p(self.depth), _p(self.xyz)
        s.zlev = _p(self.zl)
        s.en, s.n2e, s.n2e_cnt, s.gh_off, s.gh_ids = _p(self.en), _p(self.n2e), _p(self.cnt), _p(self.off), _p(self.ids)
        s.cell, s.lon_min, s.lat_min = float(mesh._gh_cell_size), float(mesh._gh_lon_min), float(mesh._gh_lat_min)
        s.r_earth = float(getattr(mesh, "r_earth", 6371000.0))
        s.nx, s.ny, s.wrap, s.far_rows = int(mesh._gh_nx), int(mesh._gh_ny), int(bool(mesh._gh_wrap_lon)), int(mesh._gh_far_rows)
        s.exact = int(bool((mesh.metadata or {}).get("exact_nearest", False)))
        s.K = 0 if self.zl is None else int(self.zl.size)
        if self.sig is not None:   # sigma interfaces, 1 at the surface to 0 at the bed
            s.sigma, s.sig, s.K = _p(self.sig), 1, int(self.sig.size)
        if getattr(mesh, "_nemo_cgrid", False):   # NEMO C-grid: the builder's tables
            g = lambda name, t: c(getattr(mesh, "_nemo_cgrid_" + name), t)
            self.cg = {"corners": g("corners", np.int32), "ji": g("elem_ji", np.int64),
                       "nlev": g("nlev", np.int32), "nlev_r": c(np.asarray(mesh._nemo_cgrid_nlev_raster).reshape(-1),
                                                                 np.int32),
                       "e2u": g("e2u", np.float64), "e1v": g("e1v", np.float64), "area": g("area", np.float64),
                       "zw": g("zw", np.float64), "e3b": g("e3b", np.float64), "e3u": g("e3u", np.float64),
                       "e3v": g("e3v", np.float64), "kbu": g("kbu", np.int32), "kbv": g("kbv", np.int32)}
            ny, nx = (int(x) for x in mesh._structured_shape)
            s.cg, s.cg_nx, s.cg_nynx = 1, nx, ny * nx
            s.cg_K = max(int(self.cg["zw"].size) - 1, 0)
            s.cg_shrunk = int(getattr(mesh, "_nemo_cgrid_partial", "shrunk") == "shrunk")
            s.cg_has_e = int(self.cg["e2u"].size > 0)
            for k, v in self.cg.items():
                setattr(s, "cg_" + k, _p(v) if v.size else None)
            s.zlev, s.K = None, 0   # the C-grid step measures depth on its own interfaces
        enb = getattr(mesh, "_elem_neighbors", None)
        self.enb = None if enb is None else c(enb, np.int32)
        s.enb = _p(self.enb)
        ecl = getattr(mesh, "elem_center_lon", None)
        self.ec_lon = None if ecl is None else c(ecl, np.float64)
        self.ec_lat = None if ecl is None else c(mesh.elem_center_lat, np.float64)
        s.ec_lon, s.ec_lat = _p(self.ec_lon), _p(self.ec_lat)
        self.s = s
        self.mesh = mesh
        self.placement = None

    def use_placement(self, placement: str) -> None:
        """Attach the depth-linear data-point table for ``placement``
        (vertical_uv.py:181-278, node layout; z-level meshes)."""
        if placement == self.placement:
            return
        if self.is_sigma:
            # sigma meshes (layer_linear only): layer centres in s, every
            # column reads every layer, wet everywhere (vertical_uv.py:196-211)
            sg = np.asarray(self.mesh.sigma, dtype=np.float64)
            self.dl_p = np.ascontiguousarray(1.0 - 0.5 * (sg[:-1] + sg[1:]))
            self.dl_last = np.full(self.lon.size, self.dl_p.size - 1, np.int32)
            self.dl_bed = np.full(self.lon.size, np.inf)
            self.s.dl_p, self.s.dl_bed, self.s.dl_last = _p(self.dl_p), _p(self.dl_bed), _p(self.dl_last)
            self.s.dl_M = int(self.dl_p.size)
            self.placement = placement
            return
        z = np.abs(np.asarray(self.mesh.sigma, dtype=np.float64))
        if placement == "level":
            p, lower = z.copy(), z
        else:
            p, lower = 0.5 * (z[:-1] + z[1:]), z[1:]
        d = np.asarray(self.mesh.depth, dtype=np.float64)
        geo = np.searchsorted(lower, d, side="right").astype(np.int64) - 1
        geo[np.isnan(d)] = 0
        last = np.minimum(geo, p.size - 1)
        decl = (getattr(self.mesh, "metadata", None) or {}).get("uv_data_last")
        if decl is not None:
            last = np.minimum(last, np.asarray(decl).astype(np.int64))
        self.dl_p = np.ascontiguousarray(p)
        self.dl_last = np.ascontiguousarray(np.maximum(last, 0), dtype=np.int32)
        self.dl_bed = np.ascontiguousarray(d.copy())
        self.s.dl_p, self.s.dl_bed, self.s.dl_last = _p(self.dl_p), _p(self.dl_bed), _p(self.dl_last)
        self.s.dl_M = int(self.dl_p.size)
        self.placement = placement


def _field_arrays(f, dtype):
    u = np.ascontiguousarray(f.u, dtype=dtype)
    v = np.ascontiguousarray(f.v, dtype=dtype)
    w = None if getattr(f, "w", None) is None else np.ascontiguousarray(f.w, dtype=dtype)
    return u, v, w


def step(state, vel, mesh, dt, time_dir, scheme: str, *, vel_next=None, dt_to_next=None, w_interp="nearest",
         diffusion=None, pid=None, release_step=None, global_step=-1, view=None, Dmin=0.5, z0b_min=0.1,
         recon=None, uv_interp="barycentric", eta_start=None, eta_end=None, edge_leastsq_bc="freeslip"):
    """One step of every particle; returns a dict of new arrays
    (lon, lat, z, status, nearest_node, failure_reason, u, v, w, and elem
    when the state carries elements: elem_search walk, the mesh's
    ``_elem_neighbors`` table required).  ``recon`` = (4 snapshots, their
    times, the step's time, direction) reconstructs the RK stages by PCHIP
    (temporal_reconstruct.py:298-325; Euler ignores it).  ``eta_start`` /
    ``eta_end``: the tracking layer's surfaces of a sigma step
    (sigma_eta_start / sigma_eta_end), None for the payload's own."""
    view = view or MeshView(mesh)
    vel_a = getattr(vel, "vel_a", vel)
    vel_b = getattr(vel, "vel_b", vel_next if vel_next is not None else vel_a)
    alpha0 = float(getattr(vel, "alpha", 0.0))
    target = vel_next if vel_next is not None else vel_a
    flds = [vel_a, vel_b, target]
    use_recon = recon is not None and scheme != "euler"
    if use_recon:
        flds = list(recon[0])
    all32 = all(np.asarray(f.u).dtype == np.float32 and np.asarray(f.v).dtype == np.float32
                and (f.w is None or np.asarray(f.w).dtype == np.float32)
                and (getattr(f, "az", None) is None or np.asarray(f.az).dtype == np.float32) for f in flds)
    dtype = np.float32 if all32 else np.float64
    arrs = [_field_arrays(f, dtype) for f in flds]
    of = OField()
    (of.ua, of.va, of.wa), (of.ub, of.vb, of.wb), (of.ut, of.vt, of.wt) = [tuple(_p(x) for x in a) for a in arrs[:3]]
    if use_recon:
        of.pchip = 1
        of.ud, of.vd, of.wd = (_p(x) for x in arrs[3])
        for k in range(4):
            of.pt[k] = float(recon[1][k])
    of.f32 = 1 if all32 else 0
    of.alpha0 = alpha0
    of.n = view.lon.size
    if uv_interp in ("leastsq", "edge_leastsq"):   # element-centre u/v (interpolate.py:52-354, 644-750, 2588-2747)
        if view.ec_lon is None:
            raise ValueError(f"uv_interp {uv_interp!r} needs the mesh's element centres")
        of.lsq = 1
        if uv_interp == "edge_leastsq":
            if view.enb is None:
                raise ValueError("uv_interp 'edge_leastsq' needs the mesh's element neighbours")
            of.lsq = 2 if edge_leastsq_bc == "freeslip" else 3
        of.n = view.ec_lon.size
        if arrs[0][2] is not None:   # 3-D: u/v (K-1, E) and w (K, N) share the stride max(E, N)
            S = max(view.ec_lon.size, view.lon.size)
            pad = lambda x: None if x is None else np.ascontiguousarray(
                np.pad(x, [(0, 0)] * (x.ndim - 1) + [(0, S - x.shape[-1])]))
            arrs = [tuple(pad(x) for x in a) for a in arrs]
            (of.ua, of.va, of.wa), (of.ub, of.vb, of.wb), (of.ut, of.vt, of.wt) = [tuple(_p(x) for x in a)
                                                                                    for a in arrs[:3]]
            if use_recon:
                of.ud, of.vd, of.wd = (_p(x) for x in arrs[3])
            of.n = S
    elif uv_interp != "barycentric":
        raise ValueError(f"uv_interp {uv_interp!r}: the oracle restates 'barycentric', 'leastsq' and "
                         "'edge_leastsq'")
    etas = [np.ascontiguousarray(getattr(f, "eta", None) if getattr(f, "eta", None) is not None
                                 else np.zeros(view.lon.size), dtype=np.float64) for f in flds]
    of.etaa, of.etab, of.etat = (_p(e) for e in etas[:3])
    if use_recon:
        of.etad = _p(etas[3])
    is3d = arrs[0][2] is not None
    placement = getattr(vel_a, "uv_vertical", "layer")
    if is3d and placement != "layer":
        view.use_placement(placement)
    os_ = OStep()
    os_.scheme = {"euler": 0, "rk2": 1, "rk4": 2}[scheme]
    os_.dims = 3 if is3d else 2
    os_.w_code = {"nearest": 0, "barycentric": 1, "leastsq": 2, "idw": 3}[w_interp]
    os_.uv_dl = 1 if (is3d and placement != "layer") else 0
    cc = {"euler": (0.0,), "rk2": (0.0, 0.5), "rk4": (0.0, 0.5, 0.5, 1.0)}[scheme]
    if use_recon:   # the stage times sim_time + time_dir * c * dt
        q, d = float(recon[2]), float(recon[3])
        for k, c in enumerate(cc):
            os_.ak[k] = q + d * c * float(dt)
    elif vel_next is not None and scheme != "euler":
        for k, c in enumerate(cc):
            os_.ak[k] = float(c) * float(dt) / float(dt_to_next)
    os_.dt, os_.td = float(dt), float(time_dir)
    os_.Dmin, os_.z0b_min = float(Dmin), float(z0b_min)
    if use_recon:   # the end-of-step surface: the reconstruction at c = 1 (integrators.py:1369-1391)
        os_.alpha_end = float(recon[2]) + float(recon[3]) * 1.0 * float(dt)
    elif vel_next is not None:   # the end-of-step surface (integrators.py:1400-1420 _sigma_end_eta)
        os_.alpha_end = float(dt) / float(dt_to_next)
    # the tracking layer's surfaces of a sigma step (integrators.py:1381-1441)
    sig_keep = [None if e is None else np.ascontiguousarray(e, dtype=np.float64) for e in (eta_start, eta_end)]
    os_.eta_s, os_.eta_e = (_p(e) for e in sig_keep)
    os_.sig_steady = 1 if (not use_recon and vel_next is None) else 0
    if diffusion is not None:
        os_.seed, os_.real_id, os_.step_i = int(diffusion.seed), int(diffusion.real_id), int(diffusion.step_i)
        os_.pid_offset = int(getattr(diffusion, "pid_offset", 0))
    if diffusion is not None and not (float(diffusion.kh_x) == 0.0 and float(diffusion.kh_y) == 0.0):
        os_.kick = 1
        os_.kh_x, os_.kh_y = float(diffusion.kh_x), float(diffusion.kh_y)
    keep_az = []
    if diffusion is not None and getattr(diffusion, "az_enabled", False):
        # integrators.py:842-938: the payload's Az field, else the constant
        az_a = getattr(vel_a, "az", None)
        az_b = getattr(vel_b, "az", None) if hasattr(vel, "vel_a") else az_a
        have = az_a is not None and az_b is not None
        az_const = max(float(getattr(diffusion, "az_const", 0.0)), 0.0)
        if not have and getattr(diffusion, "az_requires_field", False):
            raise ValueError("diffusion.var_az is configured but the payload carries no az field")
        if have or az_const != 0.0:
            if not is3d:
                raise ValueError("diffusion.az_enabled requires a 3-D run")
            os_.az_on = 1
            os_.az_const = az_const
            if have:
                os_.az_field = 1
                keep_az = [np.ascontiguousarray(az_a, dtype=dtype), np.ascontiguousarray(az_b, dtype=dtype)]
                if of.lsq and of.n != view.lon.size:   # the shared stride of 3-D element-layout fields
                    keep_az = [np.ascontiguousarray(np.pad(a, [(0, 0)] * (a.ndim - 1) + [(0, of.n - a.shape[-1])]))
                               for a in keep_az]
                of.aza, of.azb = _p(keep_az[0]), _p(keep_az[1])
    P = state.lon.shape[0]
    out = {"lon": np.array(state.lon, dtype=np.float64), "lat": np.array(state.lat, dtype=np.float64),
           "z": np.array(state.z, dtype=np.float64), "status": np.array(state.status, dtype=np.int32),
           "nearest_node": np.array(state.nearest_node, dtype=np.int32),
           "failure_reason": (np.zeros(P, np.int8) if state.failure_reason is None
                              else np.array(state.failure_reason, dtype=np.int8)),
           "u": np.zeros(P), "v": np.zeros(P), "w": np.zeros(P)}
    pid_a = None if pid is None else np.ascontiguousarray(pid, dtype=np.int64)
    rs = None if release_step is None else np.ascontiguousarray(release_step, dtype=np.int32)
    elem = getattr(state, "elem", None)
    if elem is not None:
        if view.enb is None:
            raise ValueError("walk mode needs mesh._elem_neighbors (build_elem_neighbors)")
        out["elem"] = np.array(elem, dtype=np.int32)
    lib().orc_step(C.byref(view.s), C.byref(of), C.byref(os_), P,
                   _p(out["lon"]), _p(out["lat"]), _p(out["z"]), _p(out["status"]), _p(out["nearest_node"]),
                   _p(out["failure_reason"]), _p(out["u"]), _p(out["v"]), _p(out["w"]), _p(pid_a), _p(rs),
                   int(global_step), _p(out.get("elem")))
    return out


class OBeach(C.Structure):
    _fields_ = [("use_depth", C.c_int), ("use_coastal", C.c_int), ("use_stochastic", C.c_int),
                ("on_failure", C.c_int), ("resuspension", C.c_int), ("min_wet_steps", C.c_int),
                ("depth_min", C.c_double), ("zone_depth", C.c_double), ("rewet_hysteresis", C.c_double),
                ("p_beach", C.c_double), ("p_resusp", C.c_double),
                ("seed", C.c_uint64), ("real_id", C.c_uint64), ("step_i", C.c_uint64), ("pid_offset", C.c_uint64)]


RESUSP = {"never": 0, "auto": 1, "stochastic": 2, "auto_or_stochastic": 3}


def beach(state, prev_status, mesh, coastal, wet_streak, *, criteria, depth_min, zone_depth, t_beach,
          resuspension, rewet_hysteresis, min_wet_steps, t_resuspend, seed, real_id, step_i, dt, pid_offset=0,
          view=None, eta=None, dry_mask=None):
    """The beaching hook after one step; returns (state dict, wet_streak)."""
    view = view or MeshView(mesh)
    a = OBeach()
    a.use_depth, a.use_coastal = int("depth" in criteria), int("coastal_element" in criteria)
    a.use_stochastic, a.on_failure = int("stochastic" in criteria), int("on_failure" in criteria)
    a.resuspension, a.min_wet_steps = RESUSP[resuspension], int(min_wet_steps)
    a.depth_min, a.zone_depth, a.rewet_hysteresis = float(depth_min), float(zone_depth), float(rewet_hysteresis)
    a.p_beach = float(1.0 - np.exp(-abs(dt) / t_beach)) if t_beach else 0.0
    a.p_resusp = float(1.0 - np.exp(-abs(dt) / t_resuspend)) if t_resuspend else 0.0
    a.seed, a.real_id, a.step_i, a.pid_offset = int(seed), int(real_id), int(step_i), int(pid_offset)
    out = {"status": np.array(state.status, np.int32), "nearest_node": np.array(state.nearest_node, np.int32),
           "failure_reason": np.array(state.failure_reason, np.int8)}
    prev = np.ascontiguousarray(prev_status, np.int32)
    ws = np.array(wet_streak, np.int32)
    cst = np.ascontiguousarray(coastal, np.uint8)
    lon = np.ascontiguousarray(state.lon, np.float64)
    lat = np.ascontiguousarray(state.lat, np.float64)
    e = None if eta is None else np.ascontiguousarray(eta, np.float64)
    d = None if dry_mask is None else np.ascontiguousarray(dry_mask, np.float64)
    lib().orc_beach(C.byref(view.s), C.byref(a), _p(cst), lon.size, _p(lon), _p(lat), _p(out["status"]),
                    _p(prev), _p(out["nearest_node"]), _p(out["failure_reason"]), _p(ws), _p(e), _p(d))
    return out, ws


def walk(mesh, lon, lat, start, nn, view=None) -> np.ndarray:
    """find_containing_elements_walk (mesh.py:2631-2712): containing element
    of every point, walked from ``start``, with the global fallbacks."""
    view = view or MeshView(mesh)
    lon = np.ascontiguousarray(lon, dtype=np.float64)
    lat = np.ascontiguousarray(lat, dtype=np.float64)
    st = np.ascontiguousarray(start, dtype=np.int32)
    nn = np.ascontiguousarray(nn, dtype=np.int32)
    out = np.empty(lon.size, np.int32)
    lib().orc_walk(C.byref(view.s), lon.size, _p(lon), _p(lat), _p(st), _p(nn), _p(out))
    return out


def find_nearest(mesh, lon, lat, view=None) -> np.ndarray:
    view = view or MeshView(mesh)
    lon = np.ascontiguousarray(lon, dtype=np.float64)
    lat = np.ascontiguousarray(lat, dtype=np.float64)
    out = np.empty(lon.size, np.int32)
    lib().orc_find_nearest(C.byref(view.s), lon.size, _p(lon), _p(lat), _p(out))
    return out


def cell_stats(mesh, cum, cell, lon_min, lat_min, nx, ny, wrap, lon, lat, nn, view=None):
    """mesh.py:384-461 _gh_sample_stats of one candidate grid: (occ, cost,
    unprov, approx) of every sample, cum the candidate's (ny+1, nx+1) prefix
    table of node counts."""
    view = view or MeshView(mesh)
    cum = np.ascontiguousarray(cum, dtype=np.int32)
    lon = np.ascontiguousarray(lon, dtype=np.float64)
    lat = np.ascontiguousarray(lat, dtype=np.float64)
    nn = np.ascontiguousarray(nn, dtype=np.int32)
    P = lon.size
    occ = np.empty(P, np.int64)
    cost = np.empty(P, np.float64)
    unprov = np.empty(P, np.int8)
    approx = np.empty(P, np.int8)
    lib().orc_cell_stats(C.byref(view.s), _p(cum), float(cell), float(lon_min), float(lat_min), int(nx), int(ny),
                         int(bool(wrap)), P, _p(lon), _p(lat), _p(nn), _p(occ), _p(cost), _p(unprov), _p(approx))
    return occ, cost, unprov, approx


def contain(mesh, lon, lat, nn, view=None) -> np.ndarray:
    view = view or MeshView(mesh)
    lon = np.ascontiguousarray(lon, dtype=np.float64)
    lat = np.ascontiguousarray(lat, dtype=np.float64)
    nn = np.ascontiguousarray(nn, dtype=np.int32)
    out = np.empty(lon.size, np.int32)
    lib().orc_contain(C.byref(view.s), lon.size, _p(lon), _p(lat), _p(nn), _p(out))
    return out


def normals(P, seed, real_id, step_i, pid_offset=0, comp=0) -> np.ndarray:
    g = np.empty((P, 2))
    lib().orc_normals(P, seed, real_id, step_i, pid_offset, comp, _p(g))
    return g


def node_xyz(lon, lat) -> np.ndarray:
    lon = np.ascontiguousarray(lon, dtype=np.float64)
    lat = np.ascontiguousarray(lat, dtype=np.float64)
    out = np.empty((lon.size, 3))
    lib().orc_node_xyz(lon.size, _p(lon), _p(lat), _p(out))
    return out


SAMPLE_METHODS = {"nearest": 0, "leastsq": 1, "barycentric": 2, "idw": 3}


def sample_field(values, mesh, lon, lat, z=None, *, nearest=None, alive=None, method="leastsq", view=None, eta=None,
                 Dmin=0.5):
    """sampling.py:727 sample_field for a node field of shape (N,), a
    z-level mid-layer field (K-1, N) or an interface field (K, N): the
    oracle's restatement."""
    view = view or MeshView(mesh)
    values = np.ascontiguousarray(values, dtype=np.float64)
    lon = np.ascontiguousarray(lon, dtype=np.float64)
    lat = np.ascontiguousarray(lat, dtype=np.float64)
    P = lon.size
    if nearest is None:
        nearest = find_nearest(mesh, lon, lat, view)
    nearest = np.ascontiguousarray(nearest, dtype=np.int32)
    al = None if alive is None else np.ascontiguousarray(alive, dtype=np.uint8)
    rows, zm, zz = 0, None, None
    if values.ndim == 2 and getattr(mesh, "vertical_coord", "zlevel") == "sigma":   # sampling.py:620-723
        out = np.empty(P)
        et = np.ascontiguousarray(eta, dtype=np.float64)
        zz = np.ascontiguousarray(z, dtype=np.float64)
        lib().orc_sample_sigma(C.byref(view.s), _p(values), values.shape[0], _p(et), float(Dmin), P, _p(lon),
                               _p(lat), _p(zz), _p(nearest), _p(al), SAMPLE_METHODS[method], _p(out))
        return out
    if values.ndim == 2:
        zl = np.abs(np.asarray(mesh.sigma, dtype=np.float64))
        rows = values.shape[0]
        # a mid-layer field (K-1, N) has its mid-layer depths; an interface
        # field (K, N) none (the W interpolation reads the z-levels)
        zm = None if rows == zl.size else np.ascontiguousarray(0.5 * (zl[:-1] + zl[1:]))
        zz = np.ascontiguousarray(z, dtype=np.float64)
    out = np.empty(P)
    lib().orc_sample(C.byref(view.s), _p(values), rows, _p(zm), P, _p(lon), _p(lat), _p(zz), _p(nearest), _p(al),
                     SAMPLE_METHODS[method], _p(out))
    return out
