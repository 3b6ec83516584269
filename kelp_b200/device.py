"""Device-resident state behind the step functions: one CUDA context with the
uploaded mesh, a ring of velocity snapshots and the particle arrays.

Uploads are cached by object identity (a strong reference is kept, so an id
is never reused while cached): a run that steps the same mesh and snapshots
every step pays each upload once.  Particles travel every ``step()`` call
(the reference's per-call contract returns fresh arrays); the multi-step
driver in ``tracking`` keeps them resident instead.
"""
from __future__ import annotations

import ctypes as C
from collections import OrderedDict
from typing import Optional

import numpy as np

from . import _native as N

N_SLOTS = 8


def _c(a, dtype):
    return np.ascontiguousarray(a, dtype=dtype)


def _pad_to(a, n):
    """``a`` with its last axis zero-padded to ``n`` (unchanged when it is)."""
    if a.shape[-1] == n:
        return a
    return np.ascontiguousarray(np.pad(a, [(0, 0)] * (a.ndim - 1) + [(0, n - a.shape[-1])]))


def _shared_stride(u, v, w):
    """3-D element-layout u/v (K-1, E) with node w (K, N): both padded to the
    row stride max(E, N) the least-squares kernels read them with."""
    if w is None or w.ndim != 2 or u.shape[-1] == w.shape[-1]:
        return u, v, w
    n = max(u.shape[-1], w.shape[-1])
    return _pad_to(u, n), _pad_to(v, n), _pad_to(w, n)


def mesh_desc(mesh, keep: list) -> N.MeshDesc:
    """Fill the C mesh descriptor from a mesh (duck-typed: a kelp_b200 Mesh or
    KELP's own ``kelp.core.mesh.Mesh`` after ``build_search``).  Arrays that
    need a dtype conversion are appended to ``keep`` so they outlive the call."""
    if getattr(mesh, "_gh_offsets", None) is None:
        raise RuntimeError("mesh has no grid hash: call build_search(mesh) first")
    from .mesh import ensure_node_xyz
    xyz = ensure_node_xyz(mesh)

    def k(a, dt):
        a = _c(a, dt)
        keep.append(a)
        return a

    lon = k(mesh.nodes_lon, np.float64)
    lat = k(mesh.nodes_lat, np.float64)
    en = k(mesh.elem_nodes, np.int32)
    n2e = k(mesh.node_to_elems, np.int32)
    cnt = k(mesh.node_to_elems_count, np.int32)
    off = k(mesh._gh_offsets, np.int32)
    ids = k(mesh._gh_node_ids, np.int32)
    xyz = k(xyz, np.float64)
    depth = k(mesh.depth, np.float64) if getattr(mesh, "depth", None) is not None else None
    sigma = np.asarray(getattr(mesh, "sigma", np.zeros(0)))
    zl = None
    if sigma.size > 0 and getattr(mesh, "vertical_coord", "zlevel") == "zlevel":
        zl = k(np.abs(sigma), np.float64)
    d = N.MeshDesc()
    d.n_nodes = lon.shape[0]
    d.n_elems = en.shape[0]
    d.max_v = en.shape[1]
    d.max_conn = n2e.shape[1] if n2e.ndim == 2 else 0
    d.nodes_lon, d.nodes_lat = N.ptr(lon), N.ptr(lat)
    d.depth = N.ptr(depth)
    d.elem_nodes, d.node_to_elems, d.node_to_elems_count = N.ptr(en), N.ptr(n2e), N.ptr(cnt)
    d.gh_offsets, d.gh_node_ids, d.node_xyz = N.ptr(off), N.ptr(ids), N.ptr(xyz)
    d.gh_cell_size = float(mesh._gh_cell_size)
    d.gh_lon_min = float(mesh._gh_lon_min)
    d.gh_lat_min = float(mesh._gh_lat_min)
    d.gh_nx, d.gh_ny = int(mesh._gh_nx), int(mesh._gh_ny)
    d.gh_wrap_lon = 1 if mesh._gh_wrap_lon else 0
    d.gh_far_rows = int(mesh._gh_far_rows)
    d.exact_nearest = 1 if (getattr(mesh, "metadata", None) or {}).get("exact_nearest", False) else 0
    d.r_earth = float(getattr(mesh, "r_earth", 6371000.0))
    d.z_levels = N.ptr(zl)
    d.n_levels = 0 if zl is None else int(zl.shape[0])
    return d


class DeviceContext:
    """One CUDA device context of the native library."""

    def __init__(self, device: int = 0):
        L = N.lib()
        p = C.c_void_p()
        rc = L.kc_create(int(device), C.byref(p))
        if rc:
            raise N.KcError(rc, f"kc_create(device={device}) failed: no usable CUDA device")
        self._ctx = p
        self.device = device
        self._mesh_ref = None
        self._mesh_key = None
        self._slots: "OrderedDict[int, tuple]" = OrderedDict()   # id(field) -> (slot, field)
        self.P = 0

    # -- plumbing ---------------------------------------------------------
    def _chk(self, rc, what):
        N.check(self._ctx, rc, what)

    def close(self):
        if self._ctx:
            N.lib().kc_destroy(self._ctx)
            self._ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        return self._ctx

    def synchronize(self):
        self._chk(N.lib().kc_synchronize(self._ctx), "kc_synchronize")
        self._inflight = []

    # -- mesh ---------------------------------------------------------------
    def ensure_mesh(self, mesh) -> None:
        from .mesh import ensure_node_xyz
        if getattr(mesh, "_gh_offsets", None) is not None:
            ensure_node_xyz(mesh)
        key = (id(mesh), id(mesh._gh_offsets), id(getattr(mesh, "_node_xyz", None)),
               bool((mesh.metadata or {}).get("exact_nearest", False)))
        if self._mesh_key == key and self._mesh_ref is mesh:
            return
        keep: list = []
        d = mesh_desc(mesh, keep)
        self._chk(N.lib().kc_mesh_upload(self._ctx, C.byref(d)), "kc_mesh_upload")
        self._cg_nynx = None
        if getattr(mesh, "_nemo_cgrid", False):
            self._upload_cgrid(mesh)
        self._sigma = getattr(mesh, "vertical_coord", "zlevel") == "sigma" and not getattr(mesh, "_nemo_cgrid", False)
        if self._sigma:
            sg = _c(mesh.sigma, np.float64)
            self._chk(N.lib().kc_sigma_upload(self._ctx, int(sg.size), N.ptr(sg)), "kc_sigma_upload")
        self._mesh_ref = mesh
        self._mesh_key = key
        self._slots.clear()
        self._dl_key = None
        self._coastal_key = None
        self._enb_key = None

    def _upload_cgrid(self, mesh) -> None:
        """The NEMO C-grid tables of a build_nemo_cgrid_mesh mesh (kc_cgrid_upload)."""
        g = lambda name, t: _c(np.asarray(getattr(mesh, "_nemo_cgrid_" + name)).reshape(-1), t)
        ny, nx = (int(x) for x in mesh._structured_shape)
        zw = g("zw", np.float64)
        K = max(int(zw.size) - 1, 0)
        keep = {"corners": g("corners", np.int32), "ji": g("elem_ji", np.int64), "nlev": g("nlev", np.int32),
                "nlev_r": g("nlev_raster", np.int32), "e2u": g("e2u", np.float64), "e1v": g("e1v", np.float64),
                "area": g("area", np.float64), "zw": zw, "e3b": g("e3b", np.float64), "kbu": g("kbu", np.int32),
                "e3u": g("e3u", np.float64), "kbv": g("kbv", np.int32), "e3v": g("e3v", np.float64)}
        d = N.CgridDesc()
        d.ny, d.nx, d.K = ny, nx, K
        d.partial_shrunk = int(getattr(mesh, "_nemo_cgrid_partial", "shrunk") == "shrunk")
        d.corners, d.elem_ji, d.nlev, d.nlev_raster = (N.ptr(keep[k]) for k in ("corners", "ji", "nlev", "nlev_r"))
        if keep["e2u"].size:
            d.e2u, d.e1v = N.ptr(keep["e2u"]), N.ptr(keep["e1v"])
        if K > 0:
            d.area, d.zw, d.e3b = N.ptr(keep["area"]), N.ptr(zw), N.ptr(keep["e3b"])
            d.kbu, d.e3u, d.kbv, d.e3v = (N.ptr(keep[k]) for k in ("kbu", "e3u", "kbv", "e3v"))
        self._chk(N.lib().kc_cgrid_upload(self._ctx, C.byref(d)), "kc_cgrid_upload")
        self._cg_nynx = ny * nx

    def ensure_elem_neighbors(self, mesh) -> None:
        """Upload the edge-neighbour table of the resident mesh (built by
        mesh.build_elem_neighbors on first use; cached)."""
        from .mesh import build_elem_neighbors
        self.ensure_mesh(mesh)
        if getattr(self, "_enb_key", None) == self._mesh_key:
            return
        enb = np.ascontiguousarray(build_elem_neighbors(mesh), dtype=np.int32)
        self._chk(N.lib().kc_elem_neighbors_upload(self._ctx, int(enb.shape[1]), N.ptr(enb)),
                  "kc_elem_neighbors_upload")
        self._enb_key = self._mesh_key

    def ensure_elem_centers(self, mesh) -> None:
        """Upload the element centres of the resident mesh (the least-squares
        u/v's stencil points; cached)."""
        self.ensure_mesh(mesh)
        if getattr(self, "_ec_key", None) == self._mesh_key:
            return
        lon = _c(mesh.elem_center_lon, np.float64)
        lat = _c(mesh.elem_center_lat, np.float64)
        E = np.asarray(mesh.elem_nodes).shape[0]
        if lon.shape != (E,) or lat.shape != (E,):
            raise ValueError(f"elem_center_lon/lat must hold the mesh's {E} elements, got {lon.shape}, {lat.shape}")
        self._chk(N.lib().kc_elem_centers_upload(self._ctx, N.ptr(lon), N.ptr(lat)), "kc_elem_centers_upload")
        self._ec_key = self._mesh_key

    def ensure_depth_points(self, mesh, placement: str) -> int:
        """Upload the depth-linear data-point table of ``mesh`` for
        ``placement`` (cached); returns its number of points M."""
        self.ensure_mesh(mesh)
        key = (self._mesh_key, placement, id(getattr(mesh, "depth", None)))
        if getattr(self, "_dl_key", None) == key:
            return self._dl_M
        from .vertical_uv import depth_points
        dp = depth_points(mesh, placement)
        p = _c(dp.p, np.float64)
        last = _c(dp.last, np.int32)
        bed = _c(dp.bed, np.float64)
        self._chk(N.lib().kc_depth_points_upload(self._ctx, int(p.size), N.ptr(p), N.ptr(last), N.ptr(bed)),
                  "kc_depth_points_upload")
        self._dl_key = key
        self._dl_M = int(p.size)
        return self._dl_M

    # -- snapshot ring --------------------------------------------------------
    def upload_field(self, field, slot: int, dtype=None) -> None:
        """Upload one snapshot into ring slot ``slot``: float32 or float64
        storage, or ``np.float16`` for half storage with per-row power-of-two
        scales (converted on the device from float32)."""
        u = np.asarray(field.u)
        v = np.asarray(field.v)
        w = None if getattr(field, "w", None) is None else np.asarray(field.w)
        if getattr(field, "uv_layout", None) == "nemo_cgrid" and getattr(self, "_cg_nynx", None):
            # face rasters: one row per level of ny * nx values
            nynx = self._cg_nynx
            u = u.reshape(-1, nynx) if u.ndim > 1 or u.size != nynx else u
            v = v.reshape(-1, nynx) if v.ndim > 1 or v.size != nynx else v
            w = None if w is None else w.reshape(-1, nynx)
        if dtype is None:
            dtype = np.float32 if (u.dtype == np.float32 and v.dtype == np.float32
                                   and (w is None or w.dtype == np.float32)) else np.float64
        code = {np.dtype(np.float32): N.KC_F32, np.dtype(np.float64): N.KC_F64,
                np.dtype(np.float16): N.KC_F16}[np.dtype(dtype)]
        host = np.float32 if code == N.KC_F16 else dtype
        u = _c(u, host)
        v = _c(v, host)
        w = None if w is None else _c(w, host)
        u, v, w = _shared_stride(u, v, w)
        n = u.shape[-1]
        rows = 1 if u.ndim == 1 else u.shape[0]
        wrows = 0 if w is None else (1 if w.ndim == 1 else w.shape[0])
        self._chk(N.lib().kc_field_upload(self._ctx, slot, code, n, rows, N.ptr(u), N.ptr(v), wrows, N.ptr(w)),
                  "kc_field_upload")
        if getattr(self, "_sigma", False) and w is not None:
            # the free surface of the sigma step's column heights (float64)
            eta = getattr(field, "eta", None)
            eta = np.zeros(n) if eta is None else _c(np.asarray(eta), np.float64)
            if eta.shape != (n,):
                raise ValueError(f"eta of shape {eta.shape} does not match the mesh's {n} nodes")
            self._chk(N.lib().kc_field_upload_eta(self._ctx, slot, n, N.ptr(eta)), "kc_field_upload_eta")
        az = getattr(field, "az", None)
        if az is not None and code != N.KC_F16:
            az = _pad_to(_c(np.asarray(az), host), n)
            self._chk(N.lib().kc_field_upload_az(self._ctx, slot, code, n, 1 if az.ndim == 1 else az.shape[0],
                                                 N.ptr(az)), "kc_field_upload_az")
        self.synchronize()

    def prefetch(self, fields, storage=None, busy=()) -> int:
        """Start uploading the ``fields`` a coming step will read into free
        ring slots (or the least recently used ones outside ``busy`` and the
        last step's), without waiting: kc_field_upload_async, ordered after
        the launches that read those slots.  float16 storage, eta and Az rows
        upload at the step instead.  Returns the number of uploads started."""
        dtype = self._slot_dtype(fields, storage)
        if dtype == np.dtype(np.float16) or getattr(self, "_sigma", False):
            return 0
        keep = set(busy) | set(getattr(self, "_last_slots", ()))
        started = 0
        for f in fields:
            key = (id(f), dtype)
            if key in self._slots or getattr(f, "az", None) is not None:
                keep.update(s for k, (s, _) in self._slots.items() if k == key)
                continue
            if getattr(f, "uv_layout", None) == "nemo_cgrid":
                return started
            used = {s for s, _ in self._slots.values()}
            free = [s for s in range(N_SLOTS) if s not in used and s not in keep]
            if free:
                slot = free[0]
            else:
                victims = [k for k, (s, _) in self._slots.items() if s not in keep]
                if not victims:
                    return started
                slot = self._slots.pop(victims[0])[0]
            u = _c(np.asarray(f.u), dtype)
            v = _c(np.asarray(f.v), dtype)
            w = None if getattr(f, "w", None) is None else _c(np.asarray(f.w), dtype)
            u, v, w = _shared_stride(u, v, w)
            code = N.KC_F32 if dtype == np.dtype(np.float32) else N.KC_F64
            rows = 1 if u.ndim == 1 else u.shape[0]
            wrows = 0 if w is None else (1 if w.ndim == 1 else w.shape[0])
            self._chk(N.lib().kc_field_upload_async(self._ctx, slot, code, u.shape[-1], rows, N.ptr(u), N.ptr(v),
                                                    wrows, N.ptr(w)), "kc_field_upload_async")
            self._inflight = getattr(self, "_inflight", []) + [(u, v, w)]   # alive until the copies are done
            self._slots[key] = (slot, f)
            keep.add(slot)
            started += 1
        return started

    def _slot_dtype(self, fields, storage):
        all32 = all(np.asarray(f.u).dtype == np.float32 and np.asarray(f.v).dtype == np.float32
                    and (f.w is None or np.asarray(f.w).dtype == np.float32)
                    and (getattr(f, "az", None) is None or np.asarray(f.az).dtype == np.float32) for f in fields)
        return np.dtype(storage) if storage is not None else np.dtype(np.float32 if all32 else np.float64)

    def slots_for(self, fields, storage=None) -> list:
        """Ring slots holding ``fields`` (uploading the ones not resident).
        All fields of one step share one element type: float32 only when every
        one of them is float32, unless ``storage`` names it (``np.float16``:
        half storage with per-row scales)."""
        dtype = self._slot_dtype(fields, storage)
        out = []
        pinned = set()
        for f in fields:
            key = (id(f), dtype)
            if key in self._slots:
                self._slots.move_to_end(key)
                slot = self._slots[key][0]
            else:
                used = {s for s, _ in self._slots.values()}
                free = [s for s in range(N_SLOTS) if s not in used]
                if free:
                    slot = free[0]
                else:
                    victim = next(k for k, (s, _) in self._slots.items() if s not in pinned)
                    slot = self._slots.pop(victim)[0]
                self.upload_field(f, slot, dtype)
                self._slots[key] = (slot, f)
            pinned.add(slot)
            out.append(slot)
        self._last_slots = tuple(out)
        return out

    # -- particles ------------------------------------------------------------
    def upload_particles(self, lon, lat, z, status, nn, fr=None, pid=None, release_step=None):
        lon = _c(lon, np.float64)
        lat = _c(lat, np.float64)
        z = None if z is None else _c(z, np.float64)
        status = _c(status, np.int32)
        nn = _c(nn, np.int32)
        fr = None if fr is None else _c(fr, np.int8)
        pid = None if pid is None else _c(pid, np.int64)
        rs = None if release_step is None else _c(release_step, np.int32)
        P = lon.shape[0]
        self._chk(N.lib().kc_particles_upload(self._ctx, P, N.ptr(lon), N.ptr(lat), N.ptr(z), N.ptr(status),
                                              N.ptr(nn), N.ptr(fr), N.ptr(pid), N.ptr(rs)),
                  "kc_particles_upload")
        self.P = P

    def download_status(self) -> np.ndarray:
        """The statuses of the resident particles (upload order)."""
        out = np.empty(self.P, np.int32)
        self._chk(N.lib().kc_particles_download(self._ctx, self.P, None, None, None, N.ptr(out), None, None, None,
                                                None, None), "kc_particles_download")
        return out

    def download_particles(self) -> dict:
        P = self.P
        out = {"lon": np.empty(P), "lat": np.empty(P), "z": np.empty(P),
               "status": np.empty(P, np.int32), "nearest_node": np.empty(P, np.int32),
               "failure_reason": np.empty(P, np.int8),
               "u": np.empty(P), "v": np.empty(P), "w": np.empty(P)}
        self._chk(N.lib().kc_particles_download(
            self._ctx, P, N.ptr(out["lon"]), N.ptr(out["lat"]), N.ptr(out["z"]), N.ptr(out["status"]),
            N.ptr(out["nearest_node"]), N.ptr(out["failure_reason"]), N.ptr(out["u"]), N.ptr(out["v"]),
            N.ptr(out["w"])), "kc_particles_download")
        return out

    # -- beaching ----------------------------------------------------------------
    def ensure_coastal(self, mesh, flags) -> None:
        """Upload the coastal element flags of the resident mesh (cached)."""
        self.ensure_mesh(mesh)
        key = (self._mesh_key, id(flags))
        if getattr(self, "_coastal_key", None) == key:
            return
        f = np.ascontiguousarray(flags, dtype=np.uint8)
        if f.shape != (np.asarray(mesh.elem_nodes).shape[0],):
            raise ValueError("coastal flags must have one entry per element")
        self._chk(N.lib().kc_coastal_upload(self._ctx, N.ptr(f)), "kc_coastal_upload")
        self._coastal_key = key

    def beach_state_upload(self, prev_status=None, wet_streak=None) -> None:
        prev = None if prev_status is None else _c(prev_status, np.int32)
        wet = None if wet_streak is None else _c(wet_streak, np.int32)
        for a in (prev, wet):
            if a is not None and a.shape != (self.P,):
                raise ValueError("beaching state arrays must have one entry per particle")
        self._chk(N.lib().kc_beach_state_upload(self._ctx, N.ptr(prev), N.ptr(wet)), "kc_beach_state_upload")

    def beach_state_download(self) -> np.ndarray:
        out = np.empty(self.P, np.int32)
        self._chk(N.lib().kc_beach_state_download(self._ctx, N.ptr(out)), "kc_beach_state_download")
        return out

    def beach_surface(self, eta=None, dry_mask=None) -> None:
        """kc_beach_surface: the node free surface and dry mask the next
        beaching calls read (None: off)."""
        e = None if eta is None else _c(eta, np.float64)
        d = None if dry_mask is None else _c(dry_mask, np.float64)
        n = None if self._mesh_ref is None else int(np.asarray(self._mesh_ref.nodes_lon).shape[0])
        for a in (e, d):
            if a is not None and (n is None or a.shape != (n,)):
                raise ValueError("beaching surfaces are node arrays (N,) of the uploaded mesh")
        self._chk(N.lib().kc_beach_surface(self._ctx, N.ptr(e), N.ptr(d)), "kc_beach_surface")

    def sigma_surfaces(self, eta_start=None, eta_end=None, steady: bool = False) -> None:
        """The tracking layer's surfaces at the start and end of the following
        sigma steps (kc_sigma_surfaces); None: the payload's own."""
        es = None if eta_start is None else _c(eta_start, np.float64)
        ee = None if eta_end is None else _c(eta_end, np.float64)
        n = None if self._mesh_ref is None else int(np.asarray(self._mesh_ref.nodes_lon).shape[0])
        for a in (es, ee):
            if a is not None and (n is None or a.shape != (n,)):
                raise ValueError("sigma surfaces are node arrays (N,) of the uploaded mesh")
        self._chk(N.lib().kc_sigma_surfaces(self._ctx, N.ptr(es), N.ptr(ee), int(bool(steady))),
                  "kc_sigma_surfaces")

    def sigma_surface_records(self, which: int, kind: int, slots=(), alpha: float = 0.0, times=None,
                              q: float = 0.0, steady: bool = False) -> None:
        """One tracking-layer surface (which 0 start, 1 end) evaluated on the
        device from resident slots (kc_sigma_surface_slots): kind 0 off,
        1 a record, 2 a linear blend at alpha, 3 PCHIP at time q."""
        sl = np.zeros(4, np.int32)
        sl[:len(slots)] = np.asarray(slots, dtype=np.int32)
        t = None if times is None else np.ascontiguousarray(times, dtype=np.float64)
        self._chk(N.lib().kc_sigma_surface_slots(self._ctx, int(which), int(kind), N.ptr(sl), float(alpha), N.ptr(t),
                                                 float(q), int(bool(steady))), "kc_sigma_surface_slots")

    def beach(self, args: N.BeachArgs) -> None:
        self._chk(N.lib().kc_beach(self._ctx, C.byref(args)), "kc_beach")

    # -- work -------------------------------------------------------------------
    def step(self, args: N.StepArgs) -> None:
        self._chk(N.lib().kc_step(self._ctx, C.byref(args)), "kc_step")

    def step_host(self, args: N.StepArgs, inp: dict, out: dict, chunk: int = 0) -> None:
        """One step of host-resident particles (kc_step_host): ``inp`` and
        ``out`` map lon, lat, z, status, nearest_node, failure_reason (and in
        ``out`` u, v, w) to C-contiguous arrays of the library's dtypes; absent
        or None entries are not read / not written.  Page-locked arrays
        (``pinned_empty``) let the copies overlap the step."""
        types = {"lon": np.float64, "lat": np.float64, "z": np.float64, "status": np.int32,
                 "nearest_node": np.int32, "failure_reason": np.int8, "u": np.float64, "v": np.float64,
                 "w": np.float64, "pid": np.int64, "real_id": np.int32, "release_step": np.int32,
                 "elem": np.int32}

        def pack(d, names):
            h = N.HostParticles()
            P = None
            for name in names:
                a = d.get(name)
                if a is None:
                    continue
                if a.dtype != types[name] or not a.flags.c_contiguous:
                    raise ValueError(f"{name}: expected a C-contiguous {np.dtype(types[name])} array")
                if P is None:
                    P = a.shape[0]
                elif a.shape[0] != P:
                    raise ValueError("host particle arrays of different lengths")
                setattr(h, name, a.ctypes.data)
            return h, P

        hi, P = pack(inp, ("lon", "lat", "z", "status", "nearest_node", "failure_reason", "pid", "real_id",
                           "release_step", "elem"))
        ho, P2 = pack(out, ("lon", "lat", "z", "status", "nearest_node", "failure_reason", "u", "v", "w",
                            "elem"))
        if P is None or P2 != P:
            raise ValueError("input and output particle counts differ")
        self._chk(N.lib().kc_step_host(self._ctx, C.byref(args), P, C.byref(hi), C.byref(ho), int(chunk)),
                  "kc_step_host")
        self.P = P

    def set_realization(self, real_id=None) -> None:
        """Per-particle realization ids of the resident particles (ensemble
        members in one array); None returns to the step's real_id."""
        rid = None if real_id is None else _c(real_id, np.int32)
        if rid is not None and rid.shape != (self.P,):
            raise ValueError("one realization id per resident particle")
        self._chk(N.lib().kc_particles_set_realization(self._ctx, N.ptr(rid)), "kc_particles_set_realization")

    def set_elem(self, elem=None) -> None:
        """Carried containing elements of the resident particles (elem_search
        walk; -1 = no guess); None returns to the local search.  Needs the
        neighbour table (ensure_elem_neighbors)."""
        e = None if elem is None else _c(elem, np.int32)
        if e is not None and e.shape != (self.P,):
            raise ValueError("one carried element per resident particle")
        self._chk(N.lib().kc_particles_set_elem(self._ctx, N.ptr(e)), "kc_particles_set_elem")

    def get_elem(self) -> np.ndarray:
        out = np.empty(self.P, np.int32)
        self._chk(N.lib().kc_particles_get_elem(self._ctx, self.P, N.ptr(out)), "kc_particles_get_elem")
        return out

    def sample_field(self, values, lon, lat, z=None, z_mids=None, nearest=None, alive=None,
                     method: int = 1) -> np.ndarray:
        """kc_sample_field: a node field (N,) or a mid-layer field (rows, N)
        with its mid-layer depths, sampled at the points (NaN for dead or
        anchorless ones)."""
        values = _c(values, np.float64)
        lon = _c(lon, np.float64)
        lat = _c(lat, np.float64)
        rows = values.shape[0] if values.ndim == 2 else 0
        zz = _c(z, np.float64) if rows else None
        zm = _c(z_mids, np.float64) if (rows and z_mids is not None) else None   # None: an interface field
        nn = None if nearest is None else _c(nearest, np.int32)
        al = None if alive is None else _c(np.asarray(alive).astype(np.uint8), np.uint8)
        out = np.empty(lon.shape[0], np.float64)
        self._chk(N.lib().kc_sample_field(self._ctx, N.ptr(values), rows, N.ptr(zm), lon.shape[0], N.ptr(lon),
                                          N.ptr(lat), N.ptr(zz), N.ptr(nn), N.ptr(al), int(method), N.ptr(out)),
                  "kc_sample_field")
        return out

    def sample_field_sigma(self, values, lon, lat, z, eta, Dmin, nearest=None, alive=None,
                           method: int = 1) -> np.ndarray:
        """kc_sample_field_sigma: an interface (K, N) or mid-layer (K-1, N)
        field on the resident sigma mesh with its free surface eta."""
        values = _c(values, np.float64)
        lon = _c(lon, np.float64)
        lat = _c(lat, np.float64)
        zz = _c(z, np.float64)
        et = _c(eta, np.float64)
        nn = None if nearest is None else _c(nearest, np.int32)
        al = None if alive is None else _c(np.asarray(alive).astype(np.uint8), np.uint8)
        out = np.empty(lon.shape[0], np.float64)
        self._chk(N.lib().kc_sample_field_sigma(self._ctx, N.ptr(values), values.shape[0], N.ptr(et), float(Dmin),
                                                lon.shape[0], N.ptr(lon), N.ptr(lat), N.ptr(zz), N.ptr(nn),
                                                N.ptr(al), int(method), N.ptr(out)), "kc_sample_field_sigma")
        return out

    def find_elements(self, lon, lat, nn=None) -> np.ndarray:
        """mesh.find_containing_elements on the device: the 1-ring / 2-ring
        scan around nn (None: the exact nearest node); -1 outside."""
        lon = _c(lon, np.float64)
        lat = _c(lat, np.float64)
        a = None if nn is None else _c(nn, np.int32)
        if lon.shape != lat.shape or (a is not None and a.shape != lon.shape):
            raise ValueError("lon, lat and nn must have the same length")
        out = np.empty(lon.shape[0], np.int32)
        self._chk(N.lib().kc_find_elements(self._ctx, lon.shape[0], N.ptr(lon), N.ptr(lat), N.ptr(a), N.ptr(out)),
                  "kc_find_elements")
        return out

    def find_elements_walk(self, lon, lat, start) -> np.ndarray:
        """mesh.find_containing_elements_walk on the device: the containing
        element of each point walked from start (-1: no guess); -1 outside."""
        lon = _c(lon, np.float64)
        lat = _c(lat, np.float64)
        st = _c(start, np.int32)
        if not (lon.shape == lat.shape == st.shape):
            raise ValueError("lon, lat and start must have the same length")
        out = np.empty(lon.shape[0], np.int32)
        self._chk(N.lib().kc_find_elements_walk(self._ctx, lon.shape[0], N.ptr(lon), N.ptr(lat), N.ptr(st),
                                                N.ptr(out)), "kc_find_elements_walk")
        return out

    def step_range(self, args: N.StepArgs, begin: int, count: int) -> None:
        """One step of the resident particles [begin, begin + count)."""
        self._chk(N.lib().kc_step_range(self._ctx, C.byref(args), int(begin), int(count)), "kc_step_range")

    def run_fused(self, steps, beach=None, graph: bool = True) -> None:
        """len(steps) steps in one kernel launch (kc_run_fused), the
        beaching hook after each when ``beach`` (one argument block per step)
        is given; ``graph`` replays a captured CUDA graph."""
        n = len(steps)
        arr = (N.StepArgs * n)(*steps)
        barr = None
        if beach is not None:
            if len(beach) != n:
                raise ValueError("one beaching argument block per step")
            barr = (N.BeachArgs * n)(*beach)
        self._chk(N.lib().kc_run_fused(self._ctx, arr, n, None if barr is None else C.cast(barr, C.c_void_p),
                                       int(bool(graph))), "kc_run_fused")

    def set_fused_block(self, block: int) -> None:
        """Particles per block of run_fused: 128 or 256."""
        self._chk(N.lib().kc_set_fused_block(self._ctx, int(block)), "kc_set_fused_block")

    def run(self, steps) -> None:
        arr = (N.StepArgs * len(steps))(*steps)
        self._chk(N.lib().kc_run(self._ctx, arr, len(steps)), "kc_run")

    def sort(self) -> None:
        """Re-order the resident particles by grid-hash cell (kc_sort)."""
        self._chk(N.lib().kc_sort(self._ctx), "kc_sort")

    def find_nearest(self, lon, lat) -> np.ndarray:
        lon = _c(lon, np.float64)
        lat = _c(lat, np.float64)
        out = np.empty(lon.shape[0], np.int32)
        self._chk(N.lib().kc_find_nearest(self._ctx, lon.shape[0], N.ptr(lon), N.ptr(lat), N.ptr(out)),
                  "kc_find_nearest")
        return out

    def rng_normals(self, P, seed, real_id, step_i, pid_offset=0, comp=0) -> np.ndarray:
        out = np.empty((int(P), 2))
        self._chk(N.lib().kc_rng_normals(self._ctx, int(P), int(seed), int(real_id), int(step_i), int(pid_offset),
                                         int(comp), N.ptr(out)), "kc_rng_normals")
        return out

    def grid_hash(self, lon, lat, cell_size, lon_min, lat_min, nx, ny, wrap):
        """(offsets, node_ids) of the grid hash built on the device
        (kc_grid_hash_build); lon in the branch the host chose."""
        lon = _c(lon, np.float64)
        lat = _c(lat, np.float64)
        off = np.empty(int(nx) * int(ny) + 1, np.int32)
        ids = np.empty(lon.size, np.int32)
        self._chk(N.lib().kc_grid_hash_build(self._ctx, lon.size, N.ptr(lon), N.ptr(lat), float(cell_size),
                                             float(lon_min), float(lat_min), int(nx), int(ny), int(bool(wrap)),
                                             N.ptr(off), N.ptr(ids)), "kc_grid_hash_build")
        return off, ids

    def grid_cell_stats(self, lon_branch, cell_size, lon_min, lat_min, nx, ny, wrap, lon, lat):
        """Per-sample statistics of one candidate grid-hash cell on the
        resident mesh (kc_grid_cell_stats): (nn, occ, cost, unprov, approx)."""
        lb = _c(lon_branch, np.float64)
        lon = _c(lon, np.float64)
        lat = _c(lat, np.float64)
        P = lon.size
        nn = np.empty(P, np.int32)
        occ = np.empty(P, np.int32)
        cost = np.empty(P, np.float64)
        unprov = np.empty(P, np.int8)
        approx = np.empty(P, np.int8)
        self._chk(N.lib().kc_grid_cell_stats(self._ctx, lb.size, N.ptr(lb), float(cell_size), float(lon_min),
                                             float(lat_min), int(nx), int(ny), int(bool(wrap)), P, N.ptr(lon),
                                             N.ptr(lat), N.ptr(nn), N.ptr(occ), N.ptr(cost), N.ptr(unprov),
                                             N.ptr(approx)), "kc_grid_cell_stats")
        return nn, occ, cost, unprov, approx

    def rng_domain_digests(self, corrected: bool = True) -> tuple:
        """Digests of r, cos and sin of the Box-Muller draws over all 2^32
        uniforms (kc_rng_domain_digests)."""
        out = np.zeros(3, np.uint64)
        self._chk(N.lib().kc_rng_domain_digests(self._ctx, 1 if corrected else 0, N.ptr(out)),
                  "kc_rng_domain_digests")
        return tuple(int(v) for v in out)

    def device_errors(self) -> int:
        w = C.c_int(0)
        self._chk(N.lib().kc_device_errors(self._ctx, C.byref(w)), "kc_device_errors")
        return int(w.value)

    def l2_flush(self, nbytes: int = 256 << 20) -> None:
        self._chk(N.lib().kc_l2_flush(self._ctx, int(nbytes)), "kc_l2_flush")

    def record(self, slot: int) -> None:
        self._chk(N.lib().kc_event_record(self._ctx, slot), "kc_event_record")

    def elapsed_ms(self, a: int, b: int) -> float:
        ms = C.c_float(0.0)
        self._chk(N.lib().kc_event_elapsed(self._ctx, a, b, C.byref(ms)), "kc_event_elapsed")
        return float(ms.value)


def pinned_empty(shape, dtype) -> np.ndarray:
    """A numpy array in page-locked host memory (freed when the array dies)."""
    dtype = np.dtype(dtype)
    n = int(np.prod(shape)) * dtype.itemsize
    p = C.c_void_p()
    rc = N.lib().kc_host_alloc(max(n, 1), C.byref(p))
    if rc:
        raise N.KcError(rc, "kc_host_alloc")
    buf = (C.c_char * max(n, 1)).from_address(p.value)
    arr = np.frombuffer(buf, dtype=dtype, count=int(np.prod(shape))).reshape(shape)
    import weakref
    weakref.finalize(buf, N.lib().kc_host_free, p)
    return arr


_default: Optional[DeviceContext] = None


_default_device = 0


def set_default_device(device: int) -> None:
    """Device of the process-wide context (one process per GPU: its local rank)."""
    global _default_device, _default
    if _default is not None and _default.device != device:
        _default.close()
        _default = None
    _default_device = int(device)


def default_context() -> DeviceContext:
    """The process-wide context (device 0 unless set_default_device was called),
    created on first use."""
    global _default
    if _default is None:
        _default = DeviceContext(_default_device)
    return _default
