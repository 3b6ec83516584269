"""The named benchmark workloads: seeded synthetic inputs with the shapes of
KELP's benchmark configurations, and the per-step schedule a run loop feeds
the step kernel (bracket snapshots, bracket fraction, stage alphas), built
like ``tracking._build_vel_payload`` (``src/kelp/tracking.py:3136-3206``) with
``on_exhausted: cycle`` (period = span of the records + one interval).
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import Callable, List, Optional

import numpy as np

from . import _native as N   # ctypes binding: the library itself is loaded on the first call
from . import synthetic as S


@dataclass
class Workload:
    name: str
    mesh: object
    snaps: list
    lon: np.ndarray
    lat: np.ndarray
    z: np.ndarray
    scheme: str
    dt: float
    interval: float                 # seconds between snapshots
    n_steps_run: int                # the configuration's horizon
    dims: int = 2
    w_interp: str = "nearest"
    kh: Optional[tuple] = None      # (kh_x, kh_y) of the split uniform kick
    seed: int = 0
    uv_vertical: str = "layer"      # 3-D u/v placement: layer, level or layer_linear
    # batched cohorts (one slot array for every cohort x ensemble member)
    pid: Optional[np.ndarray] = None           # RNG particle key per slot: its index within its cohort
    real_id: Optional[np.ndarray] = None       # realization (ensemble member) per slot
    release_step: Optional[np.ndarray] = None  # global step of the slot's release
    cohorts: Optional[list] = None             # (begin, count, member, cohort) blocks of the slot array
    t0_step: int = 0                           # first global step of the timed window
    description: dict = field(default_factory=dict)

    @property
    def P(self) -> int:
        return self.lon.size

    def bracket(self, k: int):
        """(idx_a, idx_b, alpha0, dt_to_next) of global step k (forward)."""
        n = len(self.snaps)
        t = k * self.dt
        period = n * self.interval
        tw = t - period * np.floor(t / period)
        ia = int(np.floor(tw / self.interval + 1e-9)) % n
        ta = ia * self.interval
        alpha = (tw - ta) / self.interval
        if abs(alpha) < 1e-12:
            alpha = 0.0
        return ia, (ia + 1) % n, alpha, (ta + self.interval) - tw

    def step_args(self, k: int, slots, precision: int = N.KC_PLAIN) -> N.StepArgs:
        ia, ib, alpha0, dtn = self.bracket(k)
        a = N.StepArgs()
        a.scheme = {"euler": N.KC_EULER, "rk2": N.KC_RK2, "rk4": N.KC_RK4}[self.scheme]
        a.dims = self.dims
        a.slot_a, a.slot_b, a.slot_t = slots[ia], slots[ib], slots[ib]
        a.alpha0 = alpha0
        cc = {"euler": (0.0,), "rk2": (0.0, 0.5), "rk4": (0.0, 0.5, 0.5, 1.0)}[self.scheme]
        if self.scheme != "euler":
            for j, c in enumerate(cc):
                a.alpha_k[j] = float(c) * self.dt / dtn
        a.dt = self.dt
        a.time_dir = 1.0
        a.w_code = 0 if self.w_interp == "nearest" else 1
        if self.kh is not None:
            a.kick = 1
            a.kh_x, a.kh_y = self.kh
            a.seed, a.real_id, a.step_i, a.pid_offset = self.seed, 0, k, 0
        a.global_step = -1 if self.release_step is None else k
        a.uv_vertical = 0 if self.uv_vertical == "layer" else 1
        a.precision = precision
        return a


def c1(P: int = 100_000, spacing: float = 0.5625) -> Workload:
    """2-D FESOM2-style: jittered (+-20 %) lon/lat lattice with a 30 % land mask
    (~127 k wet nodes, ~250 k triangles), u/v float32 on nodes (solid-body
    rotation + double gyre, 0.5 m/s), 2 snapshots 24 h apart cycled, 100 k
    particles uniform over the wet area, RK2, dt 1 h, 240 steps, no diffusion.
    Every workload's seeds are sorted by 1-degree cell (sort_seeds)."""
    m = S.lattice_mesh(spacing, 80.0, jitter=0.2, land_frac=0.3)
    snaps = S.gyre_snapshots(m, 2, amp=0.5)
    lon, lat, z = S.sort_seeds(*S.release_uniform(m, P, seed=3))
    return Workload("c1_fesom2_2d_rk2", m, snaps, lon, lat, z, "rk2", 3600.0, 86400.0, 240,
                    description={"mesh": "jittered 0.5625 deg lattice, 30% land", "nodes": int(m.n_nodes),
                                 "elements": int(m.n_elements), "particles": P, "seeds": "sorted by 1-degree cell", "scheme": "rk2",
                                 "dt_s": 3600, "steps_run": 240, "fields": "f32 node u,v, 2 snapshots 24 h"})


def c2(P: int = 1_000_000, spacing: float = 0.5625, n_levels: int = 47) -> Workload:
    """3-D depth-linear on the C1 mesh: 47 z-level interfaces (5 m .. 6000 m
    stretched), smooth bathymetry 50-6000 m, u/v/w float32 on nodes x levels
    (uv_vertical level; w from the continuity of the gyre field), 4 snapshots
    3.5 days apart cycled, 1 M particles uniform in the wet volume, RK4, dt
    30 min, 480 steps, W nearest."""
    zl = S.stretched_levels(n_levels, 5.0, 6000.0)
    m = S.lattice_mesh(spacing, 80.0, jitter=0.2, land_frac=0.3,
                       depth=lambda lo, la: S.smooth_bathymetry(lo, la, 50.0, 6000.0), sigma=zl)
    snaps = S.gyre_snapshots(m, 4, amp=0.5, z_levels=zl, decay=1000.0, w_scale=1e-3, placement="level")
    lon, lat, z = S.sort_seeds(*S.release_uniform(m, P, seed=3, depth_uniform=True))
    return Workload("c2_fesom2_3d_dl_rk4", m, snaps, lon, lat, z, "rk4", 1800.0, 3.5 * 86400.0, 480,
                    dims=3, w_interp="nearest", uv_vertical="level",
                    description={"mesh": "jittered 0.5625 deg lattice, 30% land", "nodes": int(m.n_nodes),
                                 "elements": int(m.n_elements), "levels": n_levels, "particles": P, "seeds": "sorted by 1-degree cell",
                                 "scheme": "rk4", "dt_s": 1800, "steps_run": 480,
                                 "fields": "f32 node u,v,w (47,N) depth-linear (level), 4 snapshots 3.5 d",
                                 "w_interp": "nearest"})


def c3(P: int = 6_000_000, nside: int = 512, n_levels: int = 69, n_snap: int = 2) -> Workload:
    """HEALPix nside 512 dual mesh (3.1 M pixels, ~70 % wet from smooth noise),
    69 z-level interfaces (5 m .. 6000 m stretched), u/v (68, N) and w (69, N)
    float32 (~1.8 GB per snapshot) from 256 Gaussian vortices at 0.3 m/s rms,
    snapshots 24 h apart cycled, 6 M particles uniform over the wet area and
    in the column, RK2 dt 6 h, W barycentric, split uniform random walk
    Kh = 10 m^2/s keyed to particle id and step (seed 0)."""
    from . import healpix as H
    npix = 12 * nside * nside
    pix = np.arange(npix)
    plon, plat = H.pix2lonlat(nside, pix)
    noise = S._sphere_noise(plon, plat, seed=2)
    wet = noise >= np.quantile(noise, 0.3)
    zl = S.stretched_levels(n_levels, 5.0, 6000.0)
    depth = S.smooth_bathymetry(plon, plat, 50.0, 6000.0)
    m = H.dual_mesh(nside, wet, depth, sigma=zl)
    snaps = S.vortex_snapshots(m, n_snap, z_levels=zl)
    lon, lat, z = S.sort_seeds(*S.release_uniform(m, P, seed=3, depth_uniform=True))
    return Workload("c3_healpix512_3d_rk2_kick", m, snaps, lon, lat, z, "rk2", 21600.0, 86400.0, 1460,
                    dims=3, w_interp="barycentric", kh=(10.0, 10.0), seed=0,
                    description={"mesh": f"HEALPix nside {nside} dual mesh, ~70% wet", "nodes": int(m.n_nodes),
                                 "elements": int(m.n_elements), "levels": n_levels, "particles": P, "seeds": "sorted by 1-degree cell",
                                 "scheme": "rk2", "dt_s": 21600, "steps_run": 1460,
                                 "fields": "f32 node u,v (68,N), w (69,N), 256 Gaussian vortices 0.3 m/s rms",
                                 "diffusion": "split uniform Kh=10 m^2/s", "w_interp": "barycentric"})


def c4(n_cohorts: int = 64, members: int = 8, spacing: float = 0.2, n_levels: int = 47, seed: int = 4,
       size_lo: int = 1000, size_hi: int = 500_000, release_days: float = 30.0) -> Workload:
    """Batched cohorts: a ~1 M-node jittered lattice mesh (triangles plus 25 %
    convex quads, 30 % land), 47 z-level interfaces, smooth bathymetry,
    float32 u/v (46, N) and w (47, N) on nodes (layer placement, 2 daily
    snapshots cycled); 64 release cohorts of log-uniform size 1 k - 500 k
    particles (uniform over the wet volume, seeds sorted within each cohort),
    released at uniform times over 30 days; 8 diffusion ensemble members each
    (realization ids 0..7, Kh = 50 m^2/s); RK4, dt 1 h, W barycentric, 60-day
    horizon.  Slots are member-major, then cohort: every (member, cohort) block
    is contiguous.  The timed window starts at day 30, when every cohort is
    released."""
    zl = S.stretched_levels(n_levels, 5.0, 6000.0)
    m = S.lattice_mesh(spacing, 80.0, jitter=0.2, land_frac=0.3, quad_frac=0.25,
                       depth=lambda lo, la: S.smooth_bathymetry(lo, la, 50.0, 6000.0), sigma=zl)
    snaps = S.gyre_snapshots(m, 2, amp=0.5, z_levels=zl, decay=1000.0, w_scale=1e-3)
    rng = np.random.default_rng(seed)
    sizes = np.exp(rng.uniform(np.log(size_lo), np.log(size_hi), n_cohorts)).astype(np.int64)
    dt = 3600.0
    rel = np.floor(rng.uniform(0.0, release_days * 86400.0, n_cohorts) / dt).astype(np.int32)
    base = int(sizes.sum())
    blon, blat, bz = S.release_uniform(m, base, seed=seed + 1, depth_uniform=True)
    off = np.concatenate([[0], np.cumsum(sizes)])
    parts = [S.sort_seeds(blon[off[c]:off[c + 1]], blat[off[c]:off[c + 1]], bz[off[c]:off[c + 1]])
             for c in range(n_cohorts)]
    clon = np.concatenate([p[0] for p in parts])
    clat = np.concatenate([p[1] for p in parts])
    cz = np.concatenate([p[2] for p in parts])
    cpid = np.concatenate([np.arange(s, dtype=np.int64) for s in sizes])
    crel = np.repeat(rel, sizes)
    lon = np.tile(clon, members)
    lat = np.tile(clat, members)
    z = np.tile(cz, members)
    pid = np.tile(cpid, members)
    rs = np.tile(crel, members)
    rid = np.repeat(np.arange(members, dtype=np.int32), base)
    cohorts = [(r * base + int(off[c]), int(sizes[c]), r, c) for r in range(members) for c in range(n_cohorts)]
    P = lon.size
    return Workload("c4_cohorts_3d_rk4_kick", m, snaps, lon, lat, z, "rk4", dt, 86400.0, 1440,
                    dims=3, w_interp="barycentric", kh=(50.0, 50.0), seed=0,
                    pid=pid, real_id=rid, release_step=rs, cohorts=cohorts, t0_step=int(release_days * 24),
                    description={"mesh": f"jittered {spacing} deg lattice, 25% quads, 30% land",
                                 "nodes": int(m.n_nodes), "elements": int(m.n_elements), "levels": n_levels,
                                 "particles": P, "cohorts": n_cohorts, "members": members,
                                 "cohort_sizes": [int(v) for v in sizes],
                                 "seeds": "sorted by 1-degree cell within each cohort",
                                 "release": f"uniform over {release_days:g} days", "scheme": "rk4", "dt_s": 3600,
                                 "steps_run": 1440, "fields": "f32 node u,v (46,N), w (47,N), 2 daily snapshots",
                                 "diffusion": "split uniform Kh=50 m^2/s, per-member realization ids",
                                 "w_interp": "barycentric", "timed_from_step": int(release_days * 24)})


def c3_small(P: int = 200_000) -> Workload:
    """C3's kernel on a reduced HEALPix grid (nside 128) and particle count:
    the profiling case (a few hundred MB on the device)."""
    w = c3(P=P, nside=128, n_levels=69)
    w.name = "c3small_healpix128_3d_rk2_kick"
    return w


def c4_small() -> Workload:
    """C4's structure at a test size: 8 cohorts of 500 - 5 000 particles on a
    2-degree mesh, 3 members, releases over 2 days."""
    w = c4(n_cohorts=8, members=3, spacing=2.0, size_lo=500, size_hi=5000, release_days=2.0)
    w.name = "c4small_cohorts_3d_rk4_kick"
    return w


def c5(P: int = 2_000_000, ny: int = 1021, nx: int = 1442, n_levels: int = 75, n_snap: int = 2) -> Workload:
    """NEMO C-grid 3-D on a global tripolar ORCA-like raster of 1442 x 1021
    (kelp_b200.synthetic.tripolar_grid: 1440 columns 0.25 deg apart plus the
    two E-W halo columns, a T-pivot north fold with its halo row, the two grid
    poles over land at 65 N, 73 E / 107 W), ~30 % land from smooth noise plus
    the poles, the Antarctic rows and the fold pivots; 75 z-levels (1 m ..
    5800 m stretched) with partial bottom cells over a smooth 200-5500 m
    bathymetry; face-raster u/v (75, ny*nx) of a non-divergent flow from a
    streamfunction sampled at the F-points (continuous through the seam and
    the fold; 0.5 m/s rms at the surface, decaying with depth) and w (76,
    ny*nx) float32, in canonical form (halo and fold copies from their
    canonical points, vectors with the fold sign); model face widths and cell
    areas; 2 five-day records cycled; 2 M particles uniform over the wet
    cells and in their columns; the exact C-grid RK4 in the fractional level
    coordinate, dt 1 h, 720 steps (no diffusion, no beaching: the reference's
    3-D C-grid step takes neither)."""
    from .fields import VelocityField
    from .nemo import build_cgrid_mesh, to_canonical
    rng = np.random.default_rng(5)
    lay, glamf, gphif, glamt, gphit = S.tripolar_grid(ny, nx, fold="T")
    tl, tp = glamt.reshape(-1), gphit.reshape(-1)
    noise = S._sphere_noise(tl, tp, seed=6).reshape(ny, nx)

    def sep(lo, la):
        r = np.radians
        c = np.sin(r(gphit)) * np.sin(r(la)) + np.cos(r(gphit)) * np.cos(r(la)) * np.cos(r(glamt - lo))
        return np.degrees(np.arccos(np.clip(c, -1.0, 1.0)))

    wet = (noise >= np.quantile(noise, 0.3)) & (gphit > -76.0) & (sep(73.0, 65.0) > 6.0) & (sep(-107.0, 65.0) > 6.0)
    wet = to_canonical(wet & ~lay.pivot_cells(), lay, "T") > 0.5
    depth = S.smooth_bathymetry(tl, tp, 200.0, 5500.0).reshape(ny, nx)
    zw = S.stretched_levels(n_levels + 1, 1.0, 5800.0)
    lay_d = np.diff(zw)
    nlev = np.where(wet, np.clip(np.searchsorted(zw, depth, side="left"), 1, n_levels), 0).astype(np.int32)
    bot = lay_d[np.maximum(nlev - 1, 0)]
    e3b = np.where(nlev > 0, np.clip(depth - zw[np.maximum(nlev - 1, 0)], 0.1 * bot, bot), 0.0)
    nlev = to_canonical(nlev, lay, "T").astype(np.int32)
    e3b = to_canonical(e3b, lay, "T")
    u2, v2, e2u, e1v = S.cgrid_stream_flow(glamf, gphif, amp=1.0)
    scale = 0.5 / np.sqrt(np.mean(np.concatenate([u2[wet] ** 2, v2[wet] ** 2])))
    u2 = to_canonical(u2 * scale, lay, "U", vector=True).astype(np.float32)
    v2 = to_canonical(v2 * scale, lay, "V", vector=True).astype(np.float32)
    e2u = to_canonical(e2u, lay, "U")
    e1v = to_canonical(e1v, lay, "V")
    area = to_canonical(np.maximum(e2u * e1v, 1.0), lay, "T")
    mesh = build_cgrid_mesh(glamf, gphif, wet, layout=lay, e2u=e2u, e1v=e1v, nlev2d=nlev, zw=zw, area=area,
                            e3b=e3b, name="c5_tripolar_cgrid")
    K = n_levels
    zm = 0.5 * (zw[:-1] + zw[1:])
    dec = np.exp(-zm / 800.0).astype(np.float32)[:, None]
    lev = np.arange(K)[:, None]
    wetk = lev < nlev.reshape(1, -1)
    snaps = []
    for k in range(n_snap):
        ph = np.float32(1.0 + 0.3 * k)
        u = np.where(wetk, u2.reshape(1, -1) * dec * ph, np.float32(0.0))
        v = np.where(wetk, v2.reshape(1, -1) * dec * (np.float32(2.3) - ph), np.float32(0.0))
        wt = to_canonical(1e-5 * np.sin(np.radians(4.0 * glamt + 60.0 * k)) * np.cos(np.radians(gphit)), lay, "T")
        w = np.where(np.arange(K + 1)[:, None] < nlev.reshape(1, -1), wt.astype(np.float32).reshape(1, -1),
                     np.float32(0.0))
        snaps.append(VelocityField(u=u, v=v, w=w, eta=np.zeros(ny * nx), uv_layout="nemo_cgrid"))
    # particles: uniform over the wet cells (a random point of the cell's
    # corner quad, on the sphere), uniform in the column
    n_wet = int((mesh._nemo_cgrid_nlev > 0).sum())
    pick = rng.integers(0, n_wet, P)
    cn = mesh._nemo_cgrid_corners[pick]
    la, lo = np.radians(mesh.nodes_lat[cn]), np.radians(mesh.nodes_lon[cn])
    xyz = np.stack((np.cos(la) * np.cos(lo), np.cos(la) * np.sin(lo), np.sin(la)), axis=-1)
    a, b = rng.random(P)[:, None], rng.random(P)[:, None]
    pt = ((1 - a) * (1 - b) * xyz[:, 0] + a * (1 - b) * xyz[:, 1] + a * b * xyz[:, 2] + (1 - a) * b * xyz[:, 3])
    lon = np.degrees(np.arctan2(pt[:, 1], pt[:, 0]))
    lat = np.degrees(np.arcsin(pt[:, 2] / np.linalg.norm(pt, axis=1)))
    j, i = mesh._nemo_cgrid_elem_ji[pick].T
    floor_ = zw[np.maximum(nlev[j, i] - 1, 0)] + e3b[j, i]
    z = rng.random(P) * 0.95 * floor_
    lon, lat, z = S.sort_seeds(lon, lat, z)
    return Workload("c5_nemo_cgrid_3d_rk4", mesh, snaps, lon, lat, z, "rk4", 3600.0, 5 * 86400.0, 720, dims=3,
                    description={"mesh": f"tripolar ORCA-like C-grid {nx}x{ny} (T-pivot north fold, E-W halo), "
                                         "~30% land, partial bottom cells",
                                 "nodes": int(mesh.n_nodes), "elements": int(mesh.n_elements), "levels": n_levels,
                                 "particles": P, "seeds": "sorted by 1-degree cell", "scheme": "rk4", "dt_s": 3600,
                                 "steps_run": 720, "uv_interp": "nemo_cgrid",
                                 "fields": "f32 face rasters u,v (75, ny*nx), w (76, ny*nx), 2 five-day records"})


def c5_small(P: int = 200_000) -> Workload:
    """C5's construction on a 362 x 256 tripolar raster (1 degree): the
    profiling and test case."""
    w = c5(P=P, ny=256, nx=362)
    w.name = "c5small_nemo_cgrid_3d_rk4"
    return w


WORKLOADS: dict = {"c1": c1, "c2": c2, "c3": c3, "c3small": c3_small, "c4": c4, "c4small": c4_small, "c5": c5,
                   "c5small": c5_small}
