"""Step functions with KELP's integrator signature, running on the B200.

``euler_step`` / ``rk2_step`` / ``rk4_step`` take and return the same objects
as KELP's (``src/kelp/numerics/integrators.py:5150``, ``:5611``, ``:6013``):
``step(state, vel, mesh, dt, time_dir, layer=0, *, w_interp, uv_interp,
vel_next, dt_to_next, diffusion, ...) -> ParticleState``.  ``INTEGRATORS`` /
``get_integrator`` mirror the registry (``integrators.py:6635-6660``), so the
module is a drop-in at the plugin point.

Every supported combination runs as one CUDA kernel launch per step; there is
no CPU path.  Two backend keywords select the numerical form:
``cuda_precision="plain"`` (default: the reference's float64 arithmetic) or
``"mixed"`` (float32 interpolation, float64 positions and element decisions),
and ``cuda_snapshots="f16"`` stores the snapshots as float16 with per-row
scales (mixed form only).  Combinations this build does not implement raise
``NotImplementedError`` before any device work, naming what is missing.
Argument errors raise ``ValueError`` in Python, as in the reference.
"""
from __future__ import annotations

from typing import Optional

import numpy as np

from . import _native as N
from .device import default_context
from .particles import ParticleState

_RK2_C = (0.0, 0.5)
_RK4_C = (0.0, 0.5, 0.5, 1.0)
_SCHEMES = {"euler": (N.KC_EULER, (0.0,)), "rk2": (N.KC_RK2, _RK2_C), "rk4": (N.KC_RK4, _RK4_C)}


def _is_3d(vel) -> bool:
    return getattr(vel, "w", None) is not None if not hasattr(vel, "vel_a") else (
        vel.vel_a.w is not None and vel.vel_b.w is not None)


def _zero_dead_velocity(state: ParticleState) -> ParticleState:
    """integrators.py:272-281: nothing alive -> zero velocity diagnostics."""
    if state.u is None:
        return state
    return state.replace(u=np.zeros_like(state.u), v=np.zeros_like(state.v),
                         w=None if state.w is None else np.zeros_like(state.w))


def _validate_time_aware(vel_next, dt_to_next, dt):
    if (vel_next is None) != (dt_to_next is None):
        raise ValueError("vel_next and dt_to_next must both be set or both be None")
    if dt_to_next is not None and not float(dt_to_next) > 0:
        raise ValueError(f"dt_to_next must be > 0, got {dt_to_next!r}")


def _kick_args(diffusion) -> Optional[tuple]:
    """(kh_x, kh_y, seed, real_id, step_i, pid_offset) of a split uniform kick,
    or None when no kick applies (absent, or Kh = 0: ``integrators.py:719-720``)."""
    if diffusion is None:
        return None
    if diffusion.scheme != "uniform":
        raise NotImplementedError(f"diffusion.scheme={diffusion.scheme!r} (variable Kh) is not built "
                                  "on the CUDA backend; only the uniform split kick is")
    if diffusion.composition not in ("split",):
        raise NotImplementedError(f"diffusion.composition={diffusion.composition!r} is not built on the "
                                  "CUDA backend")
    if float(diffusion.kh_x) == 0.0 and float(diffusion.kh_y) == 0.0:
        return None
    if float(diffusion.kh_x) < 0 or float(diffusion.kh_y) < 0:
        raise ValueError("Kh must be >= 0")
    return (float(diffusion.kh_x), float(diffusion.kh_y), int(diffusion.seed), int(diffusion.real_id),
            int(diffusion.step_i), int(getattr(diffusion, "pid_offset", 0)))


def _fields(vel, vel_next):
    """(vel_a, vel_b, target, alpha0) threading of the fused runners
    (integrators.py:3367-3370, :4729-4745)."""
    vel_a = getattr(vel, "vel_a", vel)
    vel_b = getattr(vel, "vel_b", vel_next if vel_next is not None else vel_a)
    alpha0 = float(getattr(vel, "alpha", 0.0))
    target = vel_next if vel_next is not None else vel_a
    return vel_a, vel_b, target, alpha0


def _sigma_mesh(mesh) -> bool:
    """A sigma mesh stepped by the s = z / H_p kernels (not a NEMO C-grid)."""
    return getattr(mesh, "vertical_coord", "zlevel") == "sigma" and not getattr(mesh, "_nemo_cgrid", False)


def _materialized(vel):
    """A LazyLerpField as the plain field its own blend makes of it (every
    array the payload carries, blended by the payload itself), for the paths
    where the reference steps the materialised field."""
    from .fields import VelocityField
    return VelocityField(u=np.asarray(vel.u), v=np.asarray(vel.v), eta=np.asarray(vel.eta), w=vel.w,
                         uv_layout=vel.uv_layout, uv_vertical=getattr(vel, "uv_vertical", "layer"),
                         az=getattr(vel, "az", None), scalars=getattr(vel, "scalars", None))


def _check_node_fields(mesh, fields, is3d, placement="layer"):
    n = mesh.nodes_lon.shape[0]
    for f in fields:
        if getattr(f, "uv_layout", "element") != "node":
            raise NotImplementedError("element-layout u/v (leastsq / edge_leastsq) is not built on the "
                                      "CUDA backend; node-layout barycentric is")
        u = np.asarray(f.u)
        if u.shape[-1] != n or np.asarray(f.v).shape != u.shape:
            raise ValueError(f"u/v of shape {u.shape} do not match the mesh's {n} nodes")
        if is3d:
            zl = np.abs(np.asarray(mesh.sigma))
            w = np.asarray(f.w)
            rows = {"layer": zl.shape[0] - 1, "level": zl.shape[0], "layer_linear": zl.shape[0] - 1}[placement]
            if w.shape != (zl.shape[0], n) or u.shape != (rows, n):
                raise ValueError(f"3-D {placement!r} fields need u/v ({rows}, {n}) and w "
                                 f"({zl.shape[0]}, {n}); got {u.shape} and {w.shape}")
            if getattr(f, "uv_vertical", "layer") != placement:
                raise ValueError("every field of one step needs the same uv_vertical placement "
                                 "(integrators.py:4534-4553)")


def _check_element_fields(mesh, fields, is3d=False):
    """Element-layout u/v for the least-squares stages: one value per element
    (io.py:180 VelocityField, uv_layout 'element'), per layer in 3-D with W on
    the nodes' interfaces."""
    E = np.asarray(mesh.elem_nodes).shape[0]
    n = np.asarray(mesh.nodes_lon).shape[0]
    K = np.asarray(mesh.sigma).shape[0]
    for f in fields:
        if getattr(f, "uv_layout", "element") != "element":
            raise ValueError("uv_interp 'leastsq' reads element-centre velocities (uv_layout='element'), "
                             f"got uv_layout={getattr(f, 'uv_layout', None)!r}")
        u = np.asarray(f.u)
        if not is3d:
            if u.shape != (E,) or np.asarray(f.v).shape != u.shape:
                raise ValueError(f"2-D element-layout u/v need shape ({E},), got {u.shape}")
            continue
        w = np.asarray(f.w)
        if u.shape != (K - 1, E) or np.asarray(f.v).shape != u.shape or w.shape != (K, n):
            raise ValueError(f"3-D element-layout fields need u/v ({K - 1}, {E}) and w ({K}, {n}); got {u.shape} "
                             f"and {w.shape}")


def _az_args(diffusion, vel, is3d, mesh):
    """(use_field, az_const) of the vertical Az kick, or None when it does
    not apply (integrators.py:842-907): the payload's Az field when it carries
    one, else the constant; a zero source skips the kick."""
    if diffusion is None or not getattr(diffusion, "az_enabled", False):
        return None
    az_field = getattr(vel, "az", None)
    az_const = max(float(getattr(diffusion, "az_const", 0.0)), 0.0)
    if az_field is None and getattr(diffusion, "az_requires_field", False):
        raise ValueError("diffusion.var_az is configured but the velocity payload carries no az field")
    if az_field is None and az_const == 0.0:
        return None
    if not is3d:
        raise ValueError("diffusion.az_enabled requires a 3-D run (Fdrift3D)")
    if getattr(mesh, "vertical_coord", "zlevel") == "sigma" and az_field is not None:
        # integrators.py:917-922: sigma meshes take the constant source only
        raise ValueError("diffusion.var_az is not supported on sigma meshes (v1) — use the constant az_const "
                         "source instead")
    return (az_field is not None, az_const)


def _check_recon(recon, dt, time_dir, c_coeffs):
    """The PCHIP bundle (snapshots, times, sim_time, direction) validated as
    reconstruct_pchip and the fused PCHIP runners do
    (temporal_reconstruct.py:218-245, integrators.py:3444-3505); returns it
    with float times."""
    try:
        snaps4, times4, q_time, direction = recon
    except (TypeError, ValueError):
        raise ValueError("recon must be (snapshots, times, sim_time, direction)") from None
    if len(snaps4) != 4 or len(times4) != 4:
        raise ValueError("reconstruct_pchip needs exactly 4 snapshots/times")
    t = [float(x) for x in times4]
    if not all(np.isfinite(x) for x in t):
        raise ValueError(f"reconstruct_pchip: non-finite times {times4}")
    if not (t[0] < t[1] < t[2] < t[3]):
        raise ValueError(f"reconstruct_pchip: times must be strictly increasing, got {times4}")
    d = float(direction)
    if d != float(time_dir):
        raise ValueError(f"recon direction {direction} disagrees with time_dir {time_dir}")
    q = float(q_time)
    tol = 1e-9 * (t[2] - t[1])
    for c in c_coeffs:
        tq = q + d * c * float(dt)
        if not (t[1] - tol <= tq <= t[2] + tol):
            raise ValueError(f"reconstruct_pchip: t_query={tq} outside the central interval [{t[1]}, {t[2]}]")
    return list(snaps4), t, q, d


def _check_call(dt, time_dir, kw, vel=None):
    if float(dt) <= 0:
        raise ValueError(f"dt must be > 0, got {dt!r}")
    if float(time_dir) not in (1.0, -1.0):
        raise ValueError(f"time_dir must be +1 or -1, got {time_dir!r}")
    diffusion = kw.get("diffusion", None)
    if (diffusion is not None and getattr(diffusion, "az_enabled", False)
            and getattr(diffusion, "scheme", "uniform") in ("em", "m1")):
        # integrators.py:824-839: checked before anything else
        raise ValueError("diffusion.az_enabled composes with scheme='uniform' only")
    if kw.get("uv_interp", "leastsq") == "nemo_cgrid" and vel is not None and _is_3d(vel):
        # nemo_cgrid.py:457-461: the 3-D C-grid step takes neither
        if diffusion is not None or kw.get("recon") is not None:
            raise NotImplementedError("the 3-D C-grid step supports neither diffusion nor temporal "
                                      "(PCHIP) reconstruction")
    return _kick_args(diffusion)


def _prepare_cgrid(vel, mesh, dt, time_dir, scheme, kw, ctx, kick):
    """prepare_step for uv_interp "nemo_cgrid" on a build_nemo_cgrid_mesh mesh:
    face-raster snapshots; 2-D steps read the surface faces
    (nemo_cgrid.py:355-388), 3-D steps are nemo_cgrid3d_step (:416-512)."""
    code, c_coeffs = _SCHEMES[scheme]
    if not getattr(mesh, "_nemo_cgrid", False):
        raise ValueError("uv_interp 'nemo_cgrid' needs a C-grid mesh (NEMO reader with mesh.nemo_grid: cgrid)")
    if kw.get("recon") is not None:
        raise NotImplementedError("PCHIP temporal reconstruction is not built on the CUDA backend")
    if not (mesh.metadata or {}).get("exact_nearest", False):
        raise NotImplementedError("the CUDA backend anchors with the exact nearest-node search only "
                                  "(mesh.exact_nearest: true, the configuration default)")
    form = kw.get("cuda_precision", "plain")
    if form not in ("plain", "mixed"):
        raise ValueError(f"cuda_precision must be 'plain' or 'mixed', got {form!r}")
    if kw.get("cuda_snapshots") not in (None, "f32", "f16"):
        raise ValueError(f"cuda_snapshots must be None, 'f32' or 'f16', got {kw.get('cuda_snapshots')!r}")
    if kw.get("cuda_snapshots") == "f16" and form != "mixed":
        raise ValueError("float16 rasters are read by the mixed form only (cuda_precision='mixed')")
    if form == "mixed" and not _is_3d(vel):
        raise NotImplementedError("the mixed form on C-grid meshes is the 3-D step")
    vel_next = kw.get("vel_next", None)
    dt_to_next = kw.get("dt_to_next", None)
    _validate_time_aware(vel_next, dt_to_next, dt)
    vel_a, vel_b, target, alpha0 = _fields(vel, vel_next)
    for f in (vel_a, vel_b, target):
        if getattr(f, "uv_layout", "element") != "nemo_cgrid":
            raise ValueError(f"uv_interp 'nemo_cgrid' needs uv_layout='nemo_cgrid', got {f.uv_layout!r}")
    is3d = _is_3d(vel)
    ctx = ctx or default_context()
    ctx.ensure_mesh(mesh)
    sa, sb, st = ctx.slots_for([vel_a, vel_b, target], snapshot_storage(kw))
    a = N.StepArgs()
    a.scheme = code
    a.dims = 3 if is3d else 2
    a.slot_a, a.slot_b, a.slot_t = sa, sb, st
    a.alpha0 = alpha0
    if vel_next is not None:
        # _make_stage_vels at the stage fractions (the C-grid 3-D step's
        # Butcher nodes are the same (0, .5, .5, 1) / (0, .5) / (0,))
        for k, c in enumerate(c_coeffs):
            a.alpha_k[k] = float(c) * float(dt) / float(dt_to_next)
    a.dt = float(dt)
    a.time_dir = float(time_dir)
    if kick is not None:
        a.kick = 1
        a.kh_x, a.kh_y, a.seed, a.real_id, a.step_i, a.pid_offset = kick
    a.global_step = -1
    a.precision = N.KC_MIXED if form == "mixed" else N.KC_PLAIN
    a.Dmin, a.z0b_min = 0.5, 0.1
    return a, is3d


def snapshot_storage(kw):
    """The snapshot slots' element type of a step's keyword set: float32 or
    float16 when named (cuda_snapshots), float32 for the mixed form, else
    None (the payload's own: float32 only when every array is)."""
    store = {None: None, "f32": np.float32, "f16": np.float16}.get(kw.get("cuda_snapshots", None))
    if kw.get("cuda_precision", "plain") == "mixed" and store is None:
        store = np.float32
    return store


def prepare_step(vel, mesh, dt, time_dir, scheme, kw, ctx=None, kick=None, elem=None):
    """Validate one step's payload and make it resident on ``ctx`` (mesh,
    depth-point table, snapshot slots); returns ``(StepArgs, is3d)``.  ``scheme``
    is ``"euler"``, ``"rk2"`` or ``"rk4"``; ``ctx`` defaults to the default
    device context, opened only after validation.  Raises ``NotImplementedError``
    for combinations the CUDA backend does not build."""
    code, c_coeffs = _SCHEMES[scheme]
    uv_interp = kw.get("uv_interp", "leastsq")
    if uv_interp == "nemo_cgrid":
        if elem is not None and _is_3d(vel):
            elem = None   # the 3-D C-grid step neither reads nor updates carried elements
        if elem is not None:
            (ctx or default_context()).ensure_elem_neighbors(mesh)
        return _prepare_cgrid(vel, mesh, dt, time_dir, scheme, kw, ctx, kick)
    lsq = uv_interp in ("leastsq", "edge_leastsq")
    if uv_interp not in ("barycentric", "leastsq", "edge_leastsq"):
        raise NotImplementedError(f"uv_interp={uv_interp!r} is not built on the CUDA backend; use 'barycentric' "
                                  "(node-layout velocities), 'leastsq' or 'edge_leastsq' (element layout)")
    edge_bc = None
    if uv_interp == "edge_leastsq":   # interpolate.py:3374-3395: the lateral boundary rule of the ghost points
        edge_bc = kw.get("edge_leastsq_bc", "freeslip")
        if edge_bc not in ("freeslip", "noslip"):
            raise ValueError(f"edge_leastsq_bc must be 'freeslip' or 'noslip', got {edge_bc!r}")
    if lsq:
        if _is_3d(vel) and (getattr(vel, "uv_vertical", "layer") != "layer" or _sigma_mesh(mesh)):
            raise NotImplementedError(f"3-D uv_interp {uv_interp!r} is built for layer fields on z-level meshes on "
                                      "the CUDA backend (depth-linear element fields and sigma meshes are not)")
        if elem is not None:
            raise NotImplementedError(f"uv_interp {uv_interp!r} with elem_search 'walk' is not built on the "
                                      "CUDA backend")
        if kw.get("cuda_precision", "plain") != "plain":
            raise NotImplementedError("uv_interp 'leastsq' runs in the plain form (cuda_precision='plain')")
    # PCHIP: the RK stages are reconstructed from the tracking layer's
    # 4-record stencil; Euler evaluates the payload itself and ignores it
    recon = kw.get("recon") if scheme != "euler" else None
    if recon is not None:
        recon = _check_recon(recon, dt, time_dir, c_coeffs)
    if not (mesh.metadata or {}).get("exact_nearest", False):
        raise NotImplementedError("the CUDA backend anchors with the exact nearest-node search only "
                                  "(mesh.exact_nearest: true, the configuration default)")
    vel_next = kw.get("vel_next", None)
    dt_to_next = kw.get("dt_to_next", None)
    _validate_time_aware(vel_next, dt_to_next, dt)
    if scheme != "euler" and dt_to_next is not None and float(dt) > float(dt_to_next) + 1e-9:
        # integrators.py:1046-1052: the RK stages would read past the bracket
        raise ValueError(f"step endpoint past next snapshot: dt={float(dt):.6f}s > "
                         f"dt_to_next={float(dt_to_next):.6f}s")
    is3d = _is_3d(vel)
    w_code = 0
    placement = "layer"
    if is3d:
        coord = getattr(mesh, "vertical_coord", "zlevel")
        if coord not in ("zlevel", "sigma"):
            raise ValueError(f"unknown mesh.vertical_coord {coord!r}")
        placement = getattr(vel, "uv_vertical", "layer")
        if placement not in ("layer", "level", "layer_linear"):
            raise ValueError(f"unknown uv_vertical {placement!r}")
        if coord == "sigma":
            if placement == "level":
                raise ValueError("uv_vertical 'level' on a sigma mesh: depth-linear u/v there is 'layer_linear' "
                                 "only (vertical_uv.py:196-211)")
            if kw.get("cuda_precision", "plain") != "plain":
                raise NotImplementedError("sigma meshes step in the plain form (cuda_precision='plain')")
            own = np.shape(vel.eta)
            for key in ("sigma_eta_start", "sigma_eta_end"):
                given = kw.get(key)
                if given is not None and np.shape(given) != own:   # integrators.py:1413-1424 _sigma_given
                    raise ValueError(f"sigma step: supplied surface has shape {np.shape(given)}, "
                                     f"the velocity field's eta {own}")
            if float(kw.get("Dmin", 0.5)) <= 0.0:
                raise ValueError("Dmin must be > 0")
        w_interp = kw.get("w_interp", "leastsq")
        codes = {"nearest": 0, "barycentric": 1, "leastsq": 2, "idw": 3}
        if w_interp not in codes:
            raise ValueError(f"unknown w_interp {w_interp!r}; expected one of {tuple(codes)}")
        w_code = codes[w_interp]
        if w_code >= 2 and kw.get("cuda_precision", "plain") != "plain":
            raise NotImplementedError(f"w_interp={w_interp!r} runs in the plain form (cuda_precision='plain')")
        if code == N.KC_RK2 and hasattr(vel, "vel_a") and float(getattr(vel, "alpha", 1.0)) == 0.0:
            # integrators.py:5691-5692 routes an endpoint LazyLerpField to the
            # unfused RK2 (:5380-5608): its stage fields are the payload
            # materialised, 1.0 a + 0.0 b, and its stage arithmetic is the
            # fused RK2's, so the fused kernel steps the materialised field
            vel = _materialized(vel)
    vel_a, vel_b, target, alpha0 = _fields(vel, vel_next)
    if lsq:
        _check_element_fields(mesh, [vel_a, vel_b, target] + (list(recon[0]) if recon is not None else []), is3d)
    else:
        _check_node_fields(mesh, [vel_a, vel_b, target] + (list(recon[0]) if recon is not None else []), is3d,
                           placement)
    form = kw.get("cuda_precision", "plain")
    if recon is not None and form != "plain":
        raise NotImplementedError("PCHIP reconstruction runs in the plain form (cuda_precision='plain')")
    if form not in ("plain", "mixed"):
        raise ValueError(f"cuda_precision must be 'plain' or 'mixed', got {form!r}")
    storage = kw.get("cuda_snapshots", None)
    if storage not in (None, "f32", "f16"):
        raise ValueError(f"cuda_snapshots must be None, 'f32' or 'f16', got {storage!r}")
    if storage == "f16" and form != "mixed":
        raise ValueError("float16 snapshots are read by the mixed form only (cuda_precision='mixed')")
    store = {None: None, "f32": np.float32, "f16": np.float16}[storage]
    if form == "mixed" and store is None:
        store = np.float32

    ctx = ctx or default_context()
    ctx.ensure_mesh(mesh)
    if elem is not None:   # elem_search: walk -- the edge walk reads the neighbour table
        ctx.ensure_elem_neighbors(mesh)
    if is3d and placement != "layer":
        ctx.ensure_depth_points(mesh, placement)
    if lsq:
        ctx.ensure_elem_centers(mesh)
    if edge_bc is not None:
        ctx.ensure_elem_neighbors(mesh)
    a = N.StepArgs()
    a.uv_lsq = 0 if not lsq else (1 if edge_bc is None else (2 if edge_bc == "freeslip" else 3))
    if recon is None:
        sa, sb, st = ctx.slots_for([vel_a, vel_b, target], store)
        a.slot_a, a.slot_b, a.slot_t = sa, sb, st
        a.alpha0 = alpha0
        if vel_next is not None and code != N.KC_EULER:
            for k, c in enumerate(c_coeffs):
                a.alpha_k[k] = float(c) * float(dt) / float(dt_to_next)
    else:
        # the stencil in four slots; each stage "alpha" is its time
        # sim_time + time_dir * c * dt (temporal_reconstruct.py:298-325)
        snaps4, times4, q_time, direction = recon
        a.slot_a, a.slot_b, a.slot_t, a.slot_d = ctx.slots_for(list(snaps4), store)
        a.pchip = 1
        for k in range(4):
            a.pchip_t[k] = times4[k]
        for k, c in enumerate(c_coeffs):
            a.alpha_k[k] = q_time + direction * c * float(dt)
    a.scheme = code
    a.dims = 3 if is3d else 2
    a.dt = float(dt)
    a.time_dir = float(time_dir)
    a.w_code = w_code
    a.uv_vertical = 1 if placement != "layer" else 0
    if kick is not None:
        a.kick = 1
        a.kh_x, a.kh_y, a.seed, a.real_id, a.step_i, a.pid_offset = kick
    a.global_step = -1
    a.precision = N.KC_MIXED if form == "mixed" else N.KC_PLAIN
    # sigma meshes: the column floor, the bed clearance and the end-of-step
    # surface's blend (integrators.py:1400-1420 _sigma_end_eta)
    a.Dmin = float(kw.get("Dmin", 0.5))
    a.z0b_min = float(kw.get("z0b_min", 0.1))
    a.alpha_end = float(dt) / float(dt_to_next) if vel_next is not None else 0.0
    if recon is not None:   # the end-of-step surface: the reconstruction at c = 1 (integrators.py:1369-1391)
        a.alpha_end = recon[2] + recon[3] * 1.0 * float(dt)
    az = _az_args(kw.get("diffusion", None), vel, is3d, mesh)
    if az is not None and recon is not None:
        raise NotImplementedError("the Az kick with PCHIP reconstruction is not built on the CUDA backend")
    if az is not None:
        if az[0] and store is np.float16:
            raise NotImplementedError("the Az field with float16 snapshots is not built on the CUDA backend")
        a.az_kick, a.az_field, a.az_const = 1, int(az[0]), float(az[1])
        d = kw["diffusion"]
        if kick is None:   # the Az draws use the step's keys even without a horizontal kick
            a.seed, a.real_id, a.step_i = int(d.seed), int(d.real_id), int(d.step_i)
            a.pid_offset = int(getattr(d, "pid_offset", 0))
    return a, is3d


def _run(state, vel, mesh, dt, time_dir, scheme, kw, ctx=None) -> ParticleState:
    kick = _check_call(dt, time_dir, kw, vel)
    if not np.any(state.alive_mask):
        return _zero_dead_velocity(state)
    a, is3d = prepare_step(vel, mesh, dt, time_dir, scheme, kw, ctx, kick=kick, elem=state.elem)
    ctx = ctx or default_context()
    fr_in = state.failure_reason
    P = state.n_particles
    inp = {"lon": np.ascontiguousarray(state.lon, dtype=np.float64),
           "lat": np.ascontiguousarray(state.lat, dtype=np.float64),
           "z": np.ascontiguousarray(state.z, dtype=np.float64) if is3d else None,
           "status": np.ascontiguousarray(state.status, dtype=np.int32),
           "nearest_node": np.ascontiguousarray(state.nearest_node, dtype=np.int32),
           "failure_reason": None if fr_in is None else np.ascontiguousarray(fr_in, dtype=np.int8)}
    out = {"lon": np.empty(P), "lat": np.empty(P), "z": np.empty(P) if is3d else None,
           "status": np.empty(P, np.int32), "nearest_node": np.empty(P, np.int32),
           "failure_reason": None if fr_in is None else np.empty(P, np.int8),
           "u": np.empty(P), "v": np.empty(P), "w": np.empty(P) if is3d else None}
    # elem_search: walk (integrators.py:5415-5416): carried elements in and
    # out (the 3-D C-grid step leaves them untouched, nemo_cgrid.py:416-512)
    walk = state.elem is not None and not (kw.get("uv_interp") == "nemo_cgrid" and is3d)
    if walk:
        inp["elem"] = np.ascontiguousarray(state.elem, dtype=np.int32)
        out["elem"] = np.empty(P, np.int32)
    if is3d and _sigma_mesh(mesh):
        # the tracking layer's surfaces of this step (integrators.py:1381-1441),
        # or the payload's own; a steady step blends its stage surfaces
        steady = kw.get("recon") is None and (kw.get("vel_next") is None or not (kw.get("dt_to_next") or 0) > 0)
        ctx.sigma_surfaces(kw.get("sigma_eta_start"), kw.get("sigma_eta_end"), steady)
    # one call: chunked upload, step and download overlapped on the device
    ctx.step_host(a, inp, out)
    err = ctx.device_errors()
    if err:
        raise N.KcError(N.KC_ERR_DEVICE, N.describe_device_errors(err))
    new = state.replace(
        lon=out["lon"], lat=out["lat"], z=out["z"] if is3d else np.array(state.z, copy=True),
        status=out["status"], nearest_node=out["nearest_node"],
        u=out["u"], v=out["v"], w=out["w"],
        failure_reason=out["failure_reason"],
    )
    if walk:
        new = new.replace(elem=out["elem"])
    return new


def euler_step(state, vel, mesh, dt, time_dir, layer: int = 0, **kwargs) -> ParticleState:
    """Forward Euler (integrators.py:5150)."""
    return _run(state, vel, mesh, dt, time_dir, "euler", kwargs)


def rk2_step(state, vel, mesh, dt, time_dir, layer: int = 0, **kwargs) -> ParticleState:
    """RK2 midpoint (integrators.py:5611)."""
    return _run(state, vel, mesh, dt, time_dir, "rk2", kwargs)


def rk4_step(state, vel, mesh, dt, time_dir, layer: int = 0, **kwargs) -> ParticleState:
    """Classical RK4 (integrators.py:6013)."""
    return _run(state, vel, mesh, dt, time_dir, "rk4", kwargs)


def _rk45_unavailable(*a, **k):
    raise NotImplementedError("rk45 (adaptive, 2-D leastsq) is not built on the CUDA backend")


INTEGRATORS = {"euler": euler_step, "rk2": rk2_step, "rk4": rk4_step, "rk45": _rk45_unavailable}


def get_integrator(name: str):
    """Registry lookup (integrators.py:6635-6660)."""
    key = str(name).lower()
    if key not in INTEGRATORS:
        raise ValueError(f"Unknown integrator {name!r}. Choose from: {sorted(INTEGRATORS)}")
    return INTEGRATORS[key]
