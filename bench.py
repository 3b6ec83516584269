"""Benchmark of the B200 time-stepping path: particle-steps/s on one node.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--workload c3]
                    [--form mixed] [--forms plain,mixed,mixed_f16]
                    [--impl b200|reference]

One step = one pass of the step kernel over every particle of the workload
(inputs resident in HBM, L2 evicted between timed steps, CUDA events on the
library's stream, the periodic re-sort inside the timed region).  Every form
in --forms is timed the same way: "plain" (the reference's float64
arithmetic), "mixed" (float32 interpolation, float64 positions and element
decisions) and "mixed_f16" (the same on float16 snapshots with per-row
scales); the headline value is --form's.  On one GPU the line also reports
each form's great-circle separation from the plain form after 24 h (all
particles) and after the configuration's horizon (a subset), and the oracle
port's CPU throughput.  Under torchrun (N > 1) every rank runs its own shard
of the same per-GPU size (weak scaling: particles are independent, nothing is
exchanged); the time is the maximum over ranks.  Rank 0 prints one JSON line.

``--impl reference`` times the reference's own CPU implementation of the step
on this host's cores, all threads: KELP's Numba step functions from the
package installed under baseline/_ref (else, or for workloads it cannot be
driven on here, the oracle C port), on the same workload, metric, unit and
config, with full-size steps where they fit the time budget.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "particle-steps/s on 1 B200, mixed vs FP64 form at ≤1 m p99 error; HBM GB/s vs peak"
UNIT = "particle-steps/s"
# workload -> the reference's published figure for this exact metric: the fused
# 3-D RK2 step on HEALPix nside 512, 69 levels, 6 M particles, 128 EPYC 7763
# cores (manual/chapters/17-performance.tex:219-233)
PUBLISHED = {"c3_healpix512_3d_rk2_kick": 10.4e6}


def env_rank():
    r = int(os.environ.get("RANK", "0"))
    w = int(os.environ.get("WORLD_SIZE", "1"))
    lr = int(os.environ.get("LOCAL_RANK", "0"))
    return r, w, lr


def shard_pid_base(rank: int, particles_per_rank: int) -> int:
    """The first global particle key of a rank's shard.  Ranks hold
    consecutive key ranges, so N ranks of P particles draw exactly the random
    numbers one run of N x P particles draws (the counter RNG is keyed by the
    global particle index): weak scaling with no data-path exchange."""
    return int(rank) * int(particles_per_rank)


def max_over_ranks(value: float, dist, device) -> float:
    """The maximum of a per-rank time over all ranks (the job's time); the
    value itself on one process."""
    if dist is None:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    NAMES = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")

    def __init__(self, device: int):
        self.lines = []
        self.proc = None
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                          "-lms", "200", "-i", str(device)], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append((time.time(), line.strip()))

    def mark(self):
        return time.time()

    def stop(self, t0, t1):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        rows = [l for (t, l) in self.lines if t0 - 0.25 <= t <= t1 + 0.25] or [l for _, l in self.lines]
        sm, mx, reasons = [], [], set()
        for l in rows:
            f = [x.strip() for x in l.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx.append(float(f[2]))
            except ValueError:
                continue
            for name, val in zip(self.NAMES, f[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def _oracle_run(wl, n_particles: int, step_iter, view=None):
    """Oracle steps over ``n_particles`` particles of the workload, evenly
    strided through the seed order; yields seconds."""
    from oracle import oracle as O
    from kelp_b200.particles import make_state
    from kelp_b200.fields import LazyLerpField
    from kelp_b200.diffusion import DiffusionStepArgs
    view = view or O.MeshView(wl.mesh)
    n = min(n_particles, wl.P)
    idx = np.linspace(0, wl.P - 1, n).astype(np.int64)   # spread over the (sorted) seed order
    st = make_state(wl.lon[idx], wl.lat[idx], wl.z[idx])
    st = st.replace(failure_reason=np.zeros(n, np.int8))
    for k in step_iter:
        ia, ib, alpha0, dtn = wl.bracket(k)
        a, b = wl.snaps[ia], wl.snaps[ib]
        vel = a if alpha0 == 0.0 else LazyLerpField(a, b, alpha0)
        diff = None if wl.kh is None else DiffusionStepArgs("uniform", wl.kh[0], wl.kh[1], wl.seed, 0, k)
        t0 = time.perf_counter()
        out = O.step(st, vel, wl.mesh, wl.dt, 1.0, wl.scheme, vel_next=b, dt_to_next=dtn, w_interp=wl.w_interp,
                     diffusion=diff, view=view)
        dt = time.perf_counter() - t0
        st = st.replace(lon=out["lon"], lat=out["lat"], z=out["z"], status=out["status"],
                        nearest_node=out["nearest_node"], failure_reason=out["failure_reason"])
        yield k, n, dt


def cpu_baseline(wl, seconds: float = 10.0, n_particles: int = 200_000):
    """The oracle port on this host's cores over a bounded sample of the
    workload: up to ``n_particles`` particles, as many steps as fit in
    ~``seconds``."""
    from oracle import oracle as O
    done, t_used, steps, n = 0, 0.0, 0, 0

    def it():
        k = 0
        while k < wl.n_steps_run:
            yield k
            k += 1

    for k, n, dt in _oracle_run(wl, n_particles, it()):
        t_used += dt
        done += n
        steps += 1
        if t_used >= seconds:
            break
    return {"value": done / t_used, "unit": UNIT, "cores": O.threads(), "kind": "port",
            "sample": f"{steps} steps x {n} particles of {wl.name} (oracle C port, {O.threads()} threads)"}


REF_DIR = os.path.join(ROOT, "baseline", "_ref")


def _reference_kelp():
    """The reference package installed under baseline/_ref (pip --target), or
    None when it (or numba) cannot be imported here."""
    if not os.path.isdir(os.path.join(REF_DIR, "kelp")):
        return None
    if REF_DIR not in sys.path:
        sys.path.insert(0, REF_DIR)
    try:
        import kelp.numerics.integrators  # noqa: F401
        return sys.modules["kelp"]
    except Exception:
        return None


class _NumbaReference:
    """The reference's own Numba step path on the workload: KELP's Mesh +
    build_search + set_exact_nearest, node-layout VelocityField /
    LazyLerpField payloads as tracking._build_vel_payload makes them, and
    kelp.numerics.integrators.rk2_step / rk4_step / euler_step with
    DiffusionStepArgs for the split kick."""

    kind = "reference"

    def __init__(self, wl):
        from kelp.core.io import LazyLerpField, VelocityField
        from kelp.core.mesh import Mesh, build_node_to_elems, build_search, set_exact_nearest
        from kelp.core.particles import ParticleState
        from kelp.numerics import integrators as RI
        from kelp.numerics.diffusion import DiffusionStepArgs
        import numba
        self.numba = numba
        self.wl, self.Lazy, self.State, self.Diff = wl, LazyLerpField, ParticleState, DiffusionStepArgs
        self.fn = {"rk2": RI.rk2_step, "rk4": RI.rk4_step, "euler": RI.euler_step}[wl.scheme]
        m = wl.mesh
        en = np.ascontiguousarray(m.elem_nodes, dtype=np.int32)
        n2e, cnt = build_node_to_elems(m.n_nodes, en)
        self.mesh = Mesh(name=wl.name, nodes_lon=np.asarray(m.nodes_lon, np.float64),
                         nodes_lat=np.asarray(m.nodes_lat, np.float64), depth=np.asarray(m.depth, np.float64),
                         elem_nodes=en, elem_center_lon=np.asarray(m.elem_center_lon),
                         elem_center_lat=np.asarray(m.elem_center_lat), node_to_elems=n2e, node_to_elems_count=cnt,
                         sigma=np.asarray(m.sigma, np.float64))
        build_search(self.mesh)
        set_exact_nearest(self.mesh, True)
        self.fields = [VelocityField(u=f.u, v=f.v, w=f.w, eta=np.asarray(f.eta), uv_layout="node",
                                     uv_vertical=wl.uv_vertical) for f in wl.snaps]

    def threads(self):
        return int(self.numba.get_num_threads())

    def state(self, idx):
        wl, n = self.wl, idx.size
        return self.State(lon=wl.lon[idx].copy(), lat=wl.lat[idx].copy(), z=wl.z[idx].copy(),
                          status=np.ones(n, np.int32), nearest_node=np.full(n, -1, np.int32),
                          failure_reason=np.zeros(n, np.int8))

    def step(self, st, k):
        wl = self.wl
        ia, ib, alpha0, dtn = wl.bracket(k)
        a, b = self.fields[ia], self.fields[ib]
        vel = a if alpha0 == 0.0 else self.Lazy(a, b, alpha0)
        kw = dict(uv_interp="barycentric", w_interp=wl.w_interp, vel_next=b, dt_to_next=dtn)
        if wl.kh is not None:
            kw["diffusion"] = self.Diff(scheme="uniform", kh_x=wl.kh[0], kh_y=wl.kh[1], seed=wl.seed, real_id=0,
                                        step_i=k, pid_offset=0)
        return self.fn(st, vel, self.mesh, wl.dt, 1.0, **kw)


class _OraclePort:
    """The C restatement in oracle/ (the reference's arithmetic, all host
    threads), for workloads the reference's step cannot be driven on here."""

    kind = "port"

    def __init__(self, wl):
        from oracle import oracle as O
        self.O, self.wl, self.view = O, wl, O.MeshView(wl.mesh)

    def threads(self):
        return int(self.O.threads())

    def state(self, idx):
        from kelp_b200.particles import make_state
        wl = self.wl
        return make_state(wl.lon[idx], wl.lat[idx], wl.z[idx]).replace(failure_reason=np.zeros(idx.size, np.int8))

    def step(self, st, k):
        from kelp_b200.fields import LazyLerpField
        from kelp_b200.diffusion import DiffusionStepArgs
        wl = self.wl
        ia, ib, alpha0, dtn = wl.bracket(k)
        a, b = wl.snaps[ia], wl.snaps[ib]
        vel = a if alpha0 == 0.0 else LazyLerpField(a, b, alpha0)
        diff = None if wl.kh is None else DiffusionStepArgs("uniform", wl.kh[0], wl.kh[1], wl.seed, 0, k)
        out = self.O.step(st, vel, wl.mesh, wl.dt, 1.0, wl.scheme, vel_next=b, dt_to_next=dtn, w_interp=wl.w_interp,
                          diffusion=diff, view=self.view)
        return st.replace(lon=out["lon"], lat=out["lat"], z=out["z"], status=out["status"],
                          nearest_node=out["nearest_node"], failure_reason=out["failure_reason"])


def run_reference(args):
    """The reference's CPU implementation of the step on this host's cores, on
    the GPU arm's workload, metric and unit.  Every timed step is a real step
    of ``n`` particles (all of the workload's when the run fits the time
    budget, else an evenly strided sample sized to it); ``ms_per_step`` is the
    measured time of those steps, nothing is extrapolated."""
    rank, world, _ = env_rank()
    if rank != 0:
        return 0
    os.environ.setdefault("NUMBA_NUM_THREADS", str(len(os.sched_getaffinity(0))))
    from kelp_b200 import workloads
    wl = workloads.WORKLOADS[args.workload]()
    impl = None
    if wl.cohorts is None and not getattr(wl.mesh, "_nemo_cgrid", False) and _reference_kelp() is not None:
        impl = _NumbaReference(wl)
    if impl is None:
        impl = _OraclePort(wl)
    P = wl.P
    # warm-up 1 compiles (Numba) on a small sample; warm-up 2 times a full step
    small = np.linspace(0, P - 1, min(P, 20_000)).astype(np.int64)
    impl.step(impl.state(small), 0)
    full = np.arange(P)
    t0 = time.perf_counter()
    impl.step(impl.state(full), 0)
    t_full = time.perf_counter() - t0
    remaining_warm = max(0, args.warmup - 2)
    n = P
    if (args.steps + remaining_warm) * t_full > args.reference_budget_s:
        n = max(1000, int(P * args.reference_budget_s / ((args.steps + remaining_warm) * t_full)))
    idx = full if n == P else np.linspace(0, P - 1, n).astype(np.int64)
    st = impl.state(idx)
    for k in range(remaining_warm):
        st = impl.step(st, 1 + k)
    times = []
    for k in range(args.steps):
        t0 = time.perf_counter()
        st = impl.step(st, 1 + remaining_warm + k)
        times.append(time.perf_counter() - t0)
    total = sum(times)
    value = n * args.steps / total
    what = ("the reference's Numba rk2/rk4/euler_step (kelp " + getattr(sys.modules.get("kelp"), "__version__", "?")
            + ", baseline/_ref)") if impl.kind == "reference" else "the oracle C port of the reference's step"
    sample = (f"{args.steps} timed steps x {n} of {P} particles"
              + ("" if n == P else " (evenly strided sample)") + f", {what}, {impl.threads()} threads; "
              f"a full {P}-particle step measured {t_full:.2f} s")
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * total / args.steps,
            "higher_is_better": True, "scaling": "weak",
            "vs_baseline": (value / PUBLISHED[wl.name]) if wl.name in PUBLISHED else None, "dtype": "f64",
            "data": "synthetic", "config": _config(wl, args, world),
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": impl.threads(), "kind": impl.kind,
                             "sample": sample, "full_step_s": t_full, "particles_per_step": n},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def _config(wl, args, world):
    """The workload's config dict, the same for both arms."""
    return {"workload": wl.name, **wl.description, "particles_per_gpu": wl.P,
            "l2": "flushed between timed steps (256 MiB write)", "parallelism": f"replicas x{world}"}


def load_traffic(workload: str, form: str = "plain"):
    """Per-launch DRAM bytes of the step kernel from the committed ncu summary
    (lines: workload form kernel bytes ...)."""
    p = os.path.join(ROOT, "profiles", "traffic.txt")
    if not os.path.exists(p):
        return None
    for line in open(p):
        f = line.split()
        if len(f) >= 4 and f[0] == workload and f[1] == form:
            return float(f[3])
    return None


FORMS = {   # name -> (kernel form, snapshot storage)
    "plain": ("plain", None),
    "mixed": ("mixed", np.float32),
    "mixed_f16": ("mixed", np.float16),
    # the mixed form in fused multi-step launches replayed as a CUDA graph,
    # launch shape from the autotuner (kc_run_fused)
    "mixed_batched": ("mixed", np.float32),
}
BATCHED = {"mixed_batched"}


def _form_args(wl, k, slots, form):
    from kelp_b200 import _native as N
    code, store = FORMS[form]
    key = "f16" if store is np.float16 else "f32"
    return wl.step_args(k, slots[key], N.KC_MIXED if code == "mixed" else N.KC_PLAIN)


def _upload(ctx, wl, idx=None, pid_base=0):
    lon, lat, z = (wl.lon, wl.lat, wl.z) if idx is None else (wl.lon[idx], wl.lat[idx], wl.z[idx])
    P = lon.size
    ctx.upload_particles(lon, lat, z, np.full(P, 1, np.int32), np.full(P, -1, np.int32), np.zeros(P, np.int8),
                         np.arange(P, dtype=np.int64) + pid_base)


def _run_steps(ctx, wl, slots, form, k0, n, sort_every):
    for j in range(n):
        if sort_every > 0 and j % sort_every == 0:
            ctx.sort()
        ctx.step(_form_args(wl, k0 + j, slots, form))
    ctx.synchronize()
    return ctx.download_particles()


def accuracy(ctx, wl, slots, forms, sort_every, n_sub):
    """Separation of each non-plain form from the plain float64 form: after
    24 h on every particle, and after the configuration's full horizon on a
    uniform subset of n_sub particles; with the dispersion of each run."""
    from kelp_b200 import accuracy as A
    out = {}
    h24 = max(1, int(round(86400.0 / wl.dt)))
    ref = {}
    _upload(ctx, wl)
    ref["24h"] = _run_steps(ctx, wl, slots, "plain", 0, h24, sort_every)
    idx = np.arange(min(n_sub, wl.P))
    _upload(ctx, wl, idx)
    ref["full"] = _run_steps(ctx, wl, slots, "plain", 0, wl.n_steps_run, sort_every)
    for form in forms:
        if form == "plain" or form in BATCHED:   # fused launches compute the per-step results bit for bit
            continue
        _upload(ctx, wl)
        t24 = _run_steps(ctx, wl, slots, form, 0, h24, sort_every)
        _upload(ctx, wl, idx)
        tfull = _run_steps(ctx, wl, slots, form, 0, wl.n_steps_run, sort_every)
        out[form] = {"after_24h": {"steps": h24, "particles": wl.P, **A.separation_stats(ref["24h"], t24)},
                     "after_horizon": {"steps": wl.n_steps_run, "particles": int(idx.size),
                                       **A.separation_stats(ref["full"], tfull)},
                     "dispersion_m2_horizon": {"plain": A.dispersion_m2(wl.lon[idx], wl.lat[idx], ref["full"]),
                                               form: A.dispersion_m2(wl.lon[idx], wl.lat[idx], tfull)}}
    return out


def run_cohorts(args, wl, ctx, local):
    """Batched cohorts (one GPU): every cohort x ensemble member in one slot
    array, stepped by fused multi-step launches (autotuned block size, steps
    per launch and re-sort interval) against one launch per cohort x member
    per step (kc_step_range), the reference's way of running them."""
    from kelp_b200 import autotune, roofline
    from kelp_b200.device import pinned_empty
    code, store = FORMS[args.form]
    slots = {"f16" if store is np.float16 else "f32": ctx.slots_for(wl.snaps, store or np.float32)}
    P = wl.P
    t0 = wl.t0_step

    def reset():
        ctx.upload_particles(wl.lon, wl.lat, wl.z, np.full(P, 4, np.int32), np.full(P, -1, np.int32),
                             np.zeros(P, np.int8), wl.pid, wl.release_step)
        ctx.set_realization(wl.real_id)

    def make_steps(k, n):
        return [_form_args(wl, kk, slots, args.form) for kk in range(k, k + n)]

    key = autotune.mesh_signature(wl.mesh, wl.dims, wl.scheme, args.form, P)
    tuned = autotune.tune(ctx, key, reset, make_steps, t0, window=args.tune_window, steps_per_launch=(1, 12),
                          sort_every=(12, 24))
    spl, se = tuned["steps_per_launch"], tuned["sort_every"]
    sampler = ClockSampler(local)
    time.sleep(0.6)
    t_wall0 = time.time()
    # batched: fused launches over every slot
    reset()
    autotune.run_window(ctx, make_steps, t0, spl, spl, se)
    ctx.synchronize()
    if ctx.device_errors():
        raise RuntimeError("device-side iteration cap hit during warm-up")
    K = max(spl, (args.steps + spl - 1) // spl * spl)
    ctx.record(0)
    autotune.run_window(ctx, make_steps, t0 + spl, K, spl, se)
    ctx.record(1)
    batched_ms = ctx.elapsed_ms(0, 1)
    batched_launches = K // spl + 15 * ((K + se - 1) // se)
    errs = ctx.device_errors()
    # one launch per cohort x member per step, no re-sort (the cohorts' slots
    # must stay contiguous)
    reset()
    Kb = max(1, min(args.steps, 4))
    for (b, cnt, r, c) in wl.cohorts:
        ctx.step_range(make_steps(t0, 1)[0], b, cnt)
    ctx.synchronize()
    ctx.record(0)
    for k in range(Kb):
        a = make_steps(t0 + 1 + k, 1)[0]
        for (b, cnt, r, c) in wl.cohorts:
            ctx.step_range(a, b, cnt)
    ctx.record(1)
    per_cohort_ms = ctx.elapsed_ms(0, 1)
    t_wall1 = time.time()
    clocks = sampler.stop(t_wall0, t_wall1)

    # end to end: page-locked host slots through kc_step_host every step
    names = {"lon": np.float64, "lat": np.float64, "z": np.float64, "status": np.int32, "nearest_node": np.int32,
             "failure_reason": np.int8, "u": np.float64, "v": np.float64, "w": np.float64}
    # one set of arrays updated in place (kc_step_host allows it: a chunk is
    # read before its new state is written back)
    buf = {n: pinned_empty((P,), t) for n, t in names.items()}
    for n, src in (("lon", wl.lon), ("lat", wl.lat), ("z", wl.z)):
        buf[n][:] = src
    buf["status"][:] = 4
    buf["nearest_node"][:] = -1
    buf["failure_reason"][:] = 0
    ids = {"pid": pinned_empty((P,), np.int64), "real_id": pinned_empty((P,), np.int32),
           "release_step": pinned_empty((P,), np.int32)}
    ids["pid"][:] = wl.pid
    ids["real_id"][:] = wl.real_id
    ids["release_step"][:] = wl.release_step
    ins = ("lon", "lat", "z", "status", "nearest_node", "failure_reason")
    ctx.step_host(make_steps(t0, 1)[0], dict({n: buf[n] for n in ins}, **ids), buf)
    e2e_steps = 3
    ctx.record(2)
    for k in range(e2e_steps):
        ctx.step_host(make_steps(t0 + 1 + k, 1)[0], dict({n: buf[n] for n in ins}, **ids), buf)
    ctx.record(3)
    e2e_ms = ctx.elapsed_ms(2, 3)

    peak, kind = peaks()
    fb = 2 if store is np.float16 else 4
    bpp = roofline.bytes_per_particle_step(wl.mesh, wl.scheme, wl.dims, fb, kick=True, w_code=1)
    value = P * K / (batched_ms * 1e-3)
    achieved = bpp["total"] * P * K / (batched_ms * 1e-3) / 1e9
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": 1, "steps": K, "warmup": spl,
            "ms_per_step": batched_ms / K, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64" if code == "plain" else "f32 interp + f64 state", "data": "synthetic",
            "config": {"workload": wl.name, "form": args.form,
                       **{k: v for k, v in wl.description.items() if k != "cohort_sizes"},
                       "l2": "inputs larger than L2 (fields 1.1 GB, slots 7.6 GB); not flushed",
                       "parallelism": "one GPU, all cohorts x members in one array"},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "peak_kind": kind, "traffic": None,
                         "algorithmic_bytes_per_particle_step": bpp["total"]},
            "forms": {"batched_fused": {"value": value, "ms_per_step": batched_ms / K, "launches": batched_launches},
                      "per_cohort_launches": {"value": P * Kb / (per_cohort_ms * 1e-3), "ms_per_step": per_cohort_ms / Kb,
                                              "launches": Kb * len(wl.cohorts)}},
            "autotune": {k: v for k, v in tuned.items() if k != "trials"},
            "autotune_trials": tuned.get("trials"),
            "e2e": {"value": P * e2e_steps / (e2e_ms * 1e-3), "unit": UNIT, "h2d_bytes_per_step": P * (33 + 16),
                    "d2h_bytes_per_step": P * 57, "steps": e2e_steps, "form": args.form,
                    "api": "kc_step_host, page-locked host arrays"},
            "gpu_launches": batched_launches, "clocks": clocks, "device_errors": errs}
    if not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(wl, n_particles=50_000)
    print(json.dumps(line), flush=True)
    return 0


def _time_batched(ctx, wl, slots, form, args, pid_base, barrier, dist, local):
    """The batched form: the autotuner's launch shape (particles per block,
    steps per launch, re-sort interval) on a short window, then args.steps
    steps in fused launches replayed from a CUDA graph, timed as one region
    (the inputs -- 3.6 GB of snapshots, 6 M particles -- exceed L2; nothing is
    flushed inside a fused launch)."""
    from kelp_b200 import autotune

    def reset():
        _upload(ctx, wl, pid_base=pid_base)

    def make_steps(k, n):
        out = []
        for kk in range(k, k + n):
            a = _form_args(wl, kk, slots, form)
            a.pid_offset = pid_base
            out.append(a)
        return out

    key = autotune.mesh_signature(wl.mesh, wl.dims, wl.scheme, form, wl.P)
    tuned = autotune.tune(ctx, key, reset, make_steps, 0, window=8, steps_per_launch=(1, 4, 8),
                          sort_every=(8, 16), use_cache=False)
    spl, se = tuned["steps_per_launch"], tuned["sort_every"]
    reset()
    autotune.run_window(ctx, make_steps, 0, args.warmup, spl, se)
    ctx.synchronize()
    if ctx.device_errors():
        raise RuntimeError("device-side iteration cap hit during warm-up")
    barrier()
    K = args.steps
    ctx.record(0)
    autotune.run_window(ctx, make_steps, args.warmup, K, spl, se)
    ctx.record(1)
    barrier()
    total = max_over_ranks(ctx.elapsed_ms(0, 1), dist, f"cuda:{local}")
    launches = (K + spl - 1) // spl + 15 * ((K + se - 1) // se)
    return {"total_ms": total, "kernel_ms": total / K, "sort_ms": 0.0, "launches": launches,
            "errors": ctx.device_errors(),
            "launch_shape": {k: tuned[k] for k in ("block", "steps_per_launch", "sort_every", "ms_per_step")}}


def run_b200(args):
    rank, world, local = env_rank()
    dist = None
    if world > 1:
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", init_method="env://", timeout=__import__("datetime").timedelta(seconds=300))
    from kelp_b200 import workloads, roofline
    from kelp_b200.device import set_default_device, default_context, pinned_empty

    wl = workloads.WORKLOADS[args.workload]()
    set_default_device(local)
    ctx = default_context()
    ctx.ensure_mesh(wl.mesh)
    if wl.cohorts is not None:
        if world > 1:
            raise SystemExit("the batched-cohort workload runs on one GPU")
        if args.form in ("auto", "mixed_batched"):
            args.form = "mixed"   # every cohort form here is batched
        return run_cohorts(args, wl, ctx, local)
    if wl.dims == 3 and wl.uv_vertical != "layer":
        ctx.ensure_depth_points(wl.mesh, wl.uv_vertical)
    forms = [f.strip() for f in args.forms.split(",") if f.strip()]
    if getattr(wl.mesh, "_nemo_cgrid", False):   # C-grid meshes: no fused multi-step launch
        forms = [f for f in forms if f not in BATCHED]
        if args.form in ("auto", "mixed_batched"):
            args.form = "mixed"
    if args.form == "auto":
        forms += [f for f in ("mixed", "mixed_batched") if f not in forms]
    elif args.form not in forms:
        forms.append(args.form)
    slots = {"f32": ctx.slots_for(wl.snaps, np.float32)}
    if any(FORMS[f][1] is np.float16 for f in forms):
        slots["f16"] = ctx.slots_for(wl.snaps, np.float16)
    P = wl.P
    pid_base = shard_pid_base(rank, P)

    def barrier():
        if dist is not None:
            dist.barrier()
        ctx.synchronize()

    sampler = ClockSampler(local)
    time.sleep(0.6)
    t_wall0 = time.time()
    timed = {}
    for form in forms:
        if form in BATCHED:
            timed[form] = _time_batched(ctx, wl, slots, form, args, pid_base, barrier, dist, local)
            continue
        _upload(ctx, wl, pid_base=pid_base)
        for k in range(args.warmup):
            if args.sort_every > 0 and k == 0:
                ctx.sort()
            ctx.step(_form_args(wl, k, slots, form))
        ctx.synchronize()
        if ctx.device_errors():
            raise RuntimeError("device-side iteration cap hit during warm-up")
        barrier()
        step_ms, sort_ms, launches = [], [], 0
        for j, k in enumerate(range(args.warmup, args.warmup + args.steps)):
            ctx.l2_flush()
            ctx.record(0)
            if args.sort_every > 0 and j % args.sort_every == 0:
                ctx.sort()
                ctx.record(2)
                launches += 15      # key kernel, radix passes, one gather per particle array
            ctx.step(_form_args(wl, k, slots, form))
            launches += 1
            ctx.record(1)
            step_ms.append(ctx.elapsed_ms(0, 1))
            if args.sort_every > 0 and j % args.sort_every == 0:
                sort_ms.append(ctx.elapsed_ms(0, 2))
        barrier()
        total = max_over_ranks(float(sum(step_ms)), dist, f"cuda:{local}")
        timed[form] = {"total_ms": total, "kernel_ms": (sum(step_ms) - sum(sort_ms)) / len(step_ms),
                       "sort_ms": float(sum(sort_ms)), "launches": launches, "errors": ctx.device_errors()}
    t_wall1 = time.time()
    clocks = sampler.stop(t_wall0, t_wall1)
    if args.form == "auto":   # the headline: the faster launch strategy of the mixed form
        args.form = min(("mixed", "mixed_batched"), key=lambda f: timed[f]["total_ms"])

    # end to end through the C-ABI host-buffer step (kc_step_host), headline
    # form: every step uploads the state from page-locked host arrays, steps
    # it and downloads the new state (positions, status, anchors, failure
    # reasons, velocities), chunked so the copies overlap the step
    names_in = {"lon": np.float64, "lat": np.float64, "z": np.float64, "status": np.int32,
                "nearest_node": np.int32, "failure_reason": np.int8}
    names_out = dict(names_in, u=np.float64, v=np.float64, w=np.float64)
    bufs = []
    for _ in range(2):
        d = {name: pinned_empty((P,), dt_) for name, dt_ in names_out.items()}
        bufs.append(d)
    bufs[0]["lon"][:] = wl.lon
    bufs[0]["lat"][:] = wl.lat
    bufs[0]["z"][:] = wl.z
    bufs[0]["status"][:] = 1
    bufs[0]["nearest_node"][:] = -1
    bufs[0]["failure_reason"][:] = 0
    e2e_steps = max(1, min(args.steps, 20))

    def e2e_args(k):
        a_ = _form_args(wl, k, slots, args.form)
        a_.pid_offset = pid_base
        return a_

    ctx.step_host(e2e_args(0), {n: bufs[0][n] for n in names_in}, bufs[1])   # warm-up
    barrier()
    ctx.record(2)
    for k in range(e2e_steps):
        src, dst = bufs[k % 2], bufs[(k + 1) % 2]
        ctx.step_host(e2e_args(k), {n: src[n] for n in names_in}, dst)
    ctx.record(3)
    e2e_ms = max_over_ranks(ctx.elapsed_ms(2, 3), dist, f"cuda:{local}")
    h2d = P * (8 + 8 + 8 + 4 + 4 + 1)
    d2h = P * (8 * 6 + 4 + 4 + 1)

    acc = None
    if world == 1 and not args.no_accuracy and len(forms) > 1:
        acc = accuracy(ctx, wl, slots, forms, args.sort_every, args.accuracy_particles)

    if rank == 0:
        peak, kind = peaks()
        per_form = {}
        for form in forms:
            fb = 2 if FORMS[form][1] is np.float16 else 4
            bpp = roofline.bytes_per_particle_step(wl.mesh, wl.scheme, wl.dims, fb, kick=wl.kh is not None,
                                                   w_code=0 if wl.w_interp == "nearest" else 1)
            t = timed[form]
            per_form[form] = {"value": world * P * args.steps / (t["total_ms"] * 1e-3),
                              "ms_per_step": t["total_ms"] / args.steps, "kernel_ms": t["kernel_ms"],
                              "achieved_gbs": bpp["total"] * P / (t["kernel_ms"] * 1e-3) / 1e9,
                              "bytes_per_particle_step": bpp["total"], "device_errors": t["errors"]}
            if "launch_shape" in t:
                per_form[form]["launch_shape"] = t["launch_shape"]
                per_form[form]["note"] = "fused launches + CUDA graph, re-sort included; inputs exceed L2, no flush"
        head = per_form[args.form]
        traffic = load_traffic(wl.name, args.form)
        value = head["value"]
        dtype = "f64" if args.form == "plain" else ("f32 interp + f64 state, f16 snapshots"
                                                    if FORMS[args.form][1] is np.float16 else
                                                    "f32 interp + f64 state")
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": head["ms_per_step"], "higher_is_better": True,
                "scaling": "weak", "vs_baseline": (value / PUBLISHED[wl.name]) if wl.name in PUBLISHED else None,
                "dtype": dtype, "data": "synthetic", "form": args.form,
                "config": _config(wl, args, world),
                "roofline": {"bound": "hbm", "achieved": head["achieved_gbs"], "peak": peak, "unit": "GB/s",
                             "frac": head["achieved_gbs"] / peak, "peak_kind": kind, "traffic": traffic,
                             "algorithmic_bytes_per_particle_step": head["bytes_per_particle_step"]},
                "forms": per_form,
                "e2e": {"value": world * P * e2e_steps / (e2e_ms * 1e-3), "unit": UNIT,
                        "h2d_bytes_per_step": h2d * world, "d2h_bytes_per_step": d2h * world,
                        "steps": e2e_steps, "form": args.form, "api": "kc_step_host, page-locked host arrays"},
                "gpu_launches": timed[args.form]["launches"], "clocks": clocks,
                "resort": {"every_steps": args.sort_every, "ms_total": timed[args.form]["sort_ms"]}}
        if acc is not None:
            line["accuracy_vs_plain"] = acc
        if world == 1 and not args.no_cpu_baseline:
            line["cpu_baseline"] = cpu_baseline(wl)
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--workload", default="c3",
                    help="c1, c2, c3 (default: the published configuration), c4 (batched cohorts), c3small, c4small")
    ap.add_argument("--form", default="auto", choices=sorted(FORMS) + ["auto"],
                    help="the form the headline value reports (auto: the faster of mixed and mixed_batched)")
    ap.add_argument("--forms", default="plain,mixed,mixed_batched,mixed_f16", help="forms timed beside it")
    ap.add_argument("--no-accuracy", action="store_true")
    ap.add_argument("--tune-window", type=int, default=12, help="steps timed per autotuner candidate (c4)")
    ap.add_argument("--accuracy-particles", type=int, default=200_000,
                    help="particles of the full-horizon separation run")
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--sort-every", type=int, default=16, help="re-sort particles by hash cell every N steps")
    ap.add_argument("--reference-budget-s", type=float, default=150.0,
                    help="CPU seconds the --impl reference timed steps may take (beyond it: a particle sample)")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return run_reference(args)
    return run_b200(args)


if __name__ == "__main__":
    sys.exit(main())
