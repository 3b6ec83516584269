"""The launch autotuner of the fused multi-step path: particles per block,
steps per launch and re-sort interval, chosen by timing on the device and
cached per mesh type.

A mesh type is what the step's cost depends on: node and element counts,
vertex count per element, mean node valence, 2-D or 3-D, scheme, numerical
form, and the particle count (to a power of two).  Each candidate runs a
short window of steps from the same uploaded state (``reset``), with the
re-sort inside the window, timed with CUDA events on the library's stream; the
fastest is kept.  The results are written to a JSON file
(``KELP_B200_TUNE_CACHE``, default ``~/.cache/kelp_b200/autotune.json``) and
reused by later runs on the same mesh type.  Tuning changes no result: every
candidate computes the same particles bit for bit (the fused launch equals
per-step launches, and the re-sort keeps every particle's keys).
"""
from __future__ import annotations

import json
import math
import os
from typing import Callable, Iterable, List, Optional

import numpy as np

DEFAULT_BLOCKS = (128, 256)
DEFAULT_STEPS_PER_LAUNCH = (1, 6, 12)
DEFAULT_SORT_EVERY = (12, 24, 48)


def cache_path() -> str:
    return os.environ.get("KELP_B200_TUNE_CACHE",
                          os.path.join(os.path.expanduser("~"), ".cache", "kelp_b200", "autotune.json"))


def mesh_signature(mesh, dims: int, scheme: str, form: str, P: int) -> str:
    en = np.asarray(mesh.elem_nodes)
    cnt = np.asarray(mesh.node_to_elems_count)
    valence = float(cnt.mean()) if cnt.size else 0.0
    pbin = 1 << max(0, int(math.log2(max(P, 1))))
    return (f"N{int(np.asarray(mesh.nodes_lon).size)}-E{en.shape[0]}-v{en.shape[1]}-val{valence:.2f}"
            f"-d{dims}-{scheme}-{form}-P{pbin}")


def _load() -> dict:
    try:
        with open(cache_path()) as fh:
            return json.load(fh)
    except (OSError, ValueError):
        return {}


def _store(db: dict) -> None:
    p = cache_path()
    try:
        os.makedirs(os.path.dirname(p), exist_ok=True)
        tmp = p + ".tmp"
        with open(tmp, "w") as fh:
            json.dump(db, fh, indent=1, sort_keys=True)
        os.replace(tmp, p)
    except OSError:
        pass   # a read-only home: tune again next time


def run_window(ctx, make_steps: Callable[[int, int], list], k0: int, n_steps: int, steps_per_launch: int,
               sort_every: int, beach: Optional[Callable[[int, int], list]] = None, graph: bool = True) -> None:
    """n_steps steps from global step k0 in fused launches of steps_per_launch
    steps, re-sorting before every sort_every-th step (a multiple of the
    launch length)."""
    k = 0
    while k < n_steps:
        n = min(steps_per_launch, n_steps - k)
        if sort_every > 0 and k % sort_every == 0:
            ctx.sort()
        ctx.run_fused(make_steps(k0 + k, n), None if beach is None else beach(k0 + k, n), graph=graph)
        k += n


def tune(ctx, key: str, reset: Callable[[], None], make_steps: Callable[[int, int], list], k0: int = 0, *,
         window: int = 24, blocks: Iterable[int] = DEFAULT_BLOCKS,
         steps_per_launch: Iterable[int] = DEFAULT_STEPS_PER_LAUNCH,
         sort_every: Iterable[int] = DEFAULT_SORT_EVERY, use_cache: bool = True) -> dict:
    """The fastest (block, steps_per_launch, sort_every) for this mesh type.

    ``reset()`` re-uploads the starting particles; ``make_steps(k, n)``
    returns the argument blocks of global steps k .. k + n - 1.  Sort
    intervals that are not a multiple of the launch length are skipped."""
    db = _load() if use_cache else {}
    if use_cache and key in db:
        out = dict(db[key])
        out["cached"] = True
        ctx.set_fused_block(out["block"])
        return out
    trials: List[dict] = []
    for blk in blocks:
        ctx.set_fused_block(blk)
        for spl in steps_per_launch:
            for se in sort_every:
                if se % spl:
                    continue
                reset()
                run_window(ctx, make_steps, k0, spl, spl, se)      # warm-up: graph capture, first anchors
                ctx.synchronize()
                ctx.record(10)
                run_window(ctx, make_steps, k0 + spl, window, spl, se)
                ctx.record(11)
                ms = ctx.elapsed_ms(10, 11) / window
                trials.append({"block": blk, "steps_per_launch": spl, "sort_every": se, "ms_per_step": ms})
    if not trials:
        raise ValueError("no admissible candidate (sort intervals must be multiples of the launch lengths)")
    best = min(trials, key=lambda t: t["ms_per_step"])
    out = dict(best, key=key, window=window, trials=trials)
    ctx.set_fused_block(best["block"])
    if use_cache:
        db[key] = {k: v for k, v in out.items() if k != "cached"}
        _store(db)
    out["cached"] = False
    return out
