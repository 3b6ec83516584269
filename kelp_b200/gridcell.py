"""The grid-hash cell rules: ``legacy`` (the reader's automatic cell) and
``occupancy`` (a ladder of smaller cells measured on sampled element
centres), KELP's ``core.mesh.choose_grid_hash_cell`` /
``apply_grid_hash_cell_rule`` / ``describe_grid_hash``
(``src/kelp/core/mesh.py:464-710``).

The per-sample work of every candidate -- each sample's exact nearest node,
the candidate's node counts and their 2-D prefix table, the 3x3 occupancy,
the outside-window flag, the certificate's verdict and the scan-cost proxy
(the reference's ``_gh_sample_stats``, ``mesh.py:384-461``) -- runs on the
device in ``kc_grid_cell_stats``.  The host keeps the decisions: the sample
(the same seeded draw), the ladder of candidate cells and its stopping rules,
the summary statistics (the same numpy reductions over the same arrays) and
the choice in either mode, with the reference's report dictionary and
reasons.
"""
from __future__ import annotations

import numpy as np

from .mesh import (_GRID_HASH_MAX_CELLS, _gh_far_rows_for, _gh_grid_geometry, _gh_lon_branch, build_grid_hash,
                   set_grid_hash_cell)

GRID_HASH_CELL_RULES = ("occupancy", "legacy")


def _ladder_row(k, cell, far_rows, nx, ny, stats, max_unprovable, max_hash_mb):
    """One candidate's summary: the window occupancy quantiles, the shares of
    empty windows, widened searches and outside-window anchors, and the mean
    scan cost (mesh.py:577-585)."""
    occ, cost, unprov, approx = stats
    n_cells = int(nx * ny)
    hash_mb = float(4.0 * (n_cells + 1) / 1e6)
    unprov_share = float(np.mean(unprov))
    return {"cell": float(cell), "far_rows": int(far_rows), "n_cells": n_cells, "hash_mb": hash_mb,
            "median": float(np.median(occ)), "p95": float(np.percentile(occ, 95)),
            "empty": float(np.mean(occ == 0)), "unprovable": unprov_share,
            "approx": float(np.mean(approx)), "mean_cost": float(np.mean(cost)),
            "eligible": bool(k == 0 or (unprov_share <= max_unprovable and hash_mb <= max_hash_mb))}


def choose_grid_hash_cell(mesh, *, ctx=None, exact=None, sample: int = 200_000, seed: int = 0,
                          min_median: int = 8, approx_tol: float = 0.005, max_far_rows: int = 64,
                          steps: int = 12, min_gain: float = 2.75, max_unprovable: float = 0.20,
                          max_hash_mb: float = 128.0):
    """Measure candidate cells on sampled element centres and pick one
    (``mesh.py:464-616``); returns ``(cell, report)`` and leaves the mesh's
    cell as it is.

    Candidates are the current cell divided by sqrt(2)^k, k = 0..steps,
    while the exact search's row budget stays within ``max_far_rows`` and the
    grid within the cell cap (the current cell is always measured).  Exact
    mode (default: the mesh's ``exact_nearest`` flag) takes the eligible
    candidate of least mean scan cost (eligible: at most ``max_unprovable``
    widened searches and a hash of at most ``max_hash_mb``), and leaves the
    current cell only for a predicted gain of at least ``min_gain``.
    Approximate mode takes the smallest candidate with no empty window, a
    median occupancy of at least ``min_median`` and no more outside-window
    anchors than the current cell's plus ``approx_tol``.  ``ctx``: the
    device context (default: the process's); the mesh is made resident on it.
    """
    from .device import default_context
    if getattr(mesh, "_gh_offsets", None) is None:
        build_grid_hash(mesh)
    if exact is None:
        exact = bool((getattr(mesh, "metadata", None) or {}).get("exact_nearest", False))
    legacy = float(mesh._gh_cell_size)
    mode = "exact" if exact else "approx"

    def keep(reason, n=0):
        return legacy, {"rule": "occupancy", "mode": mode, "legacy": legacy, "chosen": legacy,
                        "candidates": [], "sample": int(n), "reason": reason}

    E = int(np.asarray(mesh.elem_nodes).shape[0])
    if E == 0:
        return keep("no elements to sample: the reader's automatic cell")
    idx = (np.sort(np.random.default_rng(seed).choice(E, sample, replace=False)) if E > sample
           else np.arange(E))
    qlon = np.ascontiguousarray(np.asarray(mesh.elem_center_lon)[idx], dtype=np.float64)
    qlat = np.ascontiguousarray(np.asarray(mesh.elem_center_lat)[idx], dtype=np.float64)
    fin = np.isfinite(qlon) & np.isfinite(qlat)
    if not fin.all():
        qlon, qlat = qlon[fin], qlat[fin]
    if qlon.size == 0:
        return keep("no finite element centre to sample: the reader's automatic cell")
    ctx = ctx if ctx is not None else default_context()
    ctx.ensure_mesh(mesh)
    lon_b, wrap = _gh_lon_branch(np.asarray(mesh.nodes_lon, dtype=np.float64))
    lat = np.asarray(mesh.nodes_lat, dtype=np.float64)
    found = None
    rows = []
    for k in range(steps + 1):
        cell = legacy / (np.sqrt(2.0) ** k)
        far_rows = _gh_far_rows_for(mesh, cell)
        if k > 0 and far_rows > max_far_rows:
            break
        lon_min, lat_min, nx, ny = _gh_grid_geometry(lon_b, lat, cell, wrap)
        if k > 0 and nx * ny > _GRID_HASH_MAX_CELLS:
            break
        nn, occ, cost, unprov, approx = ctx.grid_cell_stats(lon_b, cell, lon_min, lat_min, nx, ny, wrap, qlon, qlat)
        if found is None:
            found = nn >= 0                       # -1 only on an empty grid
            if not found.any():
                return keep("no sample has a nearest node: the reader's automatic cell")
        stats = (occ, cost, unprov, approx) if found.all() else tuple(a[found] for a in (occ, cost, unprov, approx))
        rows.append(_ladder_row(k, cell, far_rows, nx, ny, stats, max_unprovable, max_hash_mb))
    n_used = int(np.count_nonzero(found))
    base = rows[0]
    if exact:
        best = min((r for r in rows if r["eligible"]), key=lambda r: (r["mean_cost"], -r["cell"]))
        gain = base["mean_cost"] / best["mean_cost"] if best["mean_cost"] > 0 else 1.0
        if best is not base and gain < min_gain:
            reason = (f"keep the legacy cell: the cheapest eligible candidate {best['cell']:.4g} "
                      f"deg predicts only {gain:.2f}x (< {min_gain:g}x) on the scan cost "
                      f"({best['mean_cost']:.1f} vs {base['mean_cost']:.1f} nodes/query)")
            best = base
        else:
            reason = (f"smallest mean scan cost {best['mean_cost']:.1f} nodes/query "
                      f"(legacy {base['mean_cost']:.1f}, {gain:.2f}x) among the candidates "
                      f"with widening <= {100 * max_unprovable:.0f} % and hash <= "
                      f"{max_hash_mb:g} MB")
    else:
        fit = [r for r in rows if r["empty"] == 0.0 and r["median"] >= min_median
               and r["approx"] <= base["approx"] + approx_tol
               and (r is base or r["hash_mb"] <= max_hash_mb)]
        best = min(fit, key=lambda r: r["cell"]) if fit else base
        reason = ("smallest cell with no empty window, median >= {0} and no added approximate anchor".format(min_median)
                  if fit else "no smaller cell keeps every window non-empty without approximate anchors")
    return float(best["cell"]), {"rule": "occupancy", "mode": mode, "legacy": legacy, "chosen": float(best["cell"]),
                                 "reason": reason, "candidates": rows, "sample": n_used}


def apply_grid_hash_cell_rule(mesh, rule: str = "occupancy", *, ctx=None, **chooser_kwargs) -> dict:
    """Apply a cell rule to the mesh and return its report, also kept as
    ``mesh._gh_report`` (``mesh.py:619-682``).  An explicit pin is never
    overridden; the same rule in the same mode is not re-run; another rule
    or mode after an earlier ``occupancy`` decision starts again from the
    reader's cell.  ``occupancy`` pins a different choice
    (``set_grid_hash_cell``) so later rebuilds keep it; the metadata records
    ``grid_hash_cell_rule`` and, for ``occupancy``, ``grid_hash_cell_mode``."""
    rule = str(rule).lower()
    if rule not in GRID_HASH_CELL_RULES:
        raise ValueError(f"grid_hash_cell_rule must be one of {GRID_HASH_CELL_RULES}, got {rule!r}")
    md = mesh.metadata
    if getattr(mesh, "_gh_offsets", None) is None:
        build_grid_hash(mesh)
    exact = chooser_kwargs.get("exact")
    mode = "exact" if (bool(md.get("exact_nearest", False)) if exact is None else exact) else "approx"
    earlier = md.get("grid_hash_cell_rule")
    previous = getattr(mesh, "_gh_report", None)
    if "grid_hash_cell" in md and earlier in (None, "explicit"):
        md["grid_hash_cell_rule"] = "explicit"
        mesh._gh_report = {"rule": "explicit", "chosen": float(mesh._gh_cell_size), "legacy": None, "mode": None,
                           "reason": "explicit cell (grid_hash_cell_size)", "candidates": [], "sample": 0}
        return mesh._gh_report
    if (earlier == rule and (rule == "legacy" or md.get("grid_hash_cell_mode") == mode)
            and previous is not None and previous.get("chosen") == float(mesh._gh_cell_size)):
        return previous
    if earlier is not None:
        for key in ("grid_hash_cell", "grid_hash_cell_rule", "grid_hash_cell_mode"):
            md.pop(key, None)
        build_grid_hash(mesh)
    if rule == "legacy":
        report = {"rule": "legacy", "chosen": float(mesh._gh_cell_size), "legacy": float(mesh._gh_cell_size),
                  "mode": None, "reason": "legacy rule: the reader's automatic cell", "candidates": [], "sample": 0}
    else:
        cell, report = choose_grid_hash_cell(mesh, ctx=ctx, **chooser_kwargs)
        if cell != mesh._gh_cell_size:
            set_grid_hash_cell(mesh, cell)
        md["grid_hash_cell_mode"] = mode
    md["grid_hash_cell_rule"] = rule
    mesh._gh_report = report
    return report


def describe_grid_hash(mesh) -> str:
    """One line on the cell and the rule that chose it, with the chosen
    candidate's window statistics beside the reader's cell
    (``mesh.py:685-706``)."""
    r = getattr(mesh, "_gh_report", None)
    cell = float(mesh._gh_cell_size)
    if r is not None and r.get("chosen") != cell:
        r = None
    if r is None or not r.get("candidates"):
        rule = (r or {}).get("rule") or mesh.metadata.get("grid_hash_cell_rule", "reader auto")
        return f"grid hash: cell {cell:.4g} deg ({rule}), far_rows {int(mesh._gh_far_rows)}"
    by_cell = {c["cell"]: c for c in r["candidates"]}
    base, ch = r["candidates"][0], by_cell[r["chosen"]]
    return (f"grid hash: cell {ch['cell']:.4g} deg by occupancy/{r['mode']} "
            f"(legacy {base['cell']:.4g}): window median {ch['median']:.0f} / p95 "
            f"{ch['p95']:.0f} nodes (legacy {base['median']:.0f} / {base['p95']:.0f}), "
            f"empty {100 * ch['empty']:.1f} %, widening {100 * ch['unprovable']:.1f} % "
            f"(legacy {100 * base['unprovable']:.1f} %), scan cost {ch['mean_cost']:.0f} vs "
            f"{base['mean_cost']:.0f} nodes/query, far_rows {ch['far_rows']}, "
            f"{r['sample']} centres — {r['reason']}")
