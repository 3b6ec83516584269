"""Algorithmic bytes of one particle-step: the fixed roofline denominator.

Compulsory unique bytes at element granularity with no cross-particle reuse,
EXCLUDING the grid-hash window scan (so a larger hash cell cannot inflate the
figure), computed from the mesh's own statistics:

* particle state: read lon, lat (z), status, anchor; write them back plus the
  velocity diagnostics and the failure reason -- 65 B in 2-D, 89 B in 3-D;
* per evaluation site (anchor + containment): 4 B hash offset,
  4 B x mean node valence (node->element ids), 4 B x max_v (element nodes),
  16 B x mean vertices (node lon/lat);
* per velocity stage: vertices x 2 components x 2 distinct snapshots read
  (the bracket pair; the stage target is the bracket end) x field bytes,
  per vertical row read;
* W (3-D) per stage: nearest -- 2 interfaces x 2 snapshots x field bytes;
  barycentric -- vertices x (8 B depth + 2 interfaces x 2 snapshots x bytes).

On a NEMO C-grid mesh a stage reads one cell instead: its corner ids (16 B),
raster index and wet levels (8 B), the four corner lon/lat (64 B), the four
faces of the bracket pair (4 x 2 x field bytes) and their widths (32 B); in
3-D also two interfaces of w (2 x 2 x field bytes), the cell's area, bottom
thickness and interfaces (32 B) and the four faces' partial levels (48 B); the
step converts depth to level and back in the start and end cells (2 x 28 B).
"""
from __future__ import annotations

import numpy as np

SITES = {"euler": 2, "rk2": 3, "rk4": 5}
STAGES = {"euler": 1, "rk2": 2, "rk4": 4}


def mesh_stats(mesh) -> dict:
    en = np.asarray(mesh.elem_nodes)
    valid = en >= 0
    if en.shape[1] == 4:
        valid[:, 3] &= en[:, 3] != en[:, 0]
    return {"valence": float(np.mean(mesh.node_to_elems_count)), "nv": float(valid.sum(1).mean()),
            "max_v": int(en.shape[1])}


def bytes_per_particle_step(mesh, scheme: str, dims: int, field_bytes: int, *, kick: bool = False,
                            w_code: int = 0) -> dict:
    s = mesh_stats(mesh)
    state = 65 if dims == 2 else 89
    site = 4 + 4 * s["valence"] + 4 * s["max_v"] + 16 * s["nv"]
    n_sites = SITES[scheme] + (1 if kick else 0)
    if getattr(mesh, "_nemo_cgrid", False):
        stage = 16 + 8 + 64 + 4 * 2 * field_bytes + 32
        if dims == 3:
            stage += 2 * 2 * field_bytes + 32 + 48
            state += 2 * 28
        total = state + n_sites * site + STAGES[scheme] * stage
        return {"total": float(total), "state": state, "site": site, "n_sites": n_sites, "stage": stage,
                "n_stages": STAGES[scheme], **s}
    stage = s["nv"] * 2 * 2 * field_bytes
    w = 0.0
    if dims == 3:
        w = (2 * 2 * field_bytes) if w_code == 0 else s["nv"] * (8 + 2 * 2 * field_bytes)
        stage += w
    total = state + n_sites * site + STAGES[scheme] * stage
    return {"total": float(total), "state": state, "site": site, "n_sites": n_sites, "stage": stage,
            "n_stages": STAGES[scheme], **s}
