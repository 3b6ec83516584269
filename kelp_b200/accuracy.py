"""Accuracy of a numerical form against a float64 run: great-circle
separation of the same particles after the same steps, and the dispersion
(single-particle displacement variance) each run produces.

Separation uses the haversine distance on a sphere of radius 6371 km.  Only
particles ALIVE in both runs are compared; the count of status mismatches is
reported beside the statistics.
"""
from __future__ import annotations

import numpy as np

R_EARTH = 6371000.0
DEG2RAD = np.pi / 180.0


def great_circle_m(lon1, lat1, lon2, lat2) -> np.ndarray:
    """Haversine distance in metres between (lon1, lat1) and (lon2, lat2), degrees."""
    p1, p2 = np.asarray(lat1) * DEG2RAD, np.asarray(lat2) * DEG2RAD
    dl = (np.asarray(lon2) - np.asarray(lon1)) * DEG2RAD
    h = np.sin((p2 - p1) / 2) ** 2 + np.cos(p1) * np.cos(p2) * np.sin(dl / 2) ** 2
    return 2 * R_EARTH * np.arcsin(np.sqrt(np.clip(h, 0.0, 1.0)))


def separation_stats(ref: dict, test: dict, alive: int = 1) -> dict:
    """Median / p99 / max separation (m) of the particles ALIVE in both runs,
    with the number compared and the number whose status differs."""
    both = (np.asarray(ref["status"]) == alive) & (np.asarray(test["status"]) == alive)
    d = great_circle_m(ref["lon"][both], ref["lat"][both], test["lon"][both], test["lat"][both])
    out = {"compared": int(both.sum()),
           "status_mismatch": int((np.asarray(ref["status"]) != np.asarray(test["status"])).sum())}
    if d.size:
        out.update(median_m=float(np.median(d)), p99_m=float(np.percentile(d, 99)), max_m=float(d.max()))
        if "z" in ref and "z" in test and ref["z"] is not None and test["z"] is not None:
            dz = np.abs(np.asarray(ref["z"])[both] - np.asarray(test["z"])[both])
            out.update(z_median_m=float(np.median(dz)), z_p99_m=float(np.percentile(dz, 99)))
    return out


def dispersion_m2(lon0, lat0, state: dict, alive: int = 1) -> float:
    """Mean squared great-circle displacement (m^2) from the release
    positions of the particles still ALIVE: the single-particle dispersion."""
    ok = np.asarray(state["status"]) == alive
    d = great_circle_m(np.asarray(lon0)[ok], np.asarray(lat0)[ok], state["lon"][ok], state["lat"][ok])
    return float(np.mean(d * d)) if d.size else float("nan")
