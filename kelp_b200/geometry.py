"""Geometry constants shared by the host code and (as literals) the CUDA kernels.

Values follow KELP's ``src/kelp/core/geometry.py:28-31``: the nautical-mile
metric of the tracker (111120 m per degree of latitude), the standard Earth
radius used by the local element projections, and the degree/radian factors.
"""
import numpy as np

METERS_PER_DEG_LAT = 111120.0
R_EARTH_STANDARD = 6_371_000.0
DEG2RAD = np.pi / 180.0
RAD2DEG = 180.0 / np.pi


def wrap_lon(lon):
    """Longitude folded into [-180, 180) with Python/numpy ``%`` semantics
    (``geometry.py:39-52``)."""
    return ((np.asarray(lon, dtype=np.float64) + 180.0) % 360.0) - 180.0
