"""Order-free digests of counter-RNG normal pairs, shared by the fixture
generator (make_golden.py, which runs the reference) and the GPU test.

digest(g, base) for an (n, 2) float64 array, per chunk of CHUNK rows: the sum
over rows i of mix(mix(base + i) ^ bits(g1)) + mix(mix(base + i) ^ bits(g2)
^ 1) mod 2^64, mix = one SplitMix64 round.  Equal digests mean equal bits
(up to a 2^-64 chance), and a differing chunk locates a difference."""
from __future__ import annotations

import numpy as np

CHUNK = 1 << 14


def _mix(x):
    x = x + np.uint64(0x9E3779B97F4A7C15)
    x = (x ^ (x >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
    x = (x ^ (x >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
    return x ^ (x >> np.uint64(31))


def digest(g: np.ndarray, base: int = 0, chunk: int = CHUNK) -> list:
    g = np.ascontiguousarray(g, dtype=np.float64)
    with np.errstate(over="ignore"):
        i = _mix(np.arange(base, base + g.shape[0], dtype=np.uint64))
        b = g.view(np.uint64)
        t = _mix(i ^ b[:, 0]) + _mix(i ^ b[:, 1] ^ np.uint64(1))
        return [int(c.sum(dtype=np.uint64)) for c in t.reshape(-1, chunk)]
