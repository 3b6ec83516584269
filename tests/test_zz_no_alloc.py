"""kc_find_nearest_noalloc: the nearest-node query for callers that must not
allocate device memory (cudaMalloc stalls the whole device and fails once a
host application has reserved the free memory for its own pool).  It stages
its queries in one fixed device array instead of a cudaMalloc'd buffer.

Called through the C ABI with ctypes, twice in a row on different query sets
(the second call reuses the array the first one left behind), against the
allocating kc_find_nearest; and a batch above the array's limit is rejected.
This file sorts last so that a run stopping at the first failure has run
every other test; it also passes alone in a fresh process.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MAX_POINTS = 65536


def _queries(seed, n):
    rng = np.random.default_rng(seed)
    return np.ascontiguousarray(rng.uniform(-180, 180, n)), np.ascontiguousarray(rng.uniform(-85, 85, n))


def test_noalloc_nearest_matches_allocating_entry_point():
    from kelp_b200 import _native as N
    from kelp_b200 import synthetic as S
    from kelp_b200.device import DeviceContext

    mesh = S.lattice_mesh(1.5, 80.0)
    ctx = DeviceContext(0)
    try:
        ctx.ensure_mesh(mesh)
        L = N.lib()
        for seed, n in ((1, 40000), (2, MAX_POINTS)):
            lon, lat = _queries(seed, n)
            want = np.empty(n, np.int32)
            got = np.full(n, -7, np.int32)
            N.check(ctx.handle, L.kc_find_nearest(ctx.handle, n, N.ptr(lon), N.ptr(lat), N.ptr(want)),
                    "kc_find_nearest")
            N.check(ctx.handle, L.kc_find_nearest_noalloc(ctx.handle, n, N.ptr(lon), N.ptr(lat), N.ptr(got)),
                    "kc_find_nearest_noalloc")
            np.testing.assert_array_equal(got, want)
            assert (got >= 0).all()
        lon, lat = _queries(3, MAX_POINTS + 1)
        out = np.empty(MAX_POINTS + 1, np.int32)
        rc = L.kc_find_nearest_noalloc(ctx.handle, MAX_POINTS + 1, N.ptr(lon), N.ptr(lat), N.ptr(out))
        assert rc == N.KC_ERR_ARG
        buf = C.create_string_buffer(512)
        L.kc_last_error(ctx.handle, buf, 512)
        assert b"exceed" in buf.value
    finally:
        ctx.close()
