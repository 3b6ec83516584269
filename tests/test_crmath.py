"""The correctly rounded log / sin / cos of the RNG (kelp_b200/csrc/kc_crmath.cuh)
and the Box-Muller exception tables, on the CPU.

* The header is compiled for the host (the same source and operation order as
  the device build) and checked against 200-bit mpmath: the results must be
  the correctly rounded doubles.
* The exception tables (kc_rng_exceptions.bin) are checked against the host C
  library, which the reference's Numba kernels call: at listed inputs the
  library value is the correctly rounded one moved by the recorded bit, at
  other inputs they are equal.
* The reference-generated digests of 4 x 2^20 draws (golden_rng_1m.json) are
  reproduced by the oracle (C library arithmetic), which pins the fixture and
  its digest function.
"""
import ctypes as C
import json
import os
import subprocess
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(ROOT, "kelp_b200", "csrc")
INV, HALF, TWO_PI = 1.0 / 4294967296.0, 0.5 / 4294967296.0, 2.0 * 3.141592653589793

mp = pytest.importorskip("mpmath")

SHIM = r"""
#include "kc_crmath.cuh"
extern "C" double cr_log(double x) { return kc::cr::log_cr(x); }
extern "C" void cr_sincos(double x, double* s, double* c) { kc::cr::sincos_cr(x, s, c); }
"""


@pytest.fixture(scope="module")
def cr(tmp_path_factory):
    d = tmp_path_factory.mktemp("crmath")
    src = d / "shim.cpp"
    src.write_text(SHIM)
    so = d / "libcrshim.so"
    subprocess.run(["g++", "-O2", "-ffp-contract=off", "-fno-fast-math", "-fPIC", "-shared", "-std=c++17",
                    f"-I{CSRC}", str(src), "-o", str(so)], check=True)
    L = C.CDLL(str(so))
    L.cr_log.restype = C.c_double
    L.cr_log.argtypes = [C.c_double]
    L.cr_sincos.argtypes = [C.c_double, C.POINTER(C.c_double), C.POINTER(C.c_double)]
    return L


@pytest.fixture(scope="module")
def libm():
    L = C.CDLL("libm.so.6")
    for f in ("log", "sin", "cos"):
        getattr(L, f).restype = C.c_double
        getattr(L, f).argtypes = [C.c_double]
    return L


def _sincos(cr, x):
    s, c = C.c_double(), C.c_double()
    cr.cr_sincos(x, C.byref(s), C.byref(c))
    return s.value, c.value


def test_log_correctly_rounded(cr):
    mp.mp.prec = 200
    rng = np.random.default_rng(11)
    xs = list(rng.uniform(0, 1, 3000)) + list((rng.integers(0, 2**32, 3000) + 0.5) * INV)
    xs += list(np.exp(rng.uniform(-700, 700, 2000)))
    xs += [1.0 - k * 2.0**-53 for k in range(1, 50)] + [1.0 + k * 2.0**-52 for k in range(1, 50)]
    xs += [HALF, 1.0 - HALF, 0.5, 2.0, 0.6875, 1.375, 1e-300, 1e300]
    for x in xs:
        assert cr.cr_log(float(x)) == float(mp.log(mp.mpf(float(x)))), x


def test_sincos_correctly_rounded(cr):
    mp.mp.prec = 200
    rng = np.random.default_rng(12)
    xs = list(TWO_PI * ((rng.integers(0, 2**32, 3000) + 0.5) * INV)) + list(rng.uniform(-20, 20, 3000))
    # the doubles nearest multiples of pi/2 and pi/4 (the hardest reductions)
    for k in range(-12, 13):
        v = float(mp.pi * k / 4)
        xs += [v, np.nextafter(v, np.inf), np.nextafter(v, -np.inf)]
    xs += [TWO_PI * 0.25, TWO_PI * 0.5, TWO_PI * 0.75, 1e-10, -1e-10, 0.0, -0.0, 1e5]
    for x in xs:
        s, c = _sincos(cr, float(x))
        assert s == float(mp.sin(mp.mpf(float(x)))), x
        assert c == float(mp.cos(mp.mpf(float(x)))), x


def _tables():
    """(keys, codes) of tables a and b from the build's table file."""
    path = os.path.join(ROOT, "_build", "kc_rng_exceptions.bin")
    assert os.path.exists(path), "build first: python -m kelp_b200.build writes the RNG tables"
    raw = np.fromfile(path, np.uint8)
    magic, ver, na, nb, bits = raw[:20].view(np.uint32)
    assert magic == 0x5852434B and ver == 2 and bits == 20
    nof = (1 << 20) + 1
    o = 20
    out = []
    for n in (na, nb):
        off = raw[o:o + 4 * nof].view(np.uint32).astype(np.int64); o += 4 * nof
        ent = raw[o:o + 2 * n].view(np.uint16).astype(np.int64); o += 2 * n
        assert off[0] == 0 and off[-1] == n and np.all(np.diff(off) >= 0)
        bucket = np.repeat(np.arange(1 << 20, dtype=np.int64), np.diff(off))
        keys = (bucket << 12) | (ent >> 4)
        out += [keys, ent & 15]
    assert o == raw.size
    return out


def _bump(v, code):
    b = np.array([v]).view(np.int64)[0]
    return float(np.array([b + (1 if code == 1 else -1)], np.int64).view(np.float64)[0])


def test_exception_tables_match_the_c_library(cr, libm):
    ka, ca, kb, cb = _tables()
    assert np.all(np.diff(ka.astype(np.int64)) > 0) and np.all(np.diff(kb.astype(np.int64)) > 0)
    dom = json.load(open(os.path.join(HERE, "golden", "rng_domain.json")))
    assert dom["exceptions_r"] == ka.size and dom["exceptions_trig"] == kb.size and dom["ambiguous"] == 0
    rng = np.random.default_rng(13)
    for idx in rng.choice(ka.size, min(3000, ka.size), replace=False):
        u = float(ka[idx]) * INV + HALF
        r_lib = np.sqrt(-2.0 * libm.log(u))
        r_cr = np.sqrt(-2.0 * cr.cr_log(u))
        assert r_lib == _bump(r_cr, int(ca[idx]))
    for idx in rng.choice(kb.size, min(3000, kb.size), replace=False):
        th = TWO_PI * (float(kb[idx]) * INV + HALF)
        s_cr, c_cr = _sincos(cr, th)
        code = int(cb[idx])
        want_c = c_cr if not code & 3 else _bump(c_cr, code & 3)
        want_s = s_cr if not code >> 2 else _bump(s_cr, code >> 2)
        assert libm.cos(th) == want_c and libm.sin(th) == want_s
    # indices off the tables: the library equals the correctly rounded values
    sa, sb = set(ka.tolist()), set(kb.tolist())
    for j in rng.integers(0, 2**32, 20000):
        u = float(j) * INV + HALF
        if int(j) not in sa:
            assert np.sqrt(-2.0 * libm.log(u)) == np.sqrt(-2.0 * cr.cr_log(u))
        if int(j) not in sb:
            s_cr, c_cr = _sincos(cr, TWO_PI * u)
            assert libm.sin(TWO_PI * u) == s_cr and libm.cos(TWO_PI * u) == c_cr


def test_reference_rng_digests_reproduced_by_oracle():
    sys.path.insert(0, os.path.join(HERE, "golden"))
    from rng_digest import digest
    from oracle import oracle as O
    sets = json.load(open(os.path.join(HERE, "golden", "golden_rng_1m.json")))["sets"]
    assert len(sets) == 4 and all(s["n"] == 1 << 20 for s in sets)
    for s in sets:
        g = O.normals(s["n"], int(s["seed"]), s["real_id"], s["step"], int(s["pid0"]), s["comp"])
        assert [format(d, "016x") for d in digest(g, chunk=s["chunk"])] == s["digests"]
