"""Bit-exact counter-RNG draws on the GPU (diffusion.py:180-249).

* golden_rng: 4000 reference pairs (both key components), equal bit for bit;
* golden_rng_1m: the reference's own _normal_pair over 4 x 2^20 keys, as
  per-chunk digests, equal;
* the whole Box-Muller domain: for every one of the 2^32 uniforms, the
  device's r = sqrt(-2 log u), cos(2 pi u) and sin(2 pi u) -- which fix every
  draw -- digest to the host C library's values (the reference's arithmetic,
  scanned by gen_rng_exceptions.cpp), and without the exception tables to the
  correctly rounded values.
"""
import json
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
pytestmark = pytest.mark.gpu


def test_cuda_rng_normals_equal_reference_golden():
    from kelp_b200.device import default_context
    d = np.load(os.path.join(HERE, "golden", "golden_rng.npz"))
    keys, want = d["keys"], d["normals"]
    ctx = default_context()
    got = np.empty_like(want)
    for i, k in enumerate(keys):
        seed, real_id, pid, step, comp = (int(x) for x in k)
        got[i] = ctx.rng_normals(1, seed, real_id, step, pid, comp)[0]
    mism = np.flatnonzero((got.view(np.uint64) != want.view(np.uint64)).any(axis=1))
    assert mism.size == 0, f"{mism.size} of {keys.shape[0]} pairs differ from the reference"


def test_cuda_rng_4m_reference_keys_digest():
    sys.path.insert(0, os.path.join(HERE, "golden"))
    from rng_digest import digest
    from kelp_b200.device import default_context
    ctx = default_context()
    sets = json.load(open(os.path.join(HERE, "golden", "golden_rng_1m.json")))["sets"]
    bad = 0
    for s in sets:
        g = ctx.rng_normals(s["n"], int(s["seed"]), s["real_id"], s["step"], int(s["pid0"]), s["comp"])
        assert [float.hex(float(v)) for v in g[0]] == s["first"]
        got = [format(d, "016x") for d in digest(g, chunk=s["chunk"])]
        bad += sum(a != b for a, b in zip(got, s["digests"]))
    assert bad == 0, f"{bad} chunks of {sum(len(s['digests']) for s in sets)} differ from the reference's draws"


def test_cuda_rng_whole_domain_digests():
    from kelp_b200.device import default_context
    ctx = default_context()
    dom = json.load(open(os.path.join(HERE, "golden", "rng_domain.json")))
    assert dom["domain"] == 2**32
    lib = ctx.rng_domain_digests(corrected=True)
    assert [format(v, "016x") for v in lib] == [dom["digest_r_lib"], dom["digest_cos_lib"], dom["digest_sin_lib"]]
    crd = ctx.rng_domain_digests(corrected=False)
    assert [format(v, "016x") for v in crd] == [dom["digest_r_cr"], dom["digest_cos_cr"], dom["digest_sin_cr"]]
