"""Build the native library ``kelp_b200/libkelpcuda.so`` in-tree.

The CUDA translation units are compiled for sm_100a only, with
``-fmad=false`` so no multiply-add is contracted into an FMA (the reference's
Numba kernels do not contract, and one rounding difference can flip a
nearest-node or containment decision).  The host routines are compiled with
``-ffp-contract=off`` for the same reason.  The counter RNG's exception
tables are built by scanning the whole Box-Muller input domain against this
host's C library (gen_rng_exceptions.cpp, a few minutes, only when missing
or stale) and linked into the library.  ``python -m kelp_b200.build``.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
ROOT = os.path.dirname(HERE)
BUILD = os.path.join(ROOT, "_build")
LIB = os.path.join(HERE, "libkelpcuda.so")

CU_SOURCES = ["kc_api.cu", "kc_plain_f64.cu", "kc_plain_f32.cu", "kc_mixed_f32.cu", "kc_mixed_f16.cu",
              "kc_cgrid_f64.cu", "kc_cgrid_f32.cu", "kc_cgrid_mixed.cu", "kc_sigma.cu", "kc_lsq.cu"]
CPP_SOURCES = ["kc_host.cpp", "kc_rngx.cpp"]
RNGX = os.path.join(BUILD, "kc_rng_exceptions.bin")
HEADERS = ["kc_geom.cuh", "kc_interp.cuh", "kc_step.cuh", "kc_beach.cuh", "kc_mixed.cuh", "kc_kernels.cuh", "kc_sigma.cuh",
           "kc_cgrid.cuh", "kc_sample.cuh",
           "kc_launch.h", "kc_host.h", "kc_crmath.cuh", "kc_crmath_tables.h"]

NVCC_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-lineinfo", "-std=c++17",
              "-fmad=false", "-Xcompiler", "-fPIC,-ffp-contract=off", "-Xptxas", "-v"]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found: the CUDA toolkit is required to build kelp_b200")


def _stale(out: str, deps) -> bool:
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(d) > t for d in deps)


def _rng_tables(force: bool):
    """Start the whole-domain scan of the Box-Muller inputs that writes the
    RNG's exception tables (gen_rng_exceptions.cpp), unless its output is
    current; returns the running process or None."""
    src = os.path.join(CSRC, "gen_rng_exceptions.cpp")
    deps = [src, os.path.join(CSRC, "kc_crmath.cuh"), os.path.join(CSRC, "kc_crmath_tables.h")]
    if not (force or _stale(RNGX, deps)):
        return None
    exe = os.path.join(BUILD, "gen_rng_exceptions")
    subprocess.run(["g++", "-O2", "-mfma", "-ffp-contract=off", "-std=c++17", "-pthread", f"-I{CSRC}", src, "-o", exe],
                   check=True)
    out = open(os.path.join(BUILD, "rng_domain.json"), "w")
    return subprocess.Popen([exe, RNGX + ".tmp"], stdout=out, stderr=subprocess.PIPE, text=True)


def _rng_tables_done(p) -> None:
    if p is None:
        return
    _, err = p.communicate()
    if p.returncode != 0:
        raise RuntimeError(f"the RNG exception scan failed:\n{err}")
    os.replace(RNGX + ".tmp", RNGX)
    import json
    got = json.load(open(os.path.join(BUILD, "rng_domain.json")))
    want = json.load(open(os.path.join(ROOT, "tests", "golden", "rng_domain.json")))
    if any(got[k] != want[k] for k in want if k.startswith("digest_")):
        print(f"warning: this host's C library ({got['libc']}) rounds log / sin / cos differently from the one "
              f"the fixtures were made with ({want['libc']}): the plain form's draws follow this host's",
              file=sys.stderr)


def build(verbose: bool = False, force: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    scan = _rng_tables(force)
    nvcc = _nvcc()
    hdrs = [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(ROOT, "include", "kelp_cuda.h")]
    objs = []
    jobs = []
    for src in CU_SOURCES:   # the translation units compile in parallel
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src + ".o")
        if force or _stale(o, [s] + hdrs):
            cmd = [nvcc, *NVCC_FLAGS, "-c", s, "-o", o]
            jobs.append((src, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True)))
        objs.append(o)
    for src, p in jobs:
        _, err = p.communicate()
        if p.returncode != 0:
            raise RuntimeError(f"nvcc failed for {src}:\n{err}")
        with open(os.path.join(BUILD, src + ".ptxas.txt"), "w") as fh:
            fh.write(err)
        if verbose:
            print(err)
    _rng_tables_done(scan)
    for src in CPP_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src + ".o")
        if force or _stale(o, [s, RNGX] + hdrs):
            cmd = ["g++", "-O2", "-ffp-contract=off", "-fno-fast-math", "-fPIC", "-std=c++17",
                   f'-DKC_RNGX_PATH="{RNGX}"', "-c", s, "-o", o]
            subprocess.run(cmd, check=True)
        objs.append(o)
    if force or _stale(LIB, objs):
        cmd = [nvcc, "-shared", "-gencode", "arch=compute_100a,code=sm_100a", *objs, "-o", LIB]
        subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    build(verbose="-v" in sys.argv, force="-f" in sys.argv)
    print(LIB)
