"""Write kc_crmath_tables.h: the constants of the correctly rounded log and
sin/cos in kc_crmath.cuh, evaluated at 300 bits with mpmath and split into
double-double pairs (hi = the nearest double, lo = the nearest double of the
remainder).  ``python kelp_b200/csrc/gen_crmath_tables.py``.

Tables:
  * log: 128 reciprocals c_i (10 significant bits) of the centres of the
    sub-intervals of the reduced argument m in [0.6875, 1.375) addressed by
    the top 7 mantissa bits of x, and -log(c_i) as double-double;
  * log1p series coefficients (-1)^k / (k + 1);
  * ln 2 in three parts (the first with 42 significant bits, so e * part is
    exact for any double exponent e);
  * pi/2 in three 53-bit parts (Cody-Waite reduction);
  * the Taylor coefficients (-1)^k / (2k+1)! and (-1)^k / (2k)!;
  * sin(j/64) and cos(j/64), j = 0..51, as double-double records (the fast
    path of sin / cos).
"""
from __future__ import annotations

import math
import os
from fractions import Fraction

import mpmath as mp

mp.mp.prec = 300
HERE = os.path.dirname(os.path.abspath(__file__))


def dd(v):
    """Double-double split of an mpf or Fraction."""
    if isinstance(v, Fraction):
        v = mp.mpf(v.numerator) / v.denominator
    elif not isinstance(v, mp.mpf):
        v = mp.mpf(v)
    hi = float(v)
    lo = float(v - mp.mpf(hi))
    return hi, lo


def trunc_bits(v, bits):
    """v rounded to a double with at most `bits` significant bits."""
    m, e = mp.frexp(v)
    scale = mp.mpf(2) ** bits
    return float(mp.nint(m * scale) / scale * mp.mpf(2) ** e)


def fmt(x: float) -> str:
    return float.hex(x) if x != 0.0 else "0x0p+0"


def main() -> None:
    lines = ["// Generated by gen_crmath_tables.py: constants of the correctly rounded",
             "// log and sin/cos (kc_crmath.cuh).  Do not edit by hand.",
             "#pragma once", ""]
    # log reduction table: index i = top 7 mantissa bits f of x in [1, 2);
    # i < 48: m = 1 + f in [1, 1.375), sub-interval [1 + i/128, 1 + (i+1)/128);
    # i >= 48: m = (1 + f) / 2 in [0.6875, 1), [(1 + i/128)/2, (1 + (i+1)/128)/2)
    inv, nlh, nll = [], [], []
    for i in range(128):
        lo = mp.mpf(1) + mp.mpf(i) / 128
        hi = mp.mpf(1) + mp.mpf(i + 1) / 128
        if i >= 48:
            lo, hi = lo / 2, hi / 2
        if i == 0 or i == 127:
            c = 1.0   # the sub-intervals next to 1: r = m - 1 exactly, log c = 0
        else:
            c = trunc_bits(2 / (lo + hi), 10)
        inv.append(c)
        h, l = dd(-mp.log(mp.mpf(c)))
        nlh.append(h)
        nll.append(l)

    def arr(name, vals):
        body = ", \\\n".join("    " + ", ".join(fmt(v) for v in vals[k:k + 4]) for k in range(0, len(vals), 4))
        return [f"#define {name} {{ \\", body + " }", ""]

    lines += arr("KC_CR_LOG_INV", inv)
    lines += arr("KC_CR_LOG_NLC_HI", nlh)
    lines += arr("KC_CR_LOG_NLC_LO", nll)

    # sin / cos fast path: sin(j/64), cos(j/64), j = 0..51 (|r| <= pi/4 + eps)
    tsh, tsl, tch, tcl = [], [], [], []
    for j in range(52):
        a = mp.mpf(j) / 64
        h, l = dd(mp.sin(a))
        tsh.append(h)
        tsl.append(l)
        h, l = dd(mp.cos(a))
        tch.append(h)
        tcl.append(l)
    # interleaved per j: sin hi, sin lo, cos hi, cos lo (one 32-byte record)
    lines += arr("KC_CR_TAB_SC", [v for j in range(52) for v in (tsh[j], tsl[j], tch[j], tcl[j])])

    ln2 = mp.log(2)
    ln2_1 = trunc_bits(ln2, 42)
    ln2_2 = float(ln2 - ln2_1)
    ln2_3 = float(ln2 - ln2_1 - mp.mpf(ln2_2))
    pio2 = mp.pi / 2
    p1 = float(pio2)
    p2 = float(pio2 - p1)
    p3 = float(pio2 - p1 - mp.mpf(p2))
    consts = [("kCrLn2_1", ln2_1), ("kCrLn2_2", ln2_2), ("kCrLn2_3", ln2_3),
              ("kCrPio2_1", p1), ("kCrPio2_2", p2), ("kCrPio2_3", p3),
              ("kCrTwoOverPi", float(2 / mp.pi))]
    for name, v in consts:
        lines.append(f"constexpr double {name} = {fmt(v)};")
    lines.append("")

    # log1p(r) = r * sum_k (-1)^k r^k / (k+1), k = 0..15
    l1h, l1l = [], []
    for k in range(16):
        h, l = dd(Fraction((-1) ** k, k + 1))
        l1h.append(h)
        l1l.append(l)
    # sin(r) = r * sum_k (-1)^k t^k / (2k+1)!, cos(r) = sum_k (-1)^k t^k / (2k)!, t = r^2, k = 0..14
    sh, sl, ch, cl = [], [], [], []
    for k in range(15):
        h, l = dd(Fraction((-1) ** k, math.factorial(2 * k + 1)))
        sh.append(h)
        sl.append(l)
        h, l = dd(Fraction((-1) ** k, math.factorial(2 * k)))
        ch.append(h)
        cl.append(l)
    for name, vals in (("KC_CR_L1P_HI", l1h), ("KC_CR_L1P_LO", l1l), ("KC_CR_SIN_HI", sh), ("KC_CR_SIN_LO", sl),
                       ("KC_CR_COS_HI", ch), ("KC_CR_COS_LO", cl)):
        body = ", ".join(fmt(v) for v in vals)
        lines.append(f"#define {name} {{{body}}}")
    lines.append("")
    with open(os.path.join(HERE, "kc_crmath_tables.h"), "w") as fh:
        fh.write("\n".join(lines))


if __name__ == "__main__":
    main()
