"""Correctly rounded exp for float64 arrays -- TEST INFRASTRUCTURE ONLY.

The ETD2 phi functions of the reference evaluate ``(exp(w) - 1) / w`` down to
``|w| = 1e-6``; there one ulp of ``exp`` moves ``phi1`` by ~1e-10 relative, so
the reference's own result depends on which ``exp`` the host's numpy uses
(numpy's AVX-512 ``exp`` is not correctly rounded; glibc's is in nearly all
cases).  To compare the CUDA path with the oracle at the 1e-10 level, both
can use the same correctly rounded ``exp``: this module is the numpy form of
the device routine ``cr_exp`` in ``prince_b200/csrc/prince_b200.cu`` -- the
same double-double algorithm, operation by operation, so both give the same
bits.

Method (double-double arithmetic after Dekker and Knuth, as in the QD
library of Hida, Li and Bailey): ``x = k ln2 + r`` with ``k = rint(x/ln2)``
and ``r`` in double-double, ``s = r / 2^10``, ``exp(s) - 1`` by a degree-9
Taylor polynomial in double-double, ten squarings in ``expm1`` form
``E <- 2E + E^2``, then ``(1 + E) * 2^k`` rounded once to double.  The
double-double result carries ~100 correct bits, so the final rounding is the
correctly rounded value except for inputs within ~2^-100 of a rounding
boundary.
"""

from __future__ import annotations

import numpy as np

LN2_HI = float.fromhex("0x1.62e42fefa39efp-1")
LN2_LO = float.fromhex("0x1.abc9e3b39803fp-56")
INV_LN2 = 1.4426950408889634
# 1/n! as double-double (hi, lo), n = 1..9
COEF = [
    (1.0, 0.0),
    (0.5, 0.0),
    (float.fromhex("0x1.5555555555555p-3"), float.fromhex("0x1.5555555555555p-57")),
    (float.fromhex("0x1.5555555555555p-5"), float.fromhex("0x1.5555555555555p-59")),
    (float.fromhex("0x1.1111111111111p-7"), float.fromhex("0x1.1111111111111p-63")),
    (float.fromhex("0x1.6c16c16c16c17p-10"), float.fromhex("-0x1.f49f49f49f49fp-65")),
    (float.fromhex("0x1.a01a01a01a01ap-13"), float.fromhex("0x1.a01a01a01a01ap-73")),
    (float.fromhex("0x1.a01a01a01a01ap-16"), float.fromhex("0x1.a01a01a01a01ap-76")),
    (float.fromhex("0x1.71de3a556c734p-19"), float.fromhex("-0x1.c154f8ddc6c00p-73")),
]
_SPLIT = 134217729.0  # 2^27 + 1


def _two_sum(a, b):
    s = a + b
    bb = s - a
    return s, (a - (s - bb)) + (b - bb)


def _quick(a, b):
    s = a + b
    return s, b - (s - a)


def _split(a):
    t = _SPLIT * a
    hi = t - (t - a)
    return hi, a - hi


def _two_prod(a, b):
    p = a * b
    ah, al = _split(a)
    bh, bl = _split(b)
    return p, ((ah * bh - p) + ah * bl + al * bh) + al * bl


def _dd_add(ah, al, bh, bl):
    s, e = _two_sum(ah, bh)
    t, f = _two_sum(al, bl)
    e = e + t
    s, e = _quick(s, e)
    e = e + f
    return _quick(s, e)


def _dd_mul(ah, al, bh, bl):
    p, e = _two_prod(ah, bh)
    e = e + (ah * bl + al * bh)
    return _quick(p, e)


def exp(x):
    """Correctly rounded exp of a float64 array (or scalar)."""
    x = np.asarray(x, dtype=np.float64)
    with np.errstate(over="ignore", invalid="ignore"):
        big = x > 709.782712893384
        tiny = x < -745.1332191019412
        xs = np.where(big | tiny | ~np.isfinite(x), 0.0, x)
        k = np.rint(xs * INV_LN2)
        ph, pl = _two_prod(k, LN2_HI)
        rh, rl = _two_sum(xs, -ph)
        rh, rl = _dd_add(rh, rl, -pl, np.zeros_like(pl))
        rh, rl = _dd_add(rh, rl, -(k * LN2_LO), np.zeros_like(pl))
        sh, sl = rh * 0.0009765625, rl * 0.0009765625
        th, tl = np.full_like(sh, COEF[8][0]), np.full_like(sh, COEF[8][1])
        for ch, cl in COEF[7::-1]:
            th, tl = _dd_mul(th, tl, sh, sl)
            th, tl = _dd_add(th, tl, np.full_like(sh, ch), np.full_like(sh, cl))
        eh, el = _dd_mul(th, tl, sh, sl)
        for _ in range(10):
            qh, ql = _dd_mul(eh, el, eh, el)
            eh, el = _dd_add(eh * 2.0, el * 2.0, qh, ql)
        vh, vl = _dd_add(eh, el, np.ones_like(eh), np.zeros_like(eh))
        v = np.ldexp(vh + vl, k.astype(np.int64))
        v = np.where(big, np.inf, v)
        v = np.where(tiny, 0.0, v)
        v = np.where(np.isnan(x), np.nan, v)
        v = np.where(x == np.inf, np.inf, v)
        v = np.where(x == -np.inf, 0.0, v)
    return v
