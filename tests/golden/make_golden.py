"""Generates the golden vectors under tests/golden/ (run: python tests/golden/make_golden.py).

QuickPIC-OpenSource ships no tests or reference outputs, so these vectors come
from independent implementations of what its routines compute:

* ``ranorm.npz`` -- the first draws of ranorm (source/part3d_lib77.f:1324-1383).
  Its double-precision arithmetic on (r1, r2) and (r4, r5) is a pair of
  multiplicative congruential generators on 62-bit integers,
      x <- (2**31 - 5)  * x  mod 2**62   (h1l = 65531, h1u = 32767)
      y <- (2**31 - 11) * y  mod 2**62   (h2l = 65525)
  with x = r1 * 2**31 + r2, y = r4 * 2**31 + r5, u = x / 2**62, followed by
  Box-Muller (sin first, cos cached for the next call).  This file evaluates
  that with exact Python integers, independently of the Fortran restatement.
* ``sincos.npz`` -- real sine (DST-I) and cosine (DCT-I) transforms of seeded
  lines computed with scipy.fft, the definitions the NR routines of
  source/fft2d_lib77.f:4791-5493 implement (checked in test_oracle_kat.py).
"""
import math
import os

import numpy as np
from scipy.fft import dct, dst

HERE = os.path.dirname(os.path.abspath(__file__))


def ranorm_draws(n):
    m62 = 1 << 62
    a1, a2 = (1 << 31) - 5, (1 << 31) - 11
    x = 885098780 * (1 << 31) + 1824280461
    y = 1396483093 * (1 << 31) + 55318673
    out = []
    cached = None
    while len(out) < n:
        if cached is not None:
            out.append(cached)
            cached = None
            continue
        x = (a1 * x) % m62
        temp = math.sqrt(-2.0 * math.log(x / m62))
        y = (a2 * y) % m62
        ang = 6.28318530717959 * (y / m62)
        out.append(temp * math.sin(ang))
        cached = temp * math.cos(ang)
    return np.array(out)


def main():
    np.savez(os.path.join(HERE, "ranorm.npz"), draws=ranorm_draws(256))
    rng = np.random.default_rng(20240611)
    lines, sin_out, cos_out, ns = [], [], [], []
    for ind in (4, 5, 7, 9):
        n = 1 << ind
        f = rng.standard_normal(n + 1)
        s = np.zeros(n + 1)
        s[1:n] = dst(f[1:n], type=1)
        c = dct(f, type=1)
        lines.append(np.pad(f, (0, 513 - (n + 1))))
        sin_out.append(np.pad(s, (0, 513 - (n + 1))))
        cos_out.append(np.pad(c, (0, 513 - (n + 1))))
        ns.append(ind)
    np.savez(os.path.join(HERE, "sincos.npz"), ind=np.array(ns), x=np.array(lines),
             sine=np.array(sin_out), cosine=np.array(cos_out))


if __name__ == "__main__":
    main()
