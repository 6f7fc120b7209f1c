"""Generates tests/golden/large_res64.json: exact Res64 (oracle/exact.py, GMP)
after k iterations for the large single-exponent workloads:
  p = 57885161  (3200K words)   k = 1, 10, 100, 1000
  p = 332192831 (18432K words)  k = 1, 5, 20, 50
Run from the repository root: python tests/golden/make_large.py  (~15 min)"""
import json
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
from oracle.exact import _load_gmp  # noqa: E402
import ctypes  # noqa: E402


def run(p, ks):
    g = _load_gmp()
    s, t, h, Mz = g.mpz(), g.mpz(), g.mpz(), g.mpz()
    for x in (s, t, h, Mz):
        g.__gmpz_init(ctypes.byref(x))
    g.__gmpz_set_ui(s, 4)
    g.__gmpz_setbit(Mz, p)
    g.__gmpz_sub_ui(Mz, Mz, 1)
    out = []
    t0 = time.time()
    for k in range(1, max(ks) + 1):
        g.__gmpz_mul(t, s, s)
        g.__gmpz_tdiv_q_2exp(h, t, p)
        g.__gmpz_tdiv_r_2exp(t, t, p)
        g.__gmpz_add(t, t, h)
        if g.__gmpz_cmp(t, Mz) >= 0:
            g.__gmpz_sub(t, t, Mz)
        if g.__gmpz_cmp_ui(t, 2) < 0:
            g.__gmpz_add(t, t, Mz)
        g.__gmpz_sub_ui(s, t, 2)
        if k in ks:
            r = g.__gmpz_getlimbn(s, 0)
            out.append([p, k, "0x%016x" % r])
            print(p, k, "0x%016x" % r, "%.0fs" % (time.time() - t0), flush=True)
    return out


if __name__ == "__main__":
    entries = run(57885161, {1, 10, 100, 1000}) + run(332192831, {1, 5, 20, 50})
    with open(os.path.join(HERE, "large_res64.json"), "w") as f:
        json.dump({"generator": "oracle/exact.py GMP recurrence", "entries": entries}, f, indent=1)
