"""ORACLE — test infrastructure only (tests/, the smoke check and bench.py's
cpu_baseline leg may use it; the product never does).

Exact Lucas-Lehmer arithmetic on big integers: s0 = 4, s <- s^2 - 2 mod 2^p-1
(the recurrence CUDALucas iterates in lucas_square, CUDALucas.cu:1869; its
self-test counts iterations j = 1..10000 from s0 = 4, CUDALucas.cu:2758).
Res64 is the low 64 bits of s (CUDALucas.cu:1491 find_residue removes the
shift first, so Res64 does not depend on the shift).

libgmp.so.10 is used through ctypes when present (only the runtime library is
installed, no headers); otherwise Python integers are used.
"""
import ctypes
import ctypes.util

_gmp = None


def _load_gmp():
    global _gmp
    if _gmp is not None:
        return _gmp or None
    for name in ("libgmp.so.10", ctypes.util.find_library("gmp")):
        if not name:
            continue
        try:
            g = ctypes.CDLL(name)
            break
        except OSError:
            g = None
    else:
        g = None
    if g is None:
        _gmp = False
        return None

    class mpz(ctypes.Structure):
        _fields_ = [("a", ctypes.c_int), ("s", ctypes.c_int), ("d", ctypes.c_void_p)]

    P = ctypes.POINTER(mpz)
    g.__gmpz_init.argtypes = [P]
    g.__gmpz_clear.argtypes = [P]
    g.__gmpz_set_ui.argtypes = [P, ctypes.c_ulong]
    g.__gmpz_mul.argtypes = [P, P, P]
    g.__gmpz_sub_ui.argtypes = [P, P, ctypes.c_ulong]
    g.__gmpz_add_ui.argtypes = [P, P, ctypes.c_ulong]
    g.__gmpz_tdiv_r_2exp.argtypes = [P, P, ctypes.c_ulong]
    g.__gmpz_tdiv_q_2exp.argtypes = [P, P, ctypes.c_ulong]
    g.__gmpz_add.argtypes = [P, P, P]
    g.__gmpz_sub.argtypes = [P, P, P]
    g.__gmpz_cmp.argtypes = [P, P]
    g.__gmpz_cmp_ui.argtypes = [P, ctypes.c_ulong]
    g.__gmpz_setbit.argtypes = [P, ctypes.c_ulong]
    g.__gmpz_getlimbn.argtypes = [P, ctypes.c_long]
    g.__gmpz_getlimbn.restype = ctypes.c_ulong
    g.__gmpz_sizeinbase.argtypes = [P, ctypes.c_int]
    g.__gmpz_sizeinbase.restype = ctypes.c_size_t
    g.__gmpz_export.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_size_t), ctypes.c_int,
                                ctypes.c_size_t, ctypes.c_int, ctypes.c_size_t, P]
    g.__gmpz_export.restype = ctypes.c_void_p
    g.mpz = mpz
    _gmp = g
    return g


def ll_state(p, iters, start=4):
    """Exact s_iters as a Python int (0 <= s < 2^p - 1)."""
    M = (1 << p) - 1
    g = _load_gmp()
    if g is None or p < 4096:
        s = start % M
        for _ in range(iters):
            s = (s * s - 2) % M
        return s
    s, t, h, Mz = g.mpz(), g.mpz(), g.mpz(), g.mpz()
    for x in (s, t, h, Mz):
        g.__gmpz_init(ctypes.byref(x))
    try:
        g.__gmpz_set_ui(s, start)
        g.__gmpz_setbit(Mz, p)
        g.__gmpz_sub_ui(Mz, Mz, 1)
        for _ in range(iters):
            g.__gmpz_mul(t, s, s)
            g.__gmpz_tdiv_q_2exp(h, t, p)
            g.__gmpz_tdiv_r_2exp(t, t, p)
            g.__gmpz_add(t, t, h)
            if g.__gmpz_cmp(t, Mz) >= 0:
                g.__gmpz_sub(t, t, Mz)
            if g.__gmpz_cmp_ui(t, 2) < 0:
                g.__gmpz_add(t, t, Mz)
            g.__gmpz_sub_ui(s, t, 2)
        nbytes = (g.__gmpz_sizeinbase(s, 2) + 7) // 8
        buf = ctypes.create_string_buffer(max(nbytes, 1))
        cnt = ctypes.c_size_t(0)
        g.__gmpz_export(buf, ctypes.byref(cnt), -1, 1, 0, 0, s)
        return int.from_bytes(buf.raw[: cnt.value], "little")
    finally:
        for x in (s, t, h, Mz):
            g.__gmpz_clear(ctypes.byref(x))


def res64(p, iters, start=4):
    """Low 64 bits of s_iters mod 2^p-1."""
    return ll_state(p, iters, start) & 0xFFFFFFFFFFFFFFFF


def is_mersenne_prime(p):
    """Full Lucas-Lehmer test (p odd prime)."""
    return ll_state(p, p - 2) == 0
