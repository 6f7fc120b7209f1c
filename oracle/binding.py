"""ORACLE — test infrastructure only.  ctypes binding to liboracle.so (the
CPU restatement of CUDALucas's IBDWT step in oracle/ibdwt_oracle.c)."""
import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_lib = None


def lib():
    global _lib
    if _lib is None:
        path = os.path.join(_HERE, "liboracle.so")
        if not os.path.exists(path):
            raise RuntimeError("oracle not built: run `make -C oracle`")
        L = ctypes.CDLL(path)
        vp, i, f = ctypes.c_void_p, ctypes.c_int, ctypes.c_float
        ip = ctypes.POINTER(ctypes.c_int)
        up = ctypes.POINTER(ctypes.c_uint)
        L.oracle_create.restype = vp
        L.oracle_create.argtypes = [i, i, i]
        L.oracle_destroy.argtypes = [vp]
        L.oracle_init.argtypes = [vp, ip, i]
        L.oracle_step.restype = f
        L.oracle_step.argtypes = [vp, i, i]
        L.oracle_square.restype = f
        L.oracle_square.argtypes = [vp, i]
        L.oracle_digits.argtypes = [vp, ip]
        L.oracle_offset.restype = i
        L.oracle_offset.argtypes = [vp]
        L.oracle_find_residue.restype = ctypes.c_uint64
        L.oracle_find_residue.argtypes = [ip, i, i, i]
        L.oracle_standardize_digits.restype = i
        L.oracle_standardize_digits.argtypes = [ip, i, i]
        L.oracle_pack_bits.argtypes = [ip, up, i, i]
        L.oracle_unpack_bits.argtypes = [ip, up, i, i]
        L.oracle_balance_digits.argtypes = [ip, i, i]
        L.oracle_checkpoint_checksum.restype = ctypes.c_uint
        L.oracle_checkpoint_checksum.argtypes = [ctypes.c_char_p, i]
        L.oracle_ch_sum.restype = ctypes.c_uint
        L.oracle_ch_sum.argtypes = [up, i]
        L.oracle_set_threads.restype = i
        L.oracle_set_threads.argtypes = [i]
        _lib = L
    return _lib


def _ip(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_int))


def _up(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_uint))


def set_threads(t):
    """Host threads of the oracle's parallel loops; returns the count in effect."""
    return lib().oracle_set_threads(int(t))


class Oracle:
    """One LL test on the CPU, following CUDALucas's lucas_square."""

    def __init__(self, q, n, bigcarry=True):
        self.q, self.n = q, n
        self.h = lib().oracle_create(q, n, 1 if bigcarry else 0)
        if not self.h:
            raise ValueError("oracle_create failed (q=%d, n=%d)" % (q, n))

    def __del__(self):
        if getattr(self, "h", None):
            lib().oracle_destroy(self.h)
            self.h = None

    def start(self, offset=0, digits=None):
        d = None if digits is None else _ip(np.ascontiguousarray(digits, dtype=np.int32))
        lib().oracle_init(self.h, d, int(offset))

    def step(self, iters, report=True):
        return lib().oracle_step(self.h, int(iters), 1 if report else 0)

    def digits(self):
        out = np.zeros(self.n, dtype=np.int32)
        lib().oracle_digits(self.h, _ip(out))
        return out

    @property
    def offset(self):
        return lib().oracle_offset(self.h)

    def res64(self):
        d = self.digits()
        return lib().oracle_find_residue(_ip(d), self.q, self.n, self.offset)


def find_residue(digits, q, n, offset):
    d = np.ascontiguousarray(digits, dtype=np.int32)
    return lib().oracle_find_residue(_ip(d), q, n, offset)


def standardize_digits(digits, q, n):
    d = np.array(digits, dtype=np.int32)
    z = lib().oracle_standardize_digits(_ip(d), q, n)
    return d, z


def pack_bits(digits, q, n):
    d = np.ascontiguousarray(digits, dtype=np.int32)
    out = np.zeros((q + 31) // 32 + 1, dtype=np.uint32)
    lib().oracle_pack_bits(_ip(d), _up(out), q, n)
    return out[: (q + 31) // 32]


def unpack_bits(packed, q, n):
    p = np.zeros((q + 31) // 32 + 2, dtype=np.uint32)
    p[: len(packed)] = packed
    out = np.zeros(n, dtype=np.int32)
    lib().oracle_unpack_bits(_ip(out), _up(p), q, n)
    return out


def balance_digits(digits, q, n):
    d = np.array(digits, dtype=np.int32)
    lib().oracle_balance_digits(_ip(d), q, n)
    return d


def checkpoint_checksum(buf):
    b = bytes(buf)
    return lib().oracle_checkpoint_checksum(b, len(b))
