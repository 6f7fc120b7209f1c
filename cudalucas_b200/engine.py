"""Python host mirror of the engine's C ABI (include/llb200.h).

`LLContext` is one Lucas-Lehmer test on one GPU: the object form of
CUDALucas's init_lucas / lucas_square / close_lucas (CUDALucas.cu:1344,
:1869, :1415).  Every call goes straight to libllb200.so; there is no CPU
path, and failures raise `LLError` carrying the C status code."""
import ctypes

import numpy as np

from . import native
from .native import LL_ERRCHK, LL_REPORT, Tuning  # noqa: F401


class LLError(RuntimeError):
    def __init__(self, status, msg=""):
        self.status = status
        text = native.lib().ll_status_string(status).decode()
        super().__init__("%s (status %d)%s" % (text, status, ": " + msg if msg else ""))


def _i32p(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))


def _u32p(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32))


class LLContext:
    def __init__(self, q, n, device=0, tuning=None):
        L = native.lib()
        self._h = ctypes.c_void_p()
        t = None
        if tuning:
            t = Tuning()
            for k, v in tuning.items():
                setattr(t, k, v)
            t = ctypes.byref(t)
        rc = L.ll_create(int(device), int(q), int(n), t, ctypes.byref(self._h))
        if rc:
            raise LLError(rc, "ll_create(q=%d, n=%d)" % (q, n))
        self.q, self.n = int(q), int(n)

    def close(self):
        if self._h:
            native.lib().ll_destroy(self._h)
            self._h = ctypes.c_void_p()

    __del__ = close

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _check(self, rc, what):
        if rc:
            msg = native.lib().ll_last_error(self._h)
            raise LLError(rc, "%s: %s" % (what, msg.decode() if msg else ""))

    def start(self, offset=0):
        self._check(native.lib().ll_start(self._h, int(offset)), "ll_start")

    def load_digits(self, digits, offset):
        d = np.ascontiguousarray(digits, dtype=np.int32)
        assert d.size == self.n
        self._check(native.lib().ll_load_digits(self._h, _i32p(d), int(offset)), "ll_load_digits")

    def step(self, iters, report=False, errchk=False, wait=True):
        """iters LL iterations; returns the max roundoff error when a flag
        asks for it and wait is true.  wait=False only enqueues (LL_ASYNC):
        with report=True the digits are readable once the work finishes."""
        e = ctypes.c_float(0)
        flags = (LL_REPORT if report else 0) | (LL_ERRCHK if errchk else 0)
        if not wait:
            flags |= native.LL_ASYNC
        self._check(native.lib().ll_step(self._h, int(iters), flags, ctypes.byref(e)), "ll_step")
        return float(e.value) if flags and wait else None

    def read_digits(self):
        d = np.zeros(self.n, dtype=np.int32)
        off = ctypes.c_uint32(0)
        self._check(native.lib().ll_read_digits(self._h, _i32p(d), ctypes.byref(off)), "ll_read_digits")
        return d, int(off.value)

    def res64(self):
        r = ctypes.c_uint64(0)
        self._check(native.lib().ll_res64(self._h, ctypes.byref(r)), "ll_res64")
        return int(r.value)

    def sync(self):
        self._check(native.lib().ll_sync(self._h), "ll_sync")

    def busy(self):
        r = native.lib().ll_busy(self._h)
        if r < 0:
            raise LLError(native.LL_ERR_CUDA, "ll_busy")
        return bool(r)

    def device_checkpoint(self):
        """Keeps a device copy of the digits of the last report step."""
        self._check(native.lib().ll_device_checkpoint(self._h), "ll_device_checkpoint")

    def device_restore(self):
        """Reloads the state from the device checkpoint; returns its offset."""
        off = ctypes.c_uint32(0)
        self._check(native.lib().ll_device_restore(self._h, ctypes.byref(off)), "ll_device_restore")
        return int(off.value)

    def debug_launch(self, which):
        self._check(native.lib().ll_debug_launch(self._h, int(which)), "ll_debug_launch")

    def inject_failure(self, count=1):
        native.lib().ll_debug_inject_failure(self._h, int(count))

    @property
    def offset(self):
        return int(native.lib().ll_offset(self._h))

    @property
    def stream(self):
        return native.lib().ll_stream(self._h)

    @property
    def shape(self):
        v = [ctypes.c_int32() for _ in range(5)]
        native.lib().ll_shape(self._h, *[ctypes.byref(x) for x in v])
        d = dict(zip(("W", "H", "G", "threads_wide", "threads_tall"), [x.value for x in v]))
        k = native.lib().ll_kernel_kinds(self._h)
        d["wide_specialised"], d["tall_specialised"], d["fused"] = bool(k & 1), bool(k & 2), bool(k & 4)
        d["cluster"] = bool(k & 8)
        return d


class LLBatch:
    """Many exponents advancing together (ll_batch_* in include/llb200.h)."""

    def __init__(self, qs, ns, device=0, graph_iters=10, by_length=True):
        L = native.lib()
        self.qs = [int(x) for x in qs]
        self.ns = [int(x) for x in ns]
        q = np.ascontiguousarray(self.qs, dtype=np.uint32)
        n = np.ascontiguousarray(self.ns, dtype=np.uint32)
        self._h = ctypes.c_void_p()
        rc = L.ll_batch_create(int(device), len(self.qs), _u32p(q), _u32p(n), int(graph_iters),
                               ctypes.byref(self._h))
        if rc:
            raise LLError(rc, "ll_batch_create")
        self._keep = (q, n)
        L.ll_batch_group_by_length(self._h, 1 if by_length else 0)

    @property
    def classes(self):
        """Number of length classes (members launched together per pass)."""
        return int(native.lib().ll_batch_classes(self._h))

    def close(self):
        if self._h:
            native.lib().ll_batch_destroy(self._h)
            self._h = ctypes.c_void_p()

    __del__ = close

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __len__(self):
        return len(self.qs)

    def start(self, offsets=None):
        o = np.ascontiguousarray(offsets if offsets is not None else [0] * len(self), dtype=np.uint32)
        rc = native.lib().ll_batch_start(self._h, _u32p(o))
        if rc:
            raise LLError(rc, "ll_batch_start")

    def step(self, iters, report=False, errchk=False):
        flags = (LL_REPORT if report else 0) | (LL_ERRCHK if errchk else 0)
        errs = np.zeros(len(self), dtype=np.float32)
        rc = native.lib().ll_batch_step(self._h, int(iters), flags,
                                        errs.ctypes.data_as(ctypes.POINTER(ctypes.c_float)))
        if rc:
            raise LLError(rc, "ll_batch_step")
        return errs if flags else None

    @property
    def stream(self):
        return native.lib().ll_batch_stream(self._h)

    def sync(self):
        rc = native.lib().ll_batch_sync(self._h)
        if rc:
            raise LLError(rc, "ll_batch_sync")

    def res64(self):
        out = np.zeros(len(self), dtype=np.uint64)
        rc = native.lib().ll_batch_res64(self._h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64)))
        if rc:
            raise LLError(rc, "ll_batch_res64")
        return [int(x) for x in out]


# ---- host helpers (no GPU) -------------------------------------------------
def digits_res64(digits, q, n, offset):
    d = np.ascontiguousarray(digits, dtype=np.int32)
    return int(native.lib().ll_digits_res64(_i32p(d), q, n, offset))


def standardize(digits, q, n):
    d = np.array(digits, dtype=np.int32)
    z = native.lib().ll_digits_standardize(_i32p(d), q, n)
    return d, bool(z)


def pack_bits(digits, q, n):
    d = np.ascontiguousarray(digits, dtype=np.int32)
    out = np.zeros((q + 31) // 32, dtype=np.uint32)
    native.lib().ll_pack_bits(_i32p(d), _u32p(out), q, n)
    return out


def unpack_bits(packed, q, n):
    p = np.ascontiguousarray(packed, dtype=np.uint32)
    out = np.zeros(n, dtype=np.int32)
    native.lib().ll_unpack_bits(_u32p(p), _i32p(out), q, n)
    return out


def balance_digits(digits, q, n):
    d = np.array(digits, dtype=np.int32)
    native.lib().ll_balance_digits(_i32p(d), q, n)
    return d


def checkpoint_checksum(buf):
    b = bytes(buf)
    return int(native.lib().ll_checkpoint_checksum(b, len(b)))


def additive_checksum(words):
    w = np.ascontiguousarray(words, dtype=np.uint32)
    return int(native.lib().ll_additive_checksum(_u32p(w), w.size))


def fft_bounds(q):
    lb, ub = ctypes.c_uint32(), ctypes.c_uint32()
    native.lib().ll_fft_bounds(q, ctypes.byref(lb), ctypes.byref(ub))
    return lb.value, ub.value


def choose_fft_length(q, want=0):
    return int(native.lib().ll_choose_fft_length(q, want))


def fft_table():
    cnt = native.lib().ll_fft_table(None, 0)
    out = np.zeros(cnt, dtype=np.uint32)
    native.lib().ll_fft_table(_u32p(out), cnt)
    return [int(x) for x in out]


def length_supported(n):
    return bool(native.lib().ll_length_supported(n))


def fft_table_merge(measured):
    """Installs the built-in table merged with measured lengths (ascending,
    in words), as init_ffts does with `<gpu> fft.txt`; [] restores the
    built-in table.  Returns the new table size."""
    m = np.ascontiguousarray(sorted(int(x) for x in measured), dtype=np.uint32)
    return int(native.lib().ll_fft_table_merge(_u32p(m) if m.size else None, int(m.size)))


def fft_prune(lengths, ms_per_iter):
    """The -cufftbench pruning rule: which lengths (ascending) to keep."""
    n = np.ascontiguousarray(lengths, dtype=np.uint32)
    t = np.ascontiguousarray(ms_per_iter, dtype=np.float32)
    keep = np.zeros(n.size, dtype=np.int32)
    native.lib().ll_fft_prune(_u32p(n), t.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), int(n.size),
                              _i32p(keep))
    return [bool(k) for k in keep]


def fft_max_exponent(n):
    return int(native.lib().ll_fft_max_exponent(int(n)))


def context_bytes(q, n):
    """Device memory of a context for (q, n) in bytes (0: unsupported length)."""
    return int(native.lib().ll_context_bytes(int(q), int(n), None))


def device_name(device=0):
    buf = ctypes.create_string_buffer(256)
    if native.lib().ll_device_name(int(device), buf, 256):
        raise LLError(native.LL_ERR_CUDA, "ll_device_name(%d)" % device)
    return buf.value.decode()
