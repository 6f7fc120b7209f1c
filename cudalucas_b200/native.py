"""ctypes binding to libllb200.so, the C ABI declared in include/llb200.h.

The library is built in-tree (python -m cudalucas_b200.build); importing this
module never falls back to anything else: a missing or unloadable library
raises immediately."""
import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libllb200.so")

LL_OK = 0
LL_ERR_ARG = 1
LL_ERR_SHAPE = 2
LL_ERR_CUDA = 3
LL_ERR_NOMEM = 4
LL_ERR_STATE = 5
LL_ERR_TIMEOUT = 6
LL_ERR_INJECTED = 7
LL_REPORT = 1
LL_ERRCHK = 2
LL_ASYNC = 4
LL_STATIC_MAX_WORDS = 1 << 20
LL_KERNELS_GENERIC = 1
LL_KERNELS_FUSED = 2
LL_KERNELS_NO_PREFETCH = 4
LL_KERNELS_NO_CLUSTER = 8
LL_KERNELS_CLUSTER8 = 16
LL_KERNELS_ALT_WIDE = 32


class Tuning(ctypes.Structure):
    _fields_ = [("width", ctypes.c_int32), ("rows_per_cta", ctypes.c_int32),
                ("threads_wide", ctypes.c_int32), ("threads_tall", ctypes.c_int32),
                ("graph_iters", ctypes.c_int32), ("kernels", ctypes.c_int32),
                ("cluster_variant", ctypes.c_int32), ("reserved", ctypes.c_int32)]


_lib = None


def lib():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError("libllb200.so is not built (run: python -m cudalucas_b200.build)")
    L = ctypes.CDLL(LIB_PATH)
    vp, u32, i32, u64 = ctypes.c_void_p, ctypes.c_uint32, ctypes.c_int32, ctypes.c_uint64
    i32p = ctypes.POINTER(ctypes.c_int32)
    u32p = ctypes.POINTER(ctypes.c_uint32)
    fp = ctypes.POINTER(ctypes.c_float)
    sigs = {
        "ll_create": (i32, [ctypes.c_int, u32, u32, ctypes.POINTER(Tuning), ctypes.POINTER(vp)]),
        "ll_destroy": (None, [vp]),
        "ll_start": (i32, [vp, u32]),
        "ll_load_digits": (i32, [vp, i32p, u32]),
        "ll_step": (i32, [vp, u32, u32, fp]),
        "ll_read_digits": (i32, [vp, i32p, u32p]),
        "ll_res64": (i32, [vp, ctypes.POINTER(u64)]),
        "ll_sync": (i32, [vp]),
        "ll_busy": (i32, [vp]),
        "ll_device_checkpoint": (i32, [vp]),
        "ll_device_restore": (i32, [vp, u32p]),
        "ll_context_bytes": (u64, [u32, u32, ctypes.POINTER(Tuning)]),
        "ll_exponent": (u32, [vp]),
        "ll_fft_length": (u32, [vp]),
        "ll_offset": (u32, [vp]),
        "ll_stream": (vp, [vp]),
        "ll_shape": (None, [vp, i32p, i32p, i32p, i32p, i32p]),
        "ll_last_error": (ctypes.c_char_p, [vp]),
        "ll_kernel_kinds": (i32, [vp]),
        "ll_check_tables": (i32, []),
        "ll_status_string": (ctypes.c_char_p, [i32]),
        "ll_debug_inject_failure": (None, [vp, i32]),
        "ll_debug_launch": (i32, [vp, i32]),
        "ll_step_static": (i32, [ctypes.c_int, u32, u32, u32, u32, vp, vp, fp, vp]),
        "ll_batch_create": (i32, [ctypes.c_int, i32, u32p, u32p, i32, ctypes.POINTER(vp)]),
        "ll_batch_destroy": (None, [vp]),
        "ll_batch_size": (i32, [vp]),
        "ll_batch_member": (vp, [vp, i32]),
        "ll_batch_start": (i32, [vp, u32p]),
        "ll_batch_step": (i32, [vp, u32, u32, fp]),
        "ll_batch_sync": (i32, [vp]),
        "ll_batch_stream": (vp, [vp]),
        "ll_batch_group_by_length": (i32, [vp, i32]),
        "ll_batch_classes": (i32, [vp]),
        "ll_batch_res64": (i32, [vp, ctypes.POINTER(u64)]),
        "ll_digits_res64": (u64, [i32p, u32, u32, u32]),
        "ll_digits_standardize": (i32, [i32p, u32, u32]),
        "ll_pack_bits": (None, [i32p, u32p, u32, u32]),
        "ll_unpack_bits": (None, [u32p, i32p, u32, u32]),
        "ll_balance_digits": (None, [i32p, u32, u32]),
        "ll_checkpoint_checksum": (u32, [ctypes.c_char_p, ctypes.c_size_t]),
        "ll_additive_checksum": (u32, [u32p, ctypes.c_size_t]),
        "ll_fft_bounds": (None, [u32, u32p, u32p]),
        "ll_choose_fft_length": (u32, [u32, u32]),
        "ll_fft_table": (i32, [u32p, i32]),
        "ll_length_supported": (i32, [u32]),
        "ll_fft_table_merge": (i32, [u32p, i32]),
        "ll_fft_prune": (i32, [u32p, ctypes.POINTER(ctypes.c_float), i32, i32p]),
        "ll_fft_max_exponent": (u32, [u32]),
        "ll_device_name": (i32, [ctypes.c_int, ctypes.c_char_p, ctypes.c_size_t]),
    }
    for name, (res, args) in sigs.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    _lib = L
    return L
