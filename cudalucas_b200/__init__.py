"""cudalucas_b200: a B200-native Lucas-Lehmer engine (IBDWT squaring in FP64
on sm_100a) behind a C ABI, with a Python host mirror for tests and benches."""
from .engine import (LLBatch, LLContext, LLError, additive_checksum, balance_digits,  # noqa: F401
                     checkpoint_checksum, choose_fft_length, context_bytes, device_name, digits_res64, fft_bounds,
                     fft_max_exponent, fft_prune, fft_table, fft_table_merge, length_supported, pack_bits,
                     standardize, unpack_bits)
