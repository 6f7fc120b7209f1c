"""CPU tests of libllb200.so: every symbol declared in include/llb200.h is
exported, and the host helpers agree with the oracle's restatement of the
reference's residue, packing and checksum code."""
import os
import re

import numpy as np
import pytest

import cudalucas_b200 as cl
from cudalucas_b200 import native
from oracle import binding as ob
from oracle import exact

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    src = open(os.path.join(ROOT, "include", "llb200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(ll_[a-z0-9_]+)\s*\(", src)))


def test_all_declared_symbols_exported():
    L = native.lib()
    names = header_functions()
    assert len(names) >= 25
    for nm in names:
        assert hasattr(L, nm), nm


def random_balanced(q, n, rng):
    bits = ((-np.arange(n, dtype=np.int64) * (q % n)) % n < (q % n)).astype(np.int64) + q // n
    d = rng.integers(-(1 << (bits - 1)), (1 << (bits - 1)), dtype=np.int64)
    return d.astype(np.int32), bits


def digits_value(d, bits, q):
    x = 0
    for j in range(len(d) - 1, -1, -1):
        x = (x << int(bits[j])) + int(d[j])
    return x % ((1 << q) - 1)


@pytest.mark.parametrize("q,n", [(86243, 4096), (9689, 1024), (216091, 12288)])
def test_res64_matches_reference_find_residue_and_exact(q, n):
    rng = np.random.default_rng(q)
    for trial in range(5):
        d, bits = random_balanced(q, n, rng)
        off = int(rng.integers(0, q))
        M = (1 << q) - 1
        s = (digits_value(d, bits, q) * pow(2, q - off, M)) % M
        r = cl.digits_res64(d, q, n, off)
        assert r == s & 0xFFFFFFFFFFFFFFFF
        assert r == ob.find_residue(d, q, n, off)


def test_res64_of_zero_and_all_ones():
    q, n = 9689, 1024
    z = np.zeros(n, dtype=np.int32)
    assert cl.digits_res64(z, q, n, 17) == 0
    bits = ((-np.arange(n) * (q % n)) % n < (q % n)) + q // n
    ones = ((1 << bits) - 1).astype(np.int32)
    assert cl.digits_res64(ones, q, n, 17) == 0
    assert cl.standardize(ones, q, n)[1]


@pytest.mark.parametrize("q,n", [(86243, 4096), (132049, 7168)])
def test_pack_unpack_balance_match_oracle(q, n):
    rng = np.random.default_rng(1)
    d, bits = random_balanced(q, n, rng)
    std, zero = cl.standardize(d, q, n)
    assert not zero
    assert np.all(std >= 0) and np.all(std < (1 << bits))
    ref_std, _ = ob.standardize_digits(d, q, n)
    assert np.array_equal(std, ref_std)
    packed = cl.pack_bits(std, q, n)
    assert np.array_equal(packed, ob.pack_bits(std, q, n))
    un = cl.unpack_bits(packed, q, n)
    assert np.array_equal(un, ob.unpack_bits(packed, q, n))
    assert np.array_equal(un, std)
    bal = cl.balance_digits(un, q, n)
    assert np.array_equal(bal, ob.balance_digits(un, q, n))
    M = (1 << q) - 1
    assert digits_value(bal, bits, q) == digits_value(d, bits, q)


def test_checksums_match_oracle():
    rng = np.random.default_rng(3)
    for size in (0, 1, 7, 64, 4099):
        buf = rng.integers(0, 256, size, dtype=np.uint8).tobytes()
        assert cl.checkpoint_checksum(buf) == ob.checkpoint_checksum(buf)
    words = rng.integers(0, 2**32, 100, dtype=np.uint64).astype(np.uint32)
    assert cl.additive_checksum(words) == int(words.astype(np.uint64).sum()) & 0xFFFFFFFF


def test_fft_length_policy_matches_reference_choices():
    # CUDALucas picks 14K, 3136K and 19208K for these exponents (default table)
    assert cl.choose_fft_length(216091) == 14 * 1024
    assert cl.choose_fft_length(57885161) == 3136 * 1024
    assert cl.choose_fft_length(332192831) == 19208 * 1024
    # forced lengths inside the bounds are kept (init_ffts inserts them)
    assert cl.choose_fft_length(216091, 12288) == 12288
    assert cl.choose_fft_length(57885161, 3276800) == 3276800
    assert cl.choose_fft_length(332192831, 18874368) == 18874368
    lb, ub = cl.fft_bounds(216091)
    assert (lb, ub) == (10388, 24731)
    assert len(cl.fft_table()) == 162


def test_engine_supports_every_table_length_up_to_32m():
    # two passes of at most 4096-point transforms: n/2 <= 4096 * 4096
    for n in cl.fft_table():
        if n <= 32768 * 1024:
            assert cl.length_supported(n), n


def test_create_fails_cleanly_without_gpu_or_bad_args():
    with pytest.raises(cl.LLError):
        cl.LLContext(4, 1024)          # q <= n
    with pytest.raises(cl.LLError):
        cl.LLContext(216091, 1000)     # n not a multiple of 4 of a smooth length


def test_cufftbench_pruning_rule():
    """CUDALucas.cu:2500-2513: from the longest length down, a length stays
    when it is faster than every longer one; powers of two (in K) stay."""
    K = 1024
    lens = [2048 * K, 2880 * K, 3024 * K, 3136 * K, 3200 * K, 3584 * K]
    ms = [0.050, 0.058, 0.065, 0.0998, 0.062, 0.070]
    keep = cl.fft_prune(lens, ms)
    assert keep == [True, True, False, False, True, True]
    # a power of two slower than a longer length is still kept
    assert cl.fft_prune([4096 * K, 4320 * K], [0.09, 0.08]) == [True, True]
    assert cl.fft_prune([4000 * K, 4320 * K], [0.09, 0.08]) == [False, True]


def test_measured_table_replaces_builtin_lengths_in_its_range():
    """init_ffts with a `<gpu> fft.txt` (CUDALucas.cu:975-1021): inside the
    measured range only measured lengths remain, so an exponent whose
    default length (3136K for M57885161) measured slower than 3200K gets
    3200K; outside the range the built-in lengths stay."""
    K = 1024
    lens = [2880 * K, 3024 * K, 3136 * K, 3200 * K, 3584 * K]
    ms = [0.058, 0.065, 0.0998, 0.062, 0.070]
    kept = [n for n, k in zip(lens, cl.fft_prune(lens, ms)) if k]
    try:
        size = cl.fft_table_merge(kept)
        table = cl.fft_table()
        assert size == len(table)
        assert 3136 * K not in table and 3200 * K in table
        assert cl.choose_fft_length(57885161) == 3200 * K
        assert cl.choose_fft_length(216091) == 14 * K          # below the measured range
        assert cl.choose_fft_length(332192831) == 19208 * K    # above it
        assert table == sorted(table)
    finally:
        cl.fft_table_merge([])
    assert cl.choose_fft_length(57885161) == 3136 * K
    assert len(cl.fft_table()) == 162


def test_fft_max_exponent_inverts_the_lower_bound():
    for n in (12288, 3276800, 18874368):
        q = cl.fft_max_exponent(n)
        assert cl.fft_bounds(q)[0] <= n < cl.fft_bounds(q + 1)[0]


def test_kernel_tables_are_consistent():
    """Every specialised kernel's stage-twiddle table, built on the host from
    the radix list recorded beside it, has the size the kernel reads (the
    cluster kernels' row lists of four radices included)."""
    assert native.lib().ll_check_tables() == 0
