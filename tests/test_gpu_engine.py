"""GPU parity tests: the CUDA engine (through the C ABI) against the oracle.

Res64 is compared bit-exactly; digit vectors are compared after
canonicalisation (exact value mod 2^q-1), and against the numpy model of the
engine's own carry scheme bit for bit.  The roundoff error is checked against
the reference's 0.40 limit (CUDALucas.cu:2765) and against the oracle's error
within a factor of 2 (FFT rounding differs between implementations)."""
import numpy as np
import pytest

import cudalucas_b200 as cl
import ibdwt_model
from golden_data import kats, large_entries, reference_run_entries
from oracle import exact
from oracle.binding import Oracle

pytestmark = pytest.mark.gpu
KAT = dict(kats())


def engine_run(q, n, offset, k, **tuning):
    with cl.LLContext(q, n, tuning=tuning or None) as c:
        c.start(offset)
        err = c.step(k, report=True)
        d, off = c.read_digits()
        return d, off, err, c.shape


@pytest.mark.parametrize("q,n", [(86243, 4096), (132049, 7168), (216091, 12288), (216091, 14336),
                                 (756839, 40960), (1257787, 65536), (2976221, 163840), (6972593, 393216)])
def test_parity_with_oracle(q, n):
    k = 60
    off = (q * 5) // 11
    d, o_off, err, shape = engine_run(q, n, off, k)
    o = Oracle(q, n)
    o.start(off)
    oerr = o.step(k)
    od = o.digits()
    assert o_off == o.offset
    sd, _ = cl.standardize(d, q, n)
    so, _ = cl.standardize(od, q, n)
    assert np.array_equal(sd, so)
    assert cl.digits_res64(d, q, n, o_off) == o.res64()
    assert err < 0.4
    assert err <= 2 * oerr + 1e-3 and oerr <= 2 * err + 1e-3, (err, oerr)


@pytest.mark.parametrize("q,n", [(86243, 4096), (216091, 12288), (1257787, 65536)])
def test_digits_match_engine_model_bit_for_bit(q, n):
    # the model follows the generic kernels' carry (c2 added after balancing);
    # the specialised wide pass adds c1 + c2 before, which gives other digits
    # of the same value (checked by the parity tests)
    off = q // 7
    d, _, _, shape = engine_run(q, n, off, 25, rows_per_cta=2)
    m = ibdwt_model.Model(q, n, shape["W"])
    m.start(off)
    for _ in range(25):
        m.iterate()
    assert np.array_equal(d.astype(np.int64), m.digits)


def test_report_split_equals_single_run():
    q, n = 132049, 7168
    with cl.LLContext(q, n) as c:
        c.start(3)
        c.step(40, report=True)
        c.step(60, report=True)
        d1, o1 = c.read_digits()
    d2, o2, _, _ = engine_run(q, n, 3, 100)
    assert o1 == o2
    assert np.array_equal(cl.standardize(d1, q, n)[0], cl.standardize(d2, q, n)[0])


def test_load_digits_resume_equals_continuous():
    q, n = 216091, 12288
    with cl.LLContext(q, n) as c:
        c.start(1000)
        c.step(500, report=True)
        mid, off = c.read_digits()
    with cl.LLContext(q, n) as c:
        c.load_digits(cl.balance_digits(cl.standardize(mid, q, n)[0], q, n), off)
        c.step(500, report=True)
        r_resumed = c.res64()
    assert r_resumed == exact.res64(q, 1000)


@pytest.mark.parametrize("p,r", kats("tests"))
def test_selftest_short_table(p, r):
    n = cl.choose_fft_length(p)
    with cl.LLContext(p, n) as c:
        c.start((p * 3) // 17)
        err = c.step(10000, report=True)
        assert c.res64() == r
        assert err < 0.4


@pytest.mark.slow
@pytest.mark.parametrize("p,r", kats("testl"))
def test_selftest_long_table(p, r):
    n = cl.choose_fft_length(p)
    with cl.LLContext(p, n) as c:
        c.start((p * 3) // 17)
        err = c.step(10000, report=True)
        assert c.res64() == r
        assert err < 0.4


def test_c1_full_test_216091_is_prime():
    """C1: the whole test at 12K; Res64 at every 10000 equals the reference
    binary's report lines (CUDALucas -f 12K -x 10000 216091), the final
    residue is 0."""
    q, n = 216091, 12288
    ref = {k: r for p, k, r in reference_run_entries() if p == q}
    assert len(ref) == 21
    with cl.LLContext(q, n) as c:
        c.start(0)
        done, maxerr = 0, 0.0
        while done < q - 2:
            k = min(10000, q - 2 - done)
            maxerr = max(maxerr, c.step(k, report=True))
            done += k
            if done in ref:
                assert c.res64() == ref[done], done
            if done == 10000:
                assert c.res64() == KAT[q]
        assert c.res64() == 0
        assert maxerr < 0.4


def test_c2_3200k_matches_exact_kat_and_reference_binary():
    """C2: Res64 at every 10000 through 110000 equals the reference binary's
    (CUDALucas -f 3200K -x 10000 57885161), and the exact values at 1..1000."""
    q, n = 57885161, 3276800
    checks = {k: r for p, k, r in large_entries() + reference_run_entries() if p == q and k <= 110000}
    assert all(k in checks for k in range(10000, 110001, 10000))
    with cl.LLContext(q, n) as c:
        c.start(0)
        done = 0
        for k in sorted(set(checks) | {10000}):
            err = c.step(k - done, report=True)
            done = k
            assert err < 0.4
            assert c.res64() == checks.get(k, KAT[q] if k == 10000 else None)


def test_c3_18432k_matches_exact_and_reference_binary():
    q, n = 332192831, 18874368
    checks = {k: r for p, k, r in large_entries() + reference_run_entries() if p == q}
    if not checks:
        pytest.skip("large fixture not generated")
    with cl.LLContext(q, n) as c:
        c.start(0)
        done = 0
        for k in sorted(checks):
            err = c.step(k - done, report=True)
            done = k
            assert err < 0.4
            assert c.res64() == checks[k]


@pytest.mark.parametrize("q,n,widths", [
    # N = 1024*1024: specialised rows of 512 (4 per CTA), 1024 and 2048 (2 per
    # CTA), columns with half-exchange pairing, and the generic kernels
    (36700049, 2097152, [512, 1024, 2048, None]),
    # N = 1280*768: columns of 768 and 1280 (threads of both columns in one
    # warp), rows of 1280 and 768
    (34603069, 1966080, [768, 1280, None]),
    # N = 256*512: the two-stage (16, 16) rows and columns of 256
    (4587533, 262144, [256, 512, None]),
    (2293771, 131072, [256, None]),
])
def test_kernel_variants_agree(q, n, widths):
    """Every launch shape of one length (specialised kernels for several row
    and column lengths, and the generic kernels) gives the oracle's residue
    after a few iterations and the same residue after many."""
    off = q // 3
    o = Oracle(q, n)
    o.start(off)
    o.step(8)
    want8 = o.res64()
    got8, got300 = {}, {}
    for w in widths:
        tuning = {"width": w} if w else {"width": 1024, "rows_per_cta": 2}
        with cl.LLContext(q, n, tuning=tuning) as c:
            c.start(off)
            e1 = c.step(8, report=True)
            got8[w] = c.res64()
            e2 = c.step(292, report=True)
            got300[w] = c.res64()
            assert max(e1, e2) < 0.4, (w, e1, e2)
    assert all(v == want8 for v in got8.values()), (want8, got8)
    assert len(set(got300.values())) == 1, got300


def test_independent_contexts_interleaved():
    a = cl.LLContext(86243, 4096)
    b = cl.LLContext(132049, 7168)
    a.start(11)
    b.start(22)
    for _ in range(5):
        a.step(200)
        b.step(200)
    a.step(0, report=True)
    a.step(1, report=True)
    b.step(1, report=True)
    ra, rb = a.res64(), b.res64()
    a.close()
    b.close()
    assert ra == exact.res64(86243, 1001)
    assert rb == exact.res64(132049, 1001)


def test_injected_failure_is_reported_and_recoverable():
    with cl.LLContext(86243, 4096) as c:
        c.start(0)
        c.inject_failure(1)
        with pytest.raises(cl.LLError) as ei:
            c.step(10)
        assert ei.value.status == 7
        c.step(100, report=True)
        assert c.res64() == exact.res64(86243, 100)


def test_read_digits_requires_report():
    with cl.LLContext(86243, 4096) as c:
        c.start(0)
        c.step(5)
        with pytest.raises(cl.LLError):
            c.read_digits()


@pytest.mark.parametrize("q,n", [(86243, 4096), (216091, 12288), (1257787, 65536)])
def test_words_beyond_fp64_range_report_max_error(q, n):
    """Digits far outside the balanced range push the squared words beyond
    2^51, where the roundoff reading has no fraction bits left; the wide pass
    flags it and ll_step reports an error of 1.0 (generic and specialised
    kernels)."""
    with cl.LLContext(q, n) as c:
        c.load_digits(np.full(n, 1 << 29, dtype=np.int32), 5)
        assert c.step(1, report=True) == 1.0


def _exponent_at(n, bits=17.6):
    from cudalucas_b200.fftbench import is_prime
    q = int(n * bits) | 1
    while not is_prime(q):
        q += 2
    return q


@pytest.mark.parametrize("nk", [12, 14, 50, 56, 60, 64, 70, 80, 96, 112, 120, 126, 144, 160, 162, 180, 224, 288, 320, 336,
                                360, 392, 400, 448, 576, 864, 900, 3136])
def test_specialised_columns_of_any_radix_list(nk):
    """Lengths whose columns are not 16 x M x 16 (C1's 12K, the batch set's
    50K-900K, 3136K, the default length of M57885161) run a specialised
    tall pass (tall_any) and give the oracle's residue."""
    from oracle.binding import set_threads
    n = nk * 1024
    q = _exponent_at(n)
    k = 12
    off = q // 5
    d, o_off, err, shape = engine_run(q, n, off, k, kernels=cl.native.LL_KERNELS_NO_CLUSTER)
    assert shape["tall_specialised"] and shape["wide_specialised"] and not shape["cluster"], shape
    set_threads(8)
    try:
        o = Oracle(q, n)
        o.start(off)
        oerr = o.step(k)
        want = o.res64()
    finally:
        set_threads(1)
    assert cl.digits_res64(d, q, n, o_off) == want
    assert err < 0.4 and err <= 2 * oerr + 1e-3 and oerr <= 2 * err + 1e-3, (err, oerr)


@pytest.mark.parametrize("n", [12288, 14336, 57344])
def test_fused_iterations_equal_two_launch_iterations(n):
    """On request, short lengths run their plain iterations as one
    cooperative launch with grid barriers between the passes.  The carry of
    element (m1, m2) comes from element (m1, m2-1) whichever CTA holds it, so
    the digits are bit for bit those of two launches per iteration; they
    match the oracle's residue."""
    q = _exponent_at(n)
    off = q // 3
    d1, o1, e1, s1 = engine_run(q, n, off, 700, kernels=cl.native.LL_KERNELS_FUSED)
    d2, o2, e2, s2 = engine_run(q, n, off, 700, kernels=cl.native.LL_KERNELS_NO_CLUSTER)
    assert s1["fused"] and not s2["fused"] and not s2["cluster"], (s1, s2)
    assert o1 == o2 and np.array_equal(d1, d2) and e1 == e2
    o = Oracle(q, n)
    o.start(off)
    o.step(700)
    assert cl.digits_res64(d1, q, n, o1) == o.res64()


@pytest.mark.parametrize("n", [8192, 10240, 12288, 14336, 16384, 18432, 20480, 32768, 36864, 43008, 49152, 57344])
def test_cluster_iterations_equal_two_launch_iterations(n):
    """Short lengths run every step as one launch of one thread-block
    cluster whose shared memory holds the state (cluster_iters).  After many
    iterations (several launches, a report in the last one) the digits are
    bit for bit those of two launches per iteration (the rounded values
    agree), the roundoff maximum agrees within rounding (the row transforms
    are factored differently), and the residue is the oracle's."""
    q = _exponent_at(n)
    off = q // 3
    with cl.LLContext(q, n) as c:
        assert c.shape["cluster"], c.shape
        c.start(off)
        e1 = max(c.step(333, report=True), c.step(1, report=True), c.step(366, report=True))
        d1, o1 = c.read_digits()
    d2, o2, e2, s2 = engine_run(q, n, off, 700, kernels=cl.native.LL_KERNELS_NO_CLUSTER)
    assert not s2["cluster"]
    assert o1 == o2 and np.array_equal(d1, d2), (o1, o2)
    assert e1 < 0.4 and e1 <= 1.5 * e2 + 1e-3 and e2 <= 1.5 * e1 + 1e-3, (e1, e2)
    o = Oracle(q, n)
    o.start(off)
    o.step(700)
    assert cl.digits_res64(d1, q, n, o1) == o.res64()


@pytest.mark.parametrize("tuning", [{"kernels": 16}, {"cluster_variant": 1}, {"cluster_variant": 2}])
def test_cluster_variants_agree(tuning):
    """The cluster variants of 12K (clusters of 16 or 8 CTAs, rows on 64 or
    32 threads) give the same digits as the default and the exact residue."""
    q, n = 216091, 12288
    d1, o1, e1, s1 = engine_run(q, n, 77, 500, **tuning)
    d0, o0, e0, s0 = engine_run(q, n, 77, 500)
    assert s1["cluster"] and s0["cluster"]
    assert o1 == o0 and np.array_equal(d1, d0)
    assert cl.digits_res64(d1, q, n, o1) == exact.res64(q, 500)


@pytest.mark.parametrize("n", [2097152, 3276800])
def test_alternative_row_kernel_agrees(n):
    """The alternative row kernel (rows in shared memory, 8 elements per
    thread: 1024 = 8x4x4x8, 1280 = 8x4x5x8) gives the digits of the default
    row kernel and the oracle's residue."""
    q = _exponent_at(n)
    off = q // 7
    d1, o1, e1, s1 = engine_run(q, n, off, 300, kernels=cl.native.LL_KERNELS_ALT_WIDE)
    d2, o2, e2, s2 = engine_run(q, n, off, 300)
    assert s1["W"] == s2["W"] and s1["threads_wide"] != s2["threads_wide"], (s1, s2)
    assert o1 == o2 and np.array_equal(d1, d2)
    assert e1 < 0.4 and e1 <= 1.5 * e2 + 1e-3 and e2 <= 1.5 * e1 + 1e-3, (e1, e2)
    from oracle.binding import set_threads
    set_threads(16)
    try:
        o = Oracle(q, n)
        o.start(off)
        o.step(8)
        want = o.res64()
    finally:
        set_threads(1)
    d3, o3, _, _ = engine_run(q, n, off, 8, kernels=cl.native.LL_KERNELS_ALT_WIDE)
    assert cl.digits_res64(d3, q, n, o3) == want


@pytest.mark.parametrize("nk", [6048, 6480, 7200, 7776, 8640, 10584, 10800, 11200, 12096, 12960, 14400, 17496,
                                18144, 19600, 20000, 23328, 23814, 24300, 24500, 25600, 26244])
def test_long_lengths_columns_agree_with_generic_kernels(nk):
    """The column lengths of the long table lengths (1620-4374, up to four
    stages of radices <= 16) run tall_any; after a few iterations the digits
    equal (modulo 2^q-1) those of the generic kernels, and so does Res64."""
    n = nk * 1024
    q = _exponent_at(n, 17.3)
    off = q // 9
    d1, o1, e1, s1 = engine_run(q, n, off, 6)
    assert s1["tall_specialised"], s1
    d2, o2, e2, s2 = engine_run(q, n, off, 6, kernels=cl.native.LL_KERNELS_GENERIC)
    assert not s2["tall_specialised"]
    assert o1 == o2
    assert np.array_equal(cl.standardize(d1, q, n)[0], cl.standardize(d2, q, n)[0])
    assert cl.digits_res64(d1, q, n, o1) == cl.digits_res64(d2, q, n, o2)
    assert e1 < 0.4 and e2 < 0.4


@pytest.mark.parametrize("nk", [288, 640, 1296, 1344, 1440, 2880, 14336])
def test_preferred_shapes_agree_with_heuristic_shapes(nk):
    """Lengths with a built-in launch preference (a row width, and for some
    the alternative row kernel, measured faster than the width nearest
    sqrt(N)) give the digits of the heuristic shape (any explicit tuning
    skips the preference) and the oracle's residue."""
    n = nk * 1024
    q = _exponent_at(n)
    off = q // 5
    d1, o1, e1, s1 = engine_run(q, n, off, 40)
    d2, o2, e2, s2 = engine_run(q, n, off, 40, kernels=cl.native.LL_KERNELS_NO_CLUSTER)
    assert (s1["W"], s1["threads_wide"]) != (s2["W"], s2["threads_wide"]), (s1, s2)
    assert s1["wide_specialised"] and s1["tall_specialised"]
    assert o1 == o2
    assert np.array_equal(cl.standardize(d1, q, n)[0], cl.standardize(d2, q, n)[0])
    assert e1 < 0.4 and e2 < 0.4
    if n <= 2 * 1024 * 1024:
        from oracle.binding import set_threads
        set_threads(16)
        try:
            o = Oracle(q, n)
            o.start(off)
            o.step(40)
            want = o.res64()
        finally:
            set_threads(1)
        assert cl.digits_res64(d1, q, n, o1) == want
