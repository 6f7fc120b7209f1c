"""CPU tests of the oracle: the C restatement of CUDALucas's IBDWT step
(oracle/ibdwt_oracle.c) and exact big-integer LL (oracle/exact.py), pinned to
the reference's self-test table (CUDALucas.cu:2673-2729) and to each other.
Also checks the numpy model of the engine's own two-pass algorithm."""
import numpy as np
import pytest

from golden_data import exact_entries, kats
from oracle import exact
from oracle.binding import Oracle
import ibdwt_model

KAT = dict(kats())


def test_kat_fixture_integrity():
    assert len(kats("tests")) == 20 and len(kats("testl")) == 92
    assert KAT[86243] == 0x23992CCD735A03D9
    assert KAT[57885161] == 0x76C27556683CD84D


@pytest.mark.parametrize("p", [22133, 43633, 86243, 132049])
def test_exact_matches_kat(p):
    assert exact.res64(p, 10000) == KAT[p]


@pytest.mark.parametrize("p,n,bigcarry", [(22133, 1024, 1), (43633, 2048, 0), (86243, 4096, 1),
                                          (132049, 7168, 1), (216091, 14336, 0)])
def test_oracle_ibdwt_matches_kat(p, n, bigcarry):
    o = Oracle(p, n, bigcarry=bool(bigcarry))
    o.start(offset=(p * 7) // 13)
    err = o.step(10000)
    assert err < 0.4
    assert o.res64() == KAT[p]


@pytest.mark.parametrize("p,k,r", [e for e in exact_entries() if e[0] >= 9000 and e[1] <= 500])
def test_oracle_ibdwt_matches_exact(p, k, r):
    import cudalucas_b200 as cl
    n = cl.choose_fft_length(p)
    o = Oracle(p, n)
    o.start(offset=12345 % p)
    o.step(k)
    assert o.res64() == r


@pytest.mark.parametrize("p", [9689, 9941, 11213])
def test_oracle_full_test_mersenne_prime(p):
    o = Oracle(p, 1024)
    o.start(offset=5)
    o.step(p - 2)
    assert o.res64() == 0


def test_oracle_full_test_composite():
    p = 9697  # prime exponent, 2^p-1 composite
    o = Oracle(p, 1024)
    o.start(offset=0)
    o.step(p - 2)
    assert o.res64() == exact.res64(p, p - 2) != 0


def test_exact_fixture_self_consistent():
    for p, k, r in exact_entries():
        if p < 30000:
            assert exact.res64(p, k) == r


@pytest.mark.parametrize("q,n,W", [(86243, 4096, 32), (216091, 12288, 64), (132049, 8192, 64),
                                   (1257787, 65536, 256)])
def test_engine_model_matches_exact(q, n, W):
    m = ibdwt_model.Model(q, n, W)
    m.start(offset=(q // 3))
    for _ in range(12):
        err = m.iterate()
    assert err < 0.4
    M = (1 << q) - 1
    x = ibdwt_model.digits_value(m.digits, q, n)
    s = (x * pow(2, q - m.offset, M)) % M
    assert s == exact.ll_state(q, 12)
