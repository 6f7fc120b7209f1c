"""Batched mode: members of different FFT lengths advance in one graph per
step; each member's Res64 equals the solo run's (same kernels, independent
state), and equals exact arithmetic where that is cheap."""
import numpy as np
import pytest

import cudalucas_b200 as cl
from oracle import exact

pytestmark = pytest.mark.gpu

MIX = [(86243, 4096), (132049, 7168), (216091, 12288), (1257787, 65536), (2976221, 163840),
       (6972593, 393216), (20996011, 1179648)]


def solo(q, n, off, k):
    with cl.LLContext(q, n) as c:
        c.start(off)
        c.step(k, report=True)
        return c.res64()


def test_batch_equals_solo_and_exact():
    qs, ns = zip(*MIX)
    offs = [(q * 11) // 13 for q in qs]
    k = 257  # 25 graph replays of 10 + a remainder of 7 (the last one reporting)
    with cl.LLBatch(qs, ns, graph_iters=10) as b:
        b.start(offs)
        errs = b.step(k, report=True)
        got = b.res64()
    assert all(0 < e < 0.4 for e in errs)
    for (q, n), o, r in zip(MIX, offs, got):
        assert r == solo(q, n, o, k), q
    for (q, n), r in zip(MIX[:4], got[:4]):
        assert r == exact.res64(q, k), q


@pytest.mark.parametrize("by_length", [True, False])
def test_batch_length_classes_equal_solo(by_length):
    """Members of equal length launched together per pass (one launch per
    class) or separately give the solo residues."""
    mix = [(86243, 4096), (86249, 4096), (1257787, 65536), (1257827, 65536), (1257859, 65536),
           (216091, 12288), (216103, 12288), (2976221, 163840)]
    qs, ns = zip(*mix)
    offs = [(q * 5) // 9 for q in qs]
    with cl.LLBatch(qs, ns, graph_iters=8, by_length=by_length) as b:
        if by_length:
            assert b.classes >= 2
        b.start(offs)
        b.step(83, report=True)
        got = b.res64()
    for (q, n), o, r in zip(mix, offs, got):
        assert r == solo(q, n, o, 83), q


def test_batch_steps_compose():
    qs, ns = zip(*MIX[:3])
    with cl.LLBatch(qs, ns, graph_iters=8) as b:
        b.start([1, 2, 3])
        b.step(30)
        b.step(33, report=True)
        r1 = b.res64()
    with cl.LLBatch(qs, ns, graph_iters=8) as b:
        b.start([1, 2, 3])
        b.step(63, report=True)
        r2 = b.res64()
    assert r1 == r2 == [exact.res64(q, 63) for q in qs]


def test_batch_workload_generator_is_deterministic():
    from cudalucas_b200 import workloads
    a = workloads.batch_exponents(16)
    b = workloads.batch_exponents(16)
    assert a == b and len({p for p, _ in a}) == 16
    assert all(1e6 <= p <= 2.1e7 and n > 0 for p, n in a)
