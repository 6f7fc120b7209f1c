"""The serving scheduler, on the CPU with a fake engine (exact big-integer
LL with simulated GPU time), and on the GPU (results equal solo runs)."""
import time

import pytest

from cudalucas_b200 import serve
from oracle import exact


class FakeEngine:
    """Exact LL on Python integers; a chunk 'runs' for iters * cost seconds."""

    def __init__(self, cost=1e-6):
        self.cost = cost
        self.opened = []

    def open(self, req):
        self.opened.append(req.rid)
        return {"p": req.p, "s": 4, "done_at": 0.0}

    def enqueue(self, h, iters):
        M = (1 << h["p"]) - 1
        for _ in range(iters):
            h["s"] = (h["s"] * h["s"] - 2) % M
        h["done_at"] = time.perf_counter() + iters * self.cost

    def busy(self, h):
        return time.perf_counter() < h["done_at"]

    def finish(self, h):
        self.enqueue(h, 1)
        return h["s"] & 0xFFFFFFFFFFFFFFFF, 0.1

    def close(self, h):
        pass


def make(n=12, seed=0):
    import random
    rnd = random.Random(seed)
    ps = [521, 607, 1279, 2203, 2281, 3217, 4253, 4423, 9689, 9941, 11213, 19937]
    return [serve.Request(rid=i, arrival=0.002 * i, p=ps[i % len(ps)], n=1024, iters=rnd.randint(5, 300))
            for i in range(n)]


def test_continuous_batching_results_and_latency():
    reqs = make()
    serve.Server(FakeEngine(), chunk=50).run(reqs)
    for r in reqs:
        assert r.res64 == exact.res64(r.p, r.iters)
        assert r.finished >= r.admitted >= r.arrival - 1e-3
    s = serve.summary(reqs)
    assert s["requests"] == len(reqs) and s["p99_s"] >= s["p50_s"] > 0


def test_admission_respects_device_budget():
    reqs = make(8)
    eng = FakeEngine(cost=2e-5)
    srv = serve.Server(eng, hbm_cap=2 * serve.STATE_BYTES_PER_WORD * 1024, chunk=20)
    peak = {"v": 0}
    orig_open = eng.open

    def tracking_open(req):
        h = orig_open(req)
        return h
    eng.open = tracking_open
    srv.run(reqs, realtime=False)
    assert eng.opened == sorted(eng.opened)          # FIFO admission
    assert all(r.res64 == exact.res64(r.p, r.iters) for r in reqs)


def test_request_larger_than_budget_is_rejected():
    reqs = [serve.Request(rid=0, arrival=0.0, p=521, n=1 << 20, iters=3)]
    with pytest.raises(RuntimeError):
        serve.Server(FakeEngine(), hbm_cap=1000).run(reqs)


def test_serial_baseline_matches():
    reqs = make(6)
    serve.serve_serial(FakeEngine(), reqs, realtime=False)
    assert all(r.res64 == exact.res64(r.p, r.iters) for r in reqs)


@pytest.mark.gpu
def test_gpu_serving_results_equal_solo_runs():
    import cudalucas_b200 as cl
    reqs = [serve.Request(rid=i, arrival=0.01 * i, p=p, n=cl.choose_fft_length(p), iters=k, offset=i)
            for i, (p, k) in enumerate([(86243, 3000), (132049, 1500), (216091, 4000), (1257787, 800),
                                        (2976221, 600), (86243, 2500), (756839, 1200)])]
    serve.Server(serve.GpuEngine(), chunk=400).run(reqs)
    for r in reqs:
        with cl.LLContext(r.p, r.n) as c:
            c.start(r.offset)
            c.step(r.iters, report=True)
            assert c.res64() == r.res64, r.rid
