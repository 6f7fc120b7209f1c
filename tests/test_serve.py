"""The serving scheduler, on the CPU with a fake engine (exact big-integer
LL with simulated GPU time), and on the GPU (results equal solo runs)."""
import time

import pytest

from cudalucas_b200 import serve
from oracle import exact


class FakeEngine:
    """Exact LL on Python integers; a chunk 'runs' for iters * cost seconds.
    bad_chunks: {rid: number of chunk results to report with a roundoff
    error above the limit} (the fault is in the reading, as a transient
    error would be; the state itself stays exact)."""

    def __init__(self, cost=1e-6, bad_chunks=None):
        self.cost = cost
        self.opened = []
        self.bad = dict(bad_chunks or {})
        self.restores = 0

    def footprint(self, req):
        return 16 * req.n

    def open(self, req):
        self.opened.append(req.rid)
        return {"rid": req.rid, "p": req.p, "s": 4, "ck": 4, "done_at": 0.0}

    def enqueue(self, h, iters):
        M = (1 << h["p"]) - 1
        for _ in range(iters):
            h["s"] = (h["s"] * h["s"] - 2) % M
        h["done_at"] = time.perf_counter() + iters * self.cost

    def busy(self, h):
        return time.perf_counter() < h["done_at"]

    def check(self, h):
        if self.bad.get(h["rid"], 0) > 0:
            self.bad[h["rid"]] -= 1
            return 0.45
        return 0.1

    def commit(self, h):
        h["ck"] = h["s"]

    def restore(self, h):
        self.restores += 1
        h["s"] = h["ck"]

    def result(self, h):
        return h["s"] & 0xFFFFFFFFFFFFFFFF

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
    srv = serve.Server(eng, hbm_cap=2 * 16 * 1024, chunk=20)
    srv.run(reqs, realtime=False)
    assert eng.opened == sorted(eng.opened)          # FIFO admission
    assert srv.peak_bytes <= 2 * 16 * 1024 and srv.peak_active <= 2
    assert all(r.res64 == exact.res64(r.p, r.iters) for r in reqs)


def test_chunk_over_the_error_limit_is_rerun_from_the_device_checkpoint():
    reqs = make(6)
    eng = FakeEngine(bad_chunks={2: 1, 4: 1})
    serve.Server(eng, chunk=40).run(reqs, realtime=False)
    assert eng.restores == 2
    assert all(r.error is None and r.res64 == exact.res64(r.p, r.iters) for r in reqs)


def test_request_fails_when_the_error_repeats():
    reqs = make(4)
    eng = FakeEngine(bad_chunks={1: 2})
    serve.Server(eng, chunk=40).run(reqs, realtime=False)
    assert reqs[1].res64 is None and "roundoff error" in reqs[1].error
    assert all(r.res64 == exact.res64(r.p, r.iters) for r in reqs if r.rid != 1)
    assert serve.summary(reqs)["failed"] == 1


def test_request_larger_than_budget_is_rejected():
    reqs = [serve.Request(rid=0, arrival=0.0, p=521, n=1 << 20, iters=3)]
    with pytest.raises(RuntimeError):
        serve.Server(FakeEngine(), hbm_cap=1000).run(reqs)


def test_serial_baseline_matches():
    reqs = make(6)
    serve.serve_serial(FakeEngine(), reqs, realtime=False)
    assert all(r.res64 == exact.res64(r.p, r.iters) for r in reqs)


GPU_MIX = [(86243, 3000), (132049, 1500), (216091, 4000), (1257787, 800), (2976221, 600), (86243, 2500),
           (756839, 1200)]


def gpu_requests():
    import cudalucas_b200 as cl
    return [serve.Request(rid=i, arrival=0.01 * i, p=p, n=cl.choose_fft_length(p), iters=k, offset=i)
            for i, (p, k) in enumerate(GPU_MIX)]


def solo_res64(r):
    import cudalucas_b200 as cl
    with cl.LLContext(r.p, r.n) as c:
        c.start(r.offset)
        c.step(r.iters, report=True)
        return c.res64()


@pytest.mark.gpu
def test_gpu_serving_results_equal_solo_runs():
    reqs = gpu_requests()
    serve.Server(serve.GpuEngine(), chunk=400).run(reqs)
    for r in reqs:
        assert r.error is None and r.res64 == solo_res64(r), r.rid


@pytest.mark.gpu
def test_gpu_serving_under_a_binding_memory_budget():
    """A budget that holds two of the largest requests at a time: admission
    waits, and the replies are still the solo results."""
    eng = serve.GpuEngine()
    reqs = gpu_requests()
    cap = 2 * max(eng.footprint(r) for r in reqs)
    srv = serve.Server(eng, hbm_cap=cap, chunk=400)
    srv.run(reqs)
    assert srv.peak_bytes <= cap and srv.peak_active < len(reqs)
    for r in reqs:
        assert r.error is None and r.res64 == solo_res64(r), r.rid


@pytest.mark.gpu
def test_device_checkpoint_restore_replays_identically():
    """ll_device_checkpoint / ll_device_restore: a run that goes back to its
    device checkpoint and repeats a chunk ends on the same residue."""
    import cudalucas_b200 as cl
    from oracle import exact
    q, n = 216091, cl.choose_fft_length(216091)
    with cl.LLContext(q, n) as c:
        c.start(77)
        c.step(300, report=True, wait=False)
        c.device_checkpoint()
        off = c.offset
        c.step(500, report=True)
        r1 = c.res64()
        assert c.device_restore() == off
        c.step(500, report=True)
        assert c.res64() == r1 == exact.res64(q, 800)
