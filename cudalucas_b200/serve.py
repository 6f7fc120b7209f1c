"""Serving loop: LL tests as requests, continuous batching on one GPU.

A request is (exponent p, FFT length n, iterations k); the reply is Res64 of
s_k.  Requests are admitted as they arrive while the device-state budget
allows (about 16 bytes per FP64 word: transform array, digits, carry rows;
150 GB by default), every admitted request gets its own context and stream,
and the loop keeps all of them busy: whenever a request's previous chunk of
iterations has finished on the GPU it enqueues the next chunk, so requests
that arrive while others run join the work on the device at once.  The last
iteration of a request is a report step; its Res64 is the reply.

The engine is pluggable: `GpuEngine` drives libllb200 through the C ABI;
tests drive the same scheduler with a CPU fake.
"""
import heapq
import time
from dataclasses import dataclass, field

STATE_BYTES_PER_WORD = 16


@dataclass
class Request:
    rid: int
    arrival: float
    p: int
    n: int
    iters: int
    offset: int = 0
    # filled in by the server
    admitted: float = None
    finished: float = None
    res64: int = None
    max_err: float = 0.0

    @property
    def latency(self):
        return None if self.finished is None else self.finished - self.arrival

    @property
    def footprint(self):
        return STATE_BYTES_PER_WORD * self.n


class GpuEngine:
    """Adapter from the scheduler to LLContext (one context per request)."""

    def __init__(self, device=0):
        self.device = device

    def open(self, req):
        from .engine import LLContext
        c = LLContext(req.p, req.n, device=self.device)
        c.start(req.offset)
        return c

    def enqueue(self, h, iters):
        h.step(iters)          # enqueues only (no flags)

    def busy(self, h):
        return h.busy()

    def finish(self, h):
        err = h.step(1, report=True)
        return h.res64(), err

    def close(self, h):
        h.close()


@dataclass(order=True)
class _Arrival:
    time: float
    rid: int = field(compare=True)


class Server:
    def __init__(self, engine, hbm_cap=150e9, chunk=1000, max_active=128, clock=time.perf_counter):
        self.engine = engine
        self.hbm_cap = hbm_cap
        self.chunk = chunk
        self.max_active = max_active
        self.clock = clock

    def run(self, requests, realtime=True):
        """Serves `requests` (arrival times relative to the start).  With
        realtime=False arrivals are not waited for (all are available at t=0
        in arrival order).  Returns the requests with results filled in."""
        pending = sorted(requests, key=lambda r: r.arrival)
        waiting = []                       # arrived, not yet admitted (FIFO)
        active = {}                        # rid -> [req, handle, remaining]
        used = 0
        t0 = self.clock()
        i = 0
        while i < len(pending) or waiting or active:
            now = self.clock() - t0
            while i < len(pending) and (pending[i].arrival <= now or not realtime):
                waiting.append(pending[i])
                i += 1
            # admission: FIFO while the device-state budget and slots allow
            while waiting and len(active) < self.max_active and used + waiting[0].footprint <= self.hbm_cap:
                r = waiting.pop(0)
                r.admitted = self.clock() - t0
                h = self.engine.open(r)
                active[r.rid] = [r, h, r.iters]
                used += r.footprint
            if waiting and not active:
                raise RuntimeError("request %d does not fit the device-state budget" % waiting[0].rid)
            # keep every active request busy; retire the finished ones
            progressed = False
            for rid in list(active):
                r, h, rem = active[rid]
                if self.engine.busy(h):
                    continue
                progressed = True
                if rem > 1:
                    k = min(self.chunk, rem - 1)
                    self.engine.enqueue(h, k)
                    active[rid][2] = rem - k
                else:
                    r.res64, r.max_err = self.engine.finish(h)
                    r.finished = self.clock() - t0
                    self.engine.close(h)
                    used -= r.footprint
                    del active[rid]
            if not progressed:
                time.sleep(0.0002)
        return requests


def serve_serial(engine, requests, realtime=True, clock=time.perf_counter):
    """Baseline: the same requests one at a time, in arrival order."""
    t0 = clock()
    for r in sorted(requests, key=lambda r: r.arrival):
        now = clock() - t0
        if realtime and r.arrival > now:
            time.sleep(r.arrival - now)
        r.admitted = clock() - t0
        h = engine.open(r)
        if r.iters > 1:
            engine.enqueue(h, r.iters - 1)
        while engine.busy(h):
            time.sleep(0.0002)
        r.res64, r.max_err = engine.finish(h)
        r.finished = clock() - t0
        engine.close(h)
    return requests


def summary(requests):
    import numpy as np
    lat = np.array([r.latency for r in requests])
    span = max(r.finished for r in requests) - min(r.arrival for r in requests)
    iters = sum(r.iters for r in requests)
    return {"requests": len(requests), "p50_s": float(np.percentile(lat, 50)),
            "p99_s": float(np.percentile(lat, 99)), "mean_s": float(lat.mean()),
            "makespan_s": float(span), "iter_per_s": iters / span}
