"""Serving loop: LL tests as requests, continuous batching on one GPU.

A request is (exponent p, FFT length n, iterations k); the reply is Res64 of
s_k.  Requests are admitted FIFO as they arrive while the device-memory
budget allows (each request's footprint is what its context allocates,
ll_context_bytes, plus its device checkpoint; 150 GB by default).  Contexts
are created off the scheduling loop by a worker thread, so an admission
never stalls the requests already running.  Every admitted request has its
own context and stream, and the loop keeps all of them busy: whenever a
request's chunk of iterations has finished on the GPU it reads that chunk's
roundoff maximum, keeps the chunk's final state as a device-resident
checkpoint and enqueues the next chunk.  Requests that arrive while others
run therefore join the work on the device at once.

A chunk whose roundoff error exceeds the limit is run again from the device
checkpoint (the reference's "restart from the last checkpoint to see if the
error is repeatable", CUDALucas.cu:3043-3060); if it exceeds the limit again
the request fails with that error.

The engine is pluggable: `GpuEngine` drives libllb200 through the C ABI;
tests drive the same scheduler with a CPU fake.
"""
import time
from concurrent.futures import ThreadPoolExecutor
from dataclasses import dataclass


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
    started: float = None
    finished: float = None
    res64: int = None
    max_err: float = 0.0
    retries: int = 0
    error: str = None

    @property
    def latency(self):
        return None if self.finished is None else self.finished - self.arrival


class GpuEngine:
    """Adapter from the scheduler to LLContext (one context per request)."""

    def __init__(self, device=0):
        self.device = device

    def footprint(self, req):
        from .engine import context_bytes
        return context_bytes(req.p, req.n) + 4 * req.n

    def open(self, req):
        from .engine import LLContext
        c = LLContext(req.p, req.n, device=self.device)
        c.start(req.offset)
        c.device_checkpoint()
        return c

    def enqueue(self, h, iters):
        h.step(iters, report=True, wait=False)   # enqueues only; the last iteration reports

    def busy(self, h):
        return h.busy()

    def check(self, h):
        return h.step(0, errchk=True)            # max roundoff error since the last check

    def commit(self, h):
        h.device_checkpoint()

    def restore(self, h):
        h.device_restore()

    def result(self, h):
        return h.res64()

    def close(self, h):
        h.close()


class Server:
    def __init__(self, engine, hbm_cap=150e9, chunk=1000, max_active=128, error_limit=0.35, creators=1,
                 clock=time.perf_counter):
        self.engine = engine
        self.hbm_cap = hbm_cap
        self.chunk = chunk
        self.max_active = max_active
        self.error_limit = error_limit
        self.creators = creators
        self.clock = clock
        self.peak_bytes = 0
        self.peak_active = 0

    def run(self, requests, realtime=True):
        """Serves `requests` (arrival times relative to the start).  With
        realtime=False arrivals are not waited for (all are available at t=0
        in arrival order).  Returns the requests with results filled in."""
        pending = sorted(requests, key=lambda r: r.arrival)
        waiting = []                       # arrived, not yet admitted (FIFO)
        opening = []                       # admitted, context being created: (req, future, bytes)
        active = {}                        # rid -> [req, handle, done, chunk in flight, bytes]
        used = 0
        t0 = self.clock()
        i = 0
        pool = ThreadPoolExecutor(max_workers=self.creators)
        try:
            while i < len(pending) or waiting or opening or active:
                now = self.clock() - t0
                while i < len(pending) and (pending[i].arrival <= now or not realtime):
                    waiting.append(pending[i])
                    i += 1
                # admission: FIFO while the device-memory budget and slots allow
                while waiting and len(active) + len(opening) < self.max_active:
                    need = self.engine.footprint(waiting[0])
                    if used + need > self.hbm_cap:
                        if not active and not opening:
                            raise RuntimeError("request %d does not fit the device budget" % waiting[0].rid)
                        break
                    r = waiting.pop(0)
                    r.admitted = self.clock() - t0
                    used += need
                    opening.append((r, pool.submit(self.engine.open, r), need))
                self.peak_bytes = max(self.peak_bytes, used)
                progressed = False
                # contexts created by the worker become active
                for item in list(opening):
                    r, fut, need = item
                    if fut.done():
                        opening.remove(item)
                        active[r.rid] = [r, fut.result(), 0, 0, need]
                        r.started = self.clock() - t0
                        progressed = True
                self.peak_active = max(self.peak_active, len(active))
                # keep every active request busy; retire the finished ones
                for rid in list(active):
                    r, h, done, inflight, need = active[rid]
                    if inflight and self.engine.busy(h):
                        continue
                    progressed = True
                    if inflight:
                        err = self.engine.check(h)
                        if err is not None and err > self.error_limit:
                            if r.retries == 0:
                                r.retries += 1            # run the chunk again from the checkpoint
                                self.engine.restore(h)
                                self.engine.enqueue(h, inflight)
                                continue
                            r.error = "roundoff error %.5f > %.5f" % (err, self.error_limit)
                        else:
                            r.max_err = max(r.max_err, err or 0.0)
                            done += inflight
                            r.retries = 0
                        if r.error is None and done < r.iters:
                            self.engine.commit(h)
                        inflight = 0
                    if r.error is None and done < r.iters:
                        k = min(self.chunk, r.iters - done)
                        self.engine.enqueue(h, k)
                        active[rid][2:4] = [done, k]
                        continue
                    if r.error is None:
                        r.res64 = self.engine.result(h)
                    r.finished = self.clock() - t0
                    self.engine.close(h)
                    used -= need
                    del active[rid]
                if not progressed:
                    time.sleep(0.0002)
        finally:
            pool.shutdown(wait=True)
        return requests


def serve_serial(engine, requests, realtime=True, clock=time.perf_counter):
    """Baseline: the same requests one at a time, in arrival order."""
    t0 = clock()
    for r in sorted(requests, key=lambda r: r.arrival):
        now = clock() - t0
        if realtime and r.arrival > now:
            time.sleep(r.arrival - now)
        r.admitted = r.started = clock() - t0
        h = engine.open(r)
        if r.iters:
            engine.enqueue(h, r.iters)
        while engine.busy(h):
            time.sleep(0.0002)
        r.max_err = engine.check(h) or 0.0
        r.res64 = engine.result(h)
        r.finished = clock() - t0
        engine.close(h)
    return requests


def summary(requests):
    import numpy as np
    done = [r for r in requests if r.finished is not None and r.error is None]
    lat = np.array([r.latency for r in done])
    span = max(r.finished for r in done) - min(r.arrival for r in done)
    iters = sum(r.iters for r in done)
    return {"requests": len(done), "failed": len(requests) - len(done),
            "p50_s": float(np.percentile(lat, 50)), "p99_s": float(np.percentile(lat, 99)),
            "mean_s": float(lat.mean()), "makespan_s": float(span), "iter_per_s": iters / span}
