"""Benchmark: ms per Lucas-Lehmer iteration at the 3200K FFT (p = 57885161).

One step = S LL iterations (default 10000, the reference's report interval)
of one exponent, through the engine's C ABI.  With --gpus N (one process per
GPU under torch.distributed.run) every rank runs its own independent test
(replicas: LL iterations do not shard), the time is the max over ranks and
`value` is that time divided by the iterations of all ranks.

--impl reference runs the reference itself, CUDALucas v2.06 built from its
sources for sm_100a (oracle/_ref/CUDALucas, cuFFT), on the same GPU and the
same exponent and FFT length, and reports its own printed ms/iter.
"""
import argparse
import json
import os
import re
import signal
import statistics
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOADS = {
    # name: (exponent, FFT length in words, description)
    "3200K": (57885161, 3276800, "p=57885161 at 3200K (3276800 FP64 words, 17.665 bits/word)"),
    "12K": (216091, 12288, "p=216091 at 12K (12288 FP64 words, 17.586 bits/word)"),
    "18432K": (332192831, 18874368, "p=332192831 at 18432K (18874368 FP64 words, 17.600 bits/word)"),
}
METRIC = "ms/LL iter at 3.2M FFT vs ref cuFFT"


def peaks():
    try:
        d = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def ncu_traffic(workload):
    """Per-launch DRAM bytes of the dominant kernel from the committed ncu
    summary (profiles/traffic.json), or None."""
    try:
        d = json.load(open(os.path.join(ROOT, "profiles", "traffic.json")))
        return d.get(workload)
    except Exception:
        return None


class Clocks:
    """Samples SM clocks and throttle reasons with nvidia-smi while running."""

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index),
                 "--query-gpu=clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
                 "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                 "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 8:
                continue
            try:
                sm.append(float(f[0]))
                mx = float(f[1])
            except ValueError:
                continue
            for nm, v in zip(names, f[4:8]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def dist_init(backend="nccl"):
    """One process per GPU (torchrun's RANK/LOCAL_RANK/WORLD_SIZE); NCCL on
    GPUs, gloo for the CPU tests of this plumbing.  Every rank runs its own
    exponent (replicas); the group carries only the max-over-ranks of the
    timings and the Res64 verdicts."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        if backend == "nccl":
            torch.cuda.set_device(local)
            dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                    device_id=torch.device("cuda", local))
        else:
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=60))
    return world, rank, local


def allreduce_max(x, world):
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(x)], device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def cpu_baseline(q, n, iters1, iters_all):
    """The oracle (plain C IBDWT restatement) timed on this machine's host
    cores on a bounded sample of the same workload: one thread, then all the
    cores this process may use (POSIX threads over the independent
    butterflies, pairs and carry blocks)."""
    from oracle.binding import Oracle, set_threads
    cores = len(os.sched_getaffinity(0))

    def timed(threads, iters):
        set_threads(threads)
        o = Oracle(q, n)
        o.start(0)
        o.step(1)
        t = time.perf_counter()
        o.step(iters)
        return (time.perf_counter() - t) * 1000.0 / iters

    ms1 = timed(1, iters1)
    msn = timed(cores, iters_all)
    set_threads(1)
    return {"value": round(msn, 3), "unit": "ms/iter", "cores": cores, "kind": "port",
            "sample": "%d iterations of p=%d at n=%d from s0=4 (oracle/ibdwt_oracle.c, mixed-radix C FFT, "
                      "%d POSIX threads)" % (iters_all, q, n, cores),
            "single_core": {"value": round(ms1, 3), "unit": "ms/iter", "cores": 1,
                            "sample": "%d iterations, 1 thread" % iters1}}


def reference_res64(q, n):
    """{iteration: Res64} printed by the reference binary itself for this
    exponent and length (committed fixtures tests/golden/ref_*_res64.json)."""
    out = {}
    gdir = os.path.join(ROOT, "tests", "golden")
    for name in sorted(os.listdir(gdir)):
        if name.startswith("ref_") and name.endswith("_res64.json"):
            d = json.load(open(os.path.join(gdir, name)))
            if d.get("exponent") == q and d.get("fft_words") == n:
                out.update({int(k): int(r, 16) for _, k, r in d["entries"]})
    return out


def run_ours(args, world, rank, local):
    import numpy as np
    import torch
    import cudalucas_b200 as cl

    q, n, desc = WORKLOADS[args.workload]
    S, K, W = args.iters_per_step, args.steps, args.warmup
    torch.cuda.set_device(local)
    ctx = cl.LLContext(q, n, device=local)
    ctx.start((rank * 7919) % q)
    ext = torch.cuda.ExternalStream(ctx.stream, device=torch.device("cuda", local))
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device="cuda")  # > 126 MB L2
    want = reference_res64(q, n)
    got = {}
    done = 0

    def check_step():
        # the step's last iteration wrote the digits (LL_REPORT): Res64 of
        # the state after `done` iterations, read after the step's events
        d, off = ctx.read_digits()
        got[done] = cl.digits_res64(d, q, n, off)

    # every step, warm-up and timed, is S iterations whose last one reports
    for _ in range(W):
        ctx.step(S, report=True, wait=False)
        done += S
        check_step()

    # -- device-timed region: K steps of S iterations, L2 flushed between steps
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(K)]
    barrier(world)
    torch.cuda.synchronize()
    with Clocks(local) as clk:
        for i in range(K):
            with torch.cuda.stream(ext):
                flush.zero_()
                evs[i][0].record(ext)
            ctx.step(S, report=True, wait=False)
            evs[i][1].record(ext)
            done += S
            check_step()
        ctx.sync()
        torch.cuda.synchronize()
    barrier(world)
    step_ms = [a.elapsed_time(b) for a, b in evs]
    total_ms = allreduce_max(sum(step_ms), world)
    maxerr = ctx.step(0, errchk=True)  # max over every iteration so far
    d_last, off_last = ctx.read_digits()
    it_last = done

    # -- per-pass timing on real iterations (roofline of the dominant kernel)
    R = 200
    ev = [[torch.cuda.Event(enable_timing=True) for _ in range(3)] for _ in range(R)]
    for i in range(R):
        ev[i][0].record(ext)
        ctx.debug_launch(0)
        ev[i][1].record(ext)
        ctx.debug_launch(1)
        ev[i][2].record(ext)
    ctx.sync()
    torch.cuda.synchronize()
    t_tall = sum(e[0].elapsed_time(e[1]) for e in ev) / R
    t_wide = sum(e[1].elapsed_time(e[2]) for e in ev) / R

    # -- end to end through the public API with host buffers (pinned):
    # load digits (H2D), S iterations, read digits (D2H), Res64 on the host;
    # every repetition continues from the state after the timed steps
    pinned_in = torch.from_numpy(d_last).pin_memory()
    pinned_out = torch.empty(n, dtype=torch.int32).pin_memory()
    import ctypes
    from cudalucas_b200 import native
    L = native.lib()
    pin_in = ctypes.cast(pinned_in.data_ptr(), ctypes.POINTER(ctypes.c_int32))
    pin_out = ctypes.cast(pinned_out.data_ptr(), ctypes.POINTER(ctypes.c_int32))
    offv = ctypes.c_uint32()
    errv = ctypes.c_float()
    E = max(1, min(K, 3))
    e2e_res = []
    barrier(world)
    t0 = time.perf_counter()
    for _ in range(E):
        assert L.ll_load_digits(ctx._h, pin_in, off_last) == 0
        assert L.ll_step(ctx._h, S, 1, ctypes.byref(errv)) == 0
        assert L.ll_read_digits(ctx._h, pin_out, ctypes.byref(offv)) == 0
        e2e_res.append(L.ll_digits_res64(pin_out, q, n, offv.value))
    e2e_ms = (time.perf_counter() - t0) * 1000.0
    e2e_ms = allreduce_max(e2e_ms, world)
    got_e2e = e2e_res[0]
    shape = ctx.shape
    ctx.close()

    # -- parity: Res64 after every step against the reference binary's own
    # report lines for this exponent and length (rank 0 starts at offset 0,
    # the others at other offsets; Res64 does not depend on the offset)
    checked = {k: v for k, v in got.items() if k in want}
    mismatched = sorted(k for k, v in checked.items() if want[k] != v)
    e2e_consistent = len(set(e2e_res)) == 1
    e2e_checked = (it_last + S) in want
    if e2e_checked and want[it_last + S] != got_e2e:
        mismatched.append(it_last + S)
    ok = not mismatched and e2e_consistent
    ok_all = allreduce_max(0.0 if ok else 1.0, world) == 0.0

    if rank != 0:
        return None if ok_all else {"fail": True}
    hbm, peak_kind = peaks()
    alg_bytes = 16.0 * n  # one read + one write of n FP64 words per pass
    if shape.get("cluster"):
        # one cluster-resident launch per step: the state lives in the
        # cluster's shared memory, so no pass touches HBM; the figure is the
        # array bytes of both passes per iteration over the iteration time
        t_iter = total_ms / (K * S)
        roof = {"bound": "hbm", "kernel": "cluster_iters", "achieved": round(2 * alg_bytes / (t_iter * 1e-3) / 1e9, 1),
                "peak": hbm, "peak_kind": peak_kind, "unit": "GB/s",
                "frac": round(2 * alg_bytes / (t_iter * 1e-3) / 1e9 / hbm, 4), "traffic": None,
                "alg_bytes_per_iteration": 2 * alg_bytes, "iteration_us": round(t_iter * 1000, 3),
                "note": "latency bound: the state stays in the shared memory of one thread-block cluster, "
                        "three cluster barriers per iteration; HBM is read once per launch",
                "two_launch_us": {"tall": round(t_tall * 1000, 2), "wide": round(t_wide * 1000, 2)}}
        launches = K * -(-S // 65536)
    else:
        dom, t_dom = ("wide", t_wide) if t_wide >= t_tall else ("tall", t_tall)
        achieved = alg_bytes / (t_dom * 1e-3) / 1e9
        roof = {"bound": "hbm", "kernel": dom + "_kernel", "achieved": round(achieved, 1),
                "peak": hbm, "peak_kind": peak_kind, "unit": "GB/s", "frac": round(achieved / hbm, 4),
                "traffic": ncu_traffic(args.workload), "alg_bytes_per_launch": alg_bytes,
                "launch_us": {"tall": round(t_tall * 1000, 2), "wide": round(t_wide * 1000, 2)}}
        launches = 2 * K * S
    state_mb = 8.0 * n / 1e6
    out = {
        "metric": METRIC,
        "value": round(total_ms / (K * S * world), 6),
        "unit": "ms/iter",
        "n_gpus": world,
        "steps": K,
        "warmup": W,
        "ms_per_step": round(total_ms / K, 4),
        "higher_is_better": False,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic: LL test from s0=4 (no dataset)",
        "config": {"workload": desc, "exponent": q, "fft_words": n, "iters_per_step": S,
                   "per_gpu_ms_per_iter": round(total_ms / (K * S), 6),
                   "shape": shape, "max_roundoff_error": round(maxerr, 6),
                   "bits_per_word": round(q / n, 4),
                   "l2": ("flushed (256 MB write) before each timed step; the %.3g MB state stays "
                          "L2-resident inside a step, as it does for the reference" % state_mb) if state_mb < 63 else
                         ("flushed (256 MB write) before each timed step; the %.3g MB state is larger than "
                          "L2 (126 MB), each pass streams it from HBM" % state_mb),
                   "parallelism": "replicas (one independent exponent per GPU)"},
        "res64_ok": ok_all,
        "res64": {str(k): "%016x" % v for k, v in sorted(got.items())},
        "res64_checked": {"against": "Res64 printed by the reference binary (tests/golden/ref_*_res64.json)",
                          "iterations": sorted(checked) + ([it_last + S] if e2e_checked else []),
                          "mismatched": mismatched, "e2e_repetitions_agree": e2e_consistent},
        "e2e": {"value": round(e2e_ms / (E * S * world), 6) * world, "unit": "ms/iter",
                "h2d_bytes_per_step": 4 * n + 32, "d2h_bytes_per_step": 4 * n + 32,
                "steps": E, "res64": "%016x" % got_e2e, "iteration": it_last + S,
                "path": "ll_load_digits -> ll_step(LL_REPORT) -> ll_read_digits -> ll_digits_res64"},
        "roofline": roof,
        "clocks": clk.summary(),
        "gpu_launches": launches,
    }
    if args.cpu_iters > 0:
        out["cpu_baseline"] = cpu_baseline(q, n, args.cpu_iters, args.cpu_iters_all)
    return out


def run_reference(args, world, rank, local):
    """CUDALucas itself (oracle/_ref/CUDALucas) on this GPU: same exponent,
    forced FFT length, report every S iterations; its printed wall-clock
    ms/iter over W warm-up and K timed report intervals."""
    if rank != 0:
        return None
    q, n, desc = WORKLOADS[args.workload]
    S, K, W = args.iters_per_step, args.steps, args.warmup
    exe = os.path.join(ROOT, "oracle", "_ref", "CUDALucas")
    base = {"impl": "reference", "metric": METRIC, "unit": "ms/iter", "n_gpus": world, "steps": K,
            "warmup": W, "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic: LL test from s0=4 (no dataset)"}
    if not os.path.exists(exe):
        base["unavailable"] = "reference binary oracle/_ref/CUDALucas not built (make -C oracle ref)"
        return base
    work = tempfile.mkdtemp(prefix="cudalucas_ref_")
    with open(os.path.join(work, "CUDALucas.ini"), "w") as f:
        f.write("WorkFile=worktodo.txt\nResultsFile=results.txt\nSaveAllCheckpoints=0\n"
                "SaveFolder=savefiles\nDeviceNumber=%d\nPrintDeviceInfo=0\nErrorIterations=100\n"
                "ReportIterations=%d\nCheckpointIterations=%d\nPolite=0\nPoliteValue=50\nBigCarry=0\n"
                "ErrorReset=85\nInteractive=0\nRoundoffTest=0\nThreads=256 128\nOutputHInterval=0\n"
                "Sleep=0\nSleepValue=0\nErrorLimit=40\n" % (local, S, 100 * S * (W + K + 2)))
    cmd = [exe, "-d", str(local), "-f", "%dK" % (n // 1024), "-x", str(S), str(q)]
    rx = re.compile(r"Iteration (\d+) .*?0x([0-9a-f]{16}).*?error = ([0-9.]+).*?([0-9.]+) ms/iter")
    rows = []
    t0 = time.perf_counter()
    p = subprocess.Popen(cmd, cwd=work, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True,
                         start_new_session=True)
    log = []
    try:
        for line in p.stdout:
            log.append(line.rstrip())
            m = rx.search(line)
            if m:
                rows.append((int(m.group(1)), m.group(2), float(m.group(3)), float(m.group(4))))
                if len(rows) >= W + K:
                    break
            if time.perf_counter() - t0 > 900:
                break
    finally:
        try:
            os.killpg(p.pid, signal.SIGINT)
            p.wait(timeout=60)
        except Exception:
            os.killpg(p.pid, signal.SIGKILL)
    if len(rows) < W + K:
        base["unavailable"] = "reference produced %d report lines; tail: %s" % (len(rows), " | ".join(log[-3:]))
        return base
    timed = rows[W:W + K]
    ms = statistics.mean(r[3] for r in timed)
    base.update({
        "value": round(ms, 6),
        "ms_per_step": round(ms * S, 4),
        "config": {"workload": desc, "exponent": q, "fft_words": n, "iters_per_step": S,
                   "command": " ".join(cmd[1:]), "res64": {str(r[0]): r[1] for r in rows},
                   "max_roundoff_error": max(r[2] for r in timed),
                   "timing": "CUDALucas's own wall-clock ms/iter per report interval (includes its "
                             "blocking error read-back every 100 iterations, CUDALucas.cu:2936)"},
        "e2e": {"value": round(ms, 6), "unit": "ms/iter", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "reference_run": {"value": round(ms, 6), "unit": "ms/iter", "kind": "reference", "device": "gpu",
                          "host_threads": 1,
                          "sample": "%d report intervals of %d iterations of the reference binary, a GPU "
                                    "program (cuFFT path on GPU %d); it has no host-core implementation"
                                    % (K, S, local)},
    })
    # the reference's kernel-only timing of the same length (-cufftbench,
    # CUDALucas.cu:2445-2490: cuFFT x2 + square + rcb + splice, no read-back)
    try:
        r = subprocess.run([exe, "-d", str(local), "-cufftbench", str(n // 1024), str(n // 1024), "20"], cwd=work,
                           capture_output=True, text=True, timeout=300)
        m = re.search(r"ave time = ([0-9.]+) msec", r.stdout)
        base["kernel_only"] = {"value": float(m.group(1)) if m else None, "unit": "ms/iter",
                               "command": "-cufftbench %d %d 20" % (n // 1024, n // 1024)}
    except Exception as exc:
        base["kernel_only"] = {"value": None, "error": str(exc)[:200]}
    return base


def run_batch(args, world, rank, local):
    """Batched mode: 256 primes log-uniform in [1e6, 2e7] (seed 7) at the
    length policy's FFT lengths, all advancing together (one CUDA graph per
    step), against the same exponents run one at a time over the same
    iterations.  The first step of the batch (S iterations, reported) is
    compared member by member with the solo runs."""
    import torch
    import cudalucas_b200 as cl
    from cudalucas_b200 import workloads
    torch.cuda.set_device(local)
    members = workloads.batch_exponents(args.batch_count, seed=7 + rank)
    qs, ns = zip(*members)
    offs = [(q * 7) // 11 for q in qs]
    S, K, W = args.iters_per_step, args.steps, args.warmup
    by_length = not args.batch_per_member
    b = cl.LLBatch(qs, ns, device=local, graph_iters=args.batch_graph_iters, by_length=by_length)
    classes = b.classes
    b.start(offs)
    b.step(S, report=True)           # the first warm-up step, checked against solo runs below
    res_batch = b.res64()
    for _ in range(W - 1):
        b.step(S)
    b.sync()
    ext = torch.cuda.ExternalStream(b.stream, device=torch.device("cuda", local))
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier(world)
    torch.cuda.synchronize()
    with Clocks(local) as clk:
        t0.record(ext)
        for _ in range(K):
            b.step(S)
        t1.record(ext)
        b.sync()
    ms = allreduce_max(t0.elapsed_time(t1), world)
    errs = b.step(1, report=True)
    b.close()
    other = None
    if args.batch_compare:
        # the other launch mode over the same members and steps
        b2 = cl.LLBatch(qs, ns, device=local, graph_iters=args.batch_graph_iters, by_length=not by_length)
        b2.start(offs)
        for _ in range(W):
            b2.step(S)
        b2.sync()
        ext2 = torch.cuda.ExternalStream(b2.stream, device=torch.device("cuda", local))
        u0, u1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        u0.record(ext2)
        for _ in range(K):
            b2.step(S)
        u1.record(ext2)
        b2.sync()
        b2.close()
        other = len(members) * K * S * world / (allreduce_max(u0.elapsed_time(u1), world) / 1000.0)
    # the same exponents one at a time, each the same S iterations from the
    # same offset: the serial baseline, and Res64 equal to the batch's
    Ss = args.serial_iters or S
    serial_ms = 0.0
    mismatched = []
    for (q, n), off, rb in zip(members, offs, res_batch):
        c = cl.LLContext(q, n, device=local)
        c.start(off)
        ext1 = torch.cuda.ExternalStream(c.stream, device=torch.device("cuda", local))
        a0, a1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a0.record(ext1)
        c.step(Ss, report=True, wait=False)
        a1.record(ext1)
        c.sync()
        serial_ms += a0.elapsed_time(a1)
        if Ss == S and c.res64() != rb:
            mismatched.append(q)
        c.close()
    serial_ms = allreduce_max(serial_ms, world)
    if rank != 0:
        return None
    batch_ips = len(members) * K * S * world / (ms / 1000.0)
    serial_ips = len(members) * Ss * world / (serial_ms / 1000.0)
    return {
        "metric": "batched LL iter/s (256 exponents, seed 7, 1e6..2e7)",
        "value": round(batch_ips, 1), "unit": "iter/s", "n_gpus": world, "steps": K, "warmup": W,
        "ms_per_step": round(ms / K, 3), "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic: seeded exponents, LL tests from s0=4",
        "config": {"workload": "batch: %d primes log-uniform in [1e6, 2e7] (seed 7), lengths %dK..%dK"
                               % (len(members), min(ns) // 1024, max(ns) // 1024),
                   "iters_per_step": S, "graph_iters": args.batch_graph_iters,
                   "launches": "one per pass per length class (%d classes)" % classes if by_length
                               else "one per pass per member",
                   "serial_iter_s": round(serial_ips, 1), "speedup_vs_serial": round(batch_ips / serial_ips, 3),
                   "serial_sample": "%d iterations of each exponent alone, from the batch's offsets" % Ss,
                   "other_launch_mode_iter_s": None if other is None else round(other, 1),
                   "max_roundoff_error": round(float(max(errs)), 5)},
        "res64_ok": Ss == S and not mismatched,
        "res64_checked": {"against": "each member run alone for the same %d iterations" % S,
                          "members": len(members) if Ss == S else 0, "mismatched": mismatched},
        "clocks": clk.summary(),
        "gpu_launches": 2 * (classes if by_length else len(members)) * K * S,
    }


def run_serve(args, world, rank, local):
    """Serving: Poisson arrivals at 50/s of LL requests (prime p log-uniform
    in [1e5, 5e7], k uniform in [1e3, 5e4], seed 11), continuous batching,
    against the same requests served one at a time in arrival order."""
    import torch
    from cudalucas_b200 import serve, workloads
    torch.cuda.set_device(local)
    reqs = workloads.serve_requests(args.serve_count, seed=11 + rank)

    def mk():
        return [serve.Request(rid=i, arrival=t, p=p, n=n, iters=k, offset=i) for i, (t, p, n, k) in enumerate(reqs)]
    eng = serve.GpuEngine(device=local)
    warm = mk()[:2]
    for r in warm:
        r.iters = 50
    serve.Server(eng).run(warm, realtime=False)
    barrier(world)
    srv = serve.Server(eng, chunk=args.serve_chunk, hbm_cap=args.serve_hbm_gb * 1e9)
    with Clocks(local) as clk:
        batched = srv.run(mk())
    serial = serve.serve_serial(eng, mk())
    same = all(a.res64 == b.res64 and a.error is None for a, b in zip(batched, serial))
    sb, ss = serve.summary(batched), serve.summary(serial)
    if rank != 0:
        return None
    return {
        "metric": "serve p50/p99 time-to-residue (s), Poisson 50 req/s",
        "value": round(sb["p50_s"], 4), "unit": "s", "n_gpus": world, "steps": 1, "warmup": 1,
        "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic: seeded Poisson arrivals of LL requests",
        "config": {"workload": "serve: %d requests, Poisson 50/s, p log-uniform [1e5, 5e7], k uniform [1e3, 5e4], "
                               "seed 11" % len(reqs), "chunk_iters": args.serve_chunk,
                   "hbm_cap_bytes": srv.hbm_cap, "peak_device_bytes": srv.peak_bytes,
                   "peak_active_requests": srv.peak_active,
                   "continuous": sb, "serial": ss, "results_identical": same,
                   "speedup_p50": round(ss["p50_s"] / sb["p50_s"], 3),
                   "speedup_throughput": round(sb["iter_per_s"] / ss["iter_per_s"], 3)},
        "p99": round(sb["p99_s"], 4),
        "res64_ok": same,
        "clocks": clk.summary(),
    }


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="3200K", choices=sorted(WORKLOADS) + ["batch", "serve"])
    ap.add_argument("--serve-count", type=int, default=32)
    ap.add_argument("--serve-chunk", type=int, default=1000)
    ap.add_argument("--batch-count", type=int, default=256)
    ap.add_argument("--batch-graph-iters", type=int, default=10,
                    help="iterations of every member per CUDA graph in the batch workload")
    ap.add_argument("--serial-iters", type=int, default=0,
                    help="iterations of each exponent alone in the batch workload's serial leg (0: the step size)")
    ap.add_argument("--serve-hbm-gb", type=float, default=150.0)
    ap.add_argument("--batch-compare", action="store_true",
                    help="also time the other launch mode (per member / per length class)")
    ap.add_argument("--batch-per-member", action="store_true",
                    help="launch each member's passes on their own instead of once per length class")
    ap.add_argument("--iters-per-step", type=int, default=10000)
    ap.add_argument("--cpu-iters", type=int, default=20,
                    help="oracle iterations on one host thread for cpu_baseline (0: skip)")
    ap.add_argument("--cpu-iters-all", type=int, default=100,
                    help="oracle iterations on all host cores for cpu_baseline")
    args = ap.parse_args()
    world, rank, local = dist_init()
    if args.workload == "serve":
        out = run_serve(args, world, rank, local) if args.impl == "ours" else (
            {"impl": "reference", "unavailable": "the reference has no serving mode"} if rank == 0 else None)
    elif args.workload == "batch":
        out = run_batch(args, world, rank, local) if args.impl == "ours" else (
            {"impl": "reference", "unavailable": "the reference has no batched mode"} if rank == 0 else None)
    elif args.impl == "reference":
        out = run_reference(args, world, rank, local)
    else:
        out = run_ours(args, world, rank, local)
    failed = out is not None and (out.get("fail") or out.get("res64_ok") is False)
    if out is not None and not out.get("fail"):
        print(json.dumps(out), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    if failed:
        sys.exit("Res64 differs from the reference binary's")


if __name__ == "__main__":
    main()
