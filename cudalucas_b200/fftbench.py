"""Times the engine per FFT length and launch shape: the engine's counterpart
of CUDALucas's -cufftbench / -threadbench modes (CUDALucas.cu:2413, :2144),
which time cuFFT and the reference kernels and write `<gpu> fft.txt` /
`<gpu> threads.txt`.  Here every launch choice of each length (row width W,
kernel variants; see candidate_shapes) is timed with CUDA events on the
context's stream, and the fastest is printed (and optionally written as a
tuning table).

  python -m cudalucas_b200.fftbench 3200K [18432K ...] [--iters 200]
         [--width W] [--rows G] [--kernels FLAGS] [--all-shapes] [--table FILE]

--kernels passes ll_tuning.kernels (LL_KERNELS_* flags, e.g. 8 = no
cluster-resident iterations).
"""
import argparse
import ctypes
import json
import sys
import time

from . import engine, native


def parse_len(s):
    s = s.strip().upper()
    if s.endswith("K"):
        return int(s[:-1]) * 1024
    if s.endswith("M"):
        return int(s[:-1]) * 1024 * 1024
    return int(s)


def is_prime(v):
    if v < 2:
        return False
    for p in (2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37):
        if v % p == 0:
            return v == p
    d, s = v - 1, 0
    while d % 2 == 0:
        d //= 2
        s += 1
    for a in (2, 3, 5, 7, 11, 13, 17):
        x = pow(a, d, v)
        if x in (1, v - 1):
            continue
        for _ in range(s - 1):
            x = x * x % v
            if x == v - 1:
                break
        else:
            return False
    return True


def exponent_for(n):
    """A prime exponent at ~17.6 bits per word inside the length's bounds."""
    q = int(n * 17.6) | 1
    while not is_prime(q):
        q += 2
    return q


def time_shape(q, n, iters, tuning=None, device=0):
    """Returns (ms/iter, tall us, wide us, max err, shape) for one shape."""
    import torch
    ctx = engine.LLContext(q, n, device=device, tuning=tuning)
    ctx.start(0)
    # warm-up long enough to capture the context's CUDA graph (64 iterations)
    # before the timed region
    ctx.step(130)
    ctx.sync()
    ext = torch.cuda.ExternalStream(ctx.stream)
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(ext)
    ctx.step(iters)
    b.record(ext)
    err = ctx.step(1, errchk=True)
    ms = a.elapsed_time(b) / iters
    ev = [[torch.cuda.Event(enable_timing=True) for _ in range(3)] for _ in range(20)]
    for e in ev:
        e[0].record(ext)
        ctx.debug_launch(0)
        e[1].record(ext)
        ctx.debug_launch(1)
        e[2].record(ext)
    ctx.sync()
    tall = sum(e[0].elapsed_time(e[1]) for e in ev) / len(ev) * 1000
    wide = sum(e[1].elapsed_time(e[2]) for e in ev) / len(ev) * 1000
    shape = ctx.shape
    ctx.close()
    return ms, tall, wide, err, shape


def candidate_shapes(n):
    """The launch choices the engine offers for length n: every row width W
    with the engine's own kernels for it (specialised where they exist, rows
    per CTA chosen by the engine), and for the default width the kernel
    variants (two launches instead of the cluster-resident step, the
    alternative row kernel).  Setting rows per CTA would force the generic
    kernels, so it is not a candidate."""
    N = n // 2
    out, seen = [], set()
    q = exponent_for(n)

    def add(t):
        try:
            c = engine.LLContext(q, n, tuning=t)
        except engine.LLError:
            return
        sh = c.shape
        c.close()
        key = (sh["W"], sh["G"], sh["threads_wide"], sh["threads_tall"], sh.get("cluster"))
        if key not in seen:
            seen.add(key)
            out.append((t, sh))

    add(None)
    add({"kernels": native.LL_KERNELS_NO_CLUSTER})
    add({"kernels": native.LL_KERNELS_ALT_WIDE})
    for w in range(16, 8193, 2):
        if N % w == 0:
            add({"width": w})
    return out


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("lengths", nargs="+")
    ap.add_argument("--exponent", type=int, default=0)
    ap.add_argument("--iters", type=int, default=200)
    ap.add_argument("--width", type=int, default=0)
    ap.add_argument("--rows", type=int, default=0)
    ap.add_argument("--kernels", type=int, default=0)
    ap.add_argument("--variant", type=int, default=0, help="cluster kernel variant (ll_tuning.cluster_variant)")
    ap.add_argument("--all-shapes", action="store_true")
    ap.add_argument("--table", default="")
    ap.add_argument("--device", type=int, default=0)
    args = ap.parse_args(argv)
    table = {}
    for s in args.lengths:
        n = parse_len(s)
        q = args.exponent or exponent_for(n)
        if args.all_shapes:
            shapes = [t for t, _ in candidate_shapes(n)]
        else:
            t = {}
            if args.width:
                t["width"] = args.width
            if args.rows:
                t["rows_per_cta"] = args.rows
            if args.kernels:
                t["kernels"] = args.kernels
            if args.variant:
                t["cluster_variant"] = args.variant
            shapes = [t or None]
        best = None
        for t in shapes:
            ms, tall, wide, err, shape = time_shape(q, n, args.iters, t, args.device)
            print("%8dK q=%d W=%d H=%d G=%d%s  %.4f ms/iter  tall %.1f us  wide %.1f us  err %.5f  tuning %s"
                  % (n // 1024, q, shape["W"], shape["H"], shape["G"], " cluster" if shape.get("cluster") else "",
                     ms, tall, wide, err, json.dumps(t or {}, separators=(",", ":"))), flush=True)
            if best is None or ms < best[0]:
                best = (ms, shape)
        table[n] = {"ms_per_iter": best[0], **best[1]}
    if args.table:
        with open(args.table, "w") as f:
            json.dump(table, f, indent=1)


if __name__ == "__main__":
    main()
