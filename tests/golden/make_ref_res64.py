"""Generates the reference-binary fixtures tests/golden/ref_c{1,2,3}_res64.json.

Each fixture holds the Res64 values that CUDALucas v2.06 itself prints on its
report lines (CUDALucas.cu:2996-3002), run on a B200 from the binary that
`make -C oracle ref` builds from the reference sources (oracle/_ref/CUDALucas,
cuFFT path).  The runs use a scratch directory with its own CUDALucas.ini, so
no fft.txt/threads.txt of an earlier run can change the FFT length:

  c1: CUDALucas -f 12K    -x 10000 216091      every 10000 to the end (prime)
  c2: CUDALucas -f 3200K  -x 10000 57885161    every 10000 to --c2-iters
  c3: CUDALucas -f 18432K -x 5000  332192831   every 5000 to --c3-iters

It also records the reference's kernel-only timing, `-cufftbench L L 20`
(CUDALucas.cu:2440-2500), for the three lengths.

Needs a GPU; writes to --out (default: this folder).  Example:
  python tests/golden/make_ref_res64.py --out /tmp/golden
"""
import argparse
import json
import os
import re
import signal
import subprocess
import sys
import tempfile
import time

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
EXE = os.path.join(ROOT, "oracle", "_ref", "CUDALucas")

INI = ("WorkFile=worktodo.txt\nResultsFile=results.txt\nSaveAllCheckpoints=0\nSaveFolder=savefiles\n"
       "DeviceNumber=0\nPrintDeviceInfo=0\nErrorIterations=100\nReportIterations=%d\n"
       "CheckpointIterations=100000000\nPolite=0\nPoliteValue=50\nBigCarry=0\nErrorReset=85\n"
       "Interactive=0\nRoundoffTest=0\nThreads=256 128\nOutputHInterval=0\nSleep=0\nSleepValue=0\n"
       "ErrorLimit=40\n")
REPORT = re.compile(r"Iteration (\d+) .*?0x([0-9a-f]{16}).*?error = ([0-9.]+).*?([0-9.]+) ms/iter")
FINAL = re.compile(r"M\( (\d+) \)([PC])(?:, 0x([0-9a-f]{16}))?")


def run_reference(args, every, stop_after, timeout):
    """Runs the binary, returns (report rows, final line match or None, log)."""
    work = tempfile.mkdtemp(prefix="llref_")
    with open(os.path.join(work, "CUDALucas.ini"), "w") as f:
        f.write(INI % every)
    p = subprocess.Popen([EXE] + args, cwd=work, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True,
                         start_new_session=True)
    rows, final, log = [], None, []
    t0 = time.time()
    try:
        for line in p.stdout:
            log.append(line.rstrip())
            m = REPORT.search(line)
            if m:
                rows.append((int(m.group(1)), "0x" + m.group(2), float(m.group(3)), float(m.group(4))))
                if stop_after and rows[-1][0] >= stop_after:
                    break
            f = FINAL.search(line)
            if f:
                final = f
                break
            if time.time() - t0 > timeout:
                break
    finally:
        if p.poll() is None:
            os.killpg(p.pid, signal.SIGINT)
            try:
                p.wait(timeout=60)
            except subprocess.TimeoutExpired:
                os.killpg(p.pid, signal.SIGKILL)
    return rows, final, log


def fixture(name, q, n, every, stop_after, timeout):
    args = ["-d", "0", "-f", "%dK" % (n // 1024), "-x", str(every), str(q)]
    rows, final, log = run_reference(args, every, stop_after, timeout)
    if not rows:
        raise SystemExit("%s: no report lines; tail: %s" % (name, " | ".join(log[-5:])))
    out = {
        "generator": "reference binary (oracle/_ref/CUDALucas, CUDALucas v2.06 built for sm_100a with cuFFT) "
                     "on a B200: CUDALucas %s; Res64 values from its report lines "
                     "(tests/golden/make_ref_res64.py)" % " ".join(args),
        "exponent": q,
        "fft_words": n,
        "entries": [[q, k, r] for k, r, _, _ in rows],
        "max_roundoff_error": max(e for _, _, e, _ in rows),
        "ms_per_iter": [t for _, _, _, t in rows],
    }
    if final:
        out["final"] = {"line": final.group(0), "prime": final.group(2) == "P", "iterations": q - 2}
    return out


def cufftbench(lengths_k):
    """The reference's kernel-only timing (cuFFT x2 + square + rcb + splice,
    50 iterations per pass, CUDALucas.cu:2445-2490)."""
    res = {}
    for lk in lengths_k:
        work = tempfile.mkdtemp(prefix="llbench_")
        with open(os.path.join(work, "CUDALucas.ini"), "w") as f:
            f.write(INI % 10000)
        r = subprocess.run([EXE, "-d", "0", "-cufftbench", str(lk), str(lk), "20"], cwd=work, capture_output=True,
                           text=True, timeout=600)
        m = re.search(r"fft size = (\d+)K, ave time = ([0-9.]+) msec", r.stdout)
        res["%dK" % lk] = float(m.group(2)) if m else None
    return res


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=HERE)
    ap.add_argument("--only", default="c1,c2,c3,bench")
    ap.add_argument("--c2-iters", type=int, default=250000)
    ap.add_argument("--c3-iters", type=int, default=25000)
    a = ap.parse_args()
    os.makedirs(a.out, exist_ok=True)
    todo = a.only.split(",")
    jobs = {
        "c1": ("ref_c1_res64.json", 216091, 12288, 10000, 0, 600),
        "c2": ("ref_c2_res64.json", 57885161, 3276800, 10000, a.c2_iters, 900),
        "c3": ("ref_c3_res64.json", 332192831, 18874368, 5000, a.c3_iters, 900),
    }
    for key in ("c1", "c2", "c3"):
        if key in todo:
            fn, q, n, every, stop, tmo = jobs[key]
            d = fixture(key, q, n, every, stop, tmo)
            with open(os.path.join(a.out, fn), "w") as f:
                json.dump(d, f, indent=1)
            print(key, len(d["entries"]), "entries", d.get("final", ""), flush=True)
    if "bench" in todo:
        b = cufftbench([12, 3200, 18432])
        with open(os.path.join(a.out, "ref_cufftbench.json"), "w") as f:
            json.dump({"generator": "CUDALucas -cufftbench L L 20 (tests/golden/make_ref_res64.py)",
                       "unit": "ms/iter", "ave_time": b}, f, indent=1)
        print("cufftbench", b, flush=True)


if __name__ == "__main__":
    sys.exit(main())
