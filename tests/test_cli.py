"""CPU tests of the llucas command-line host: version/help, the worktodo
grammar of CUDALucas (parse.c:241-471: Test=/DoubleCheck=, optional AID and
FFT length, comments, validity rules of valid_assignment)."""
import os
import subprocess

import pytest

from cudalucas_b200 import build

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def cli():
    return build.build_cli()


def run(cli, *args, cwd=None):
    return subprocess.run([cli, *args], capture_output=True, text=True, cwd=cwd, timeout=60)


def test_version_and_help(cli):
    r = run(cli, "-v")
    assert r.returncode == 0 and "llucas" in r.stdout
    r = run(cli, "-h")
    assert r.returncode == 0 and "Usage" in r.stdout


def test_worktodo_grammar(cli, tmp_path):
    wt = tmp_path / "worktodo.txt"
    wt.write_text("Test=N/A,216091,12K\n# comment\n// also a comment\nDoubleCheck=ABCDEF0123,57885161\n"
                  "Test=86243\n\nTest=86244\nBogus=1\nTest=7001\nTest=AID,332192831,18432K # tail\n"
                  "test=132049,7K\n")
    r = run(cli, "-worktodo-check", str(wt))
    assert r.returncode == 0
    lines = r.stdout.strip().split("\n")
    assert lines[0] == "assignment exponent=216091 fft=12288 key=N/A valid=1"
    assert lines[1] == "assignment exponent=57885161 fft=0 key=ABCDEF0123 valid=1"
    assert lines[2] == "assignment exponent=86243 fft=0 key= valid=1"
    assert lines[3] == "assignment exponent=86244 fft=0 key= valid=-1"       # not prime
    assert lines[4] == "invalid"                                              # no Test=
    assert lines[5] == "assignment exponent=7001 fft=0 key= valid=0"         # below 7500
    assert lines[6] == "assignment exponent=332192831 fft=18874368 key=AID valid=1"
    assert lines[7] == "assignment exponent=132049 fft=7168 key= valid=1"


def test_unsupported_modes_fail_cleanly(cli):
    r = run(cli, "-memtest")
    assert r.returncode == 2 and "not provided" in r.stderr


# ---------------------------------------------------------------- GPU flows --
INI = ("WorkFile=worktodo.txt\nResultsFile=results.txt\nSaveAllCheckpoints=0\nSaveFolder=savefiles\n"
       "DeviceNumber=0\nErrorIterations=100\nReportIterations=10000\nCheckpointIterations=10000\n"
       "ErrorLimit=40\nErrorReset=85\n")


@pytest.mark.gpu
def test_cli_full_test_of_a_mersenne_prime(cli, tmp_path):
    (tmp_path / "CUDALucas.ini").write_text(INI)
    (tmp_path / "worktodo.txt").write_text("Test=N/A,86243,4K\nTest=86249\n")
    r = run(cli, "worktodo.txt", cwd=str(tmp_path))
    assert r.returncode == 0, r.stderr
    res = (tmp_path / "results.txt").read_text().strip().split("\n")
    assert res[0].startswith("M( 86243 )P, offset = ")
    assert res[1].startswith("M( 86249 )C, 0x")
    from oracle import exact
    assert res[1].split(",")[1].strip() == "0x%016x" % exact.res64(86249, 86247)
    assert (tmp_path / "worktodo.txt").read_text().strip() == ""
    assert "Iteration 10000 / 86243, 0x23992ccd735a03d9" in r.stdout


@pytest.mark.gpu
def test_cli_checkpoint_resume_and_file_format(cli, tmp_path):
    """Interrupt after the first checkpoint, check the c<q> file byte layout
    (packed residue + 10-word trailer + CRC), resume to completion."""
    import signal
    import time
    import numpy as np
    import cudalucas_b200 as cl
    from oracle import exact
    (tmp_path / "CUDALucas.ini").write_text(INI)
    q = 132049
    p = subprocess.Popen([cli, str(q)], cwd=str(tmp_path), stdout=subprocess.PIPE, stderr=subprocess.PIPE,
                         text=True)
    t0 = time.time()
    while not (tmp_path / ("c%d" % q)).exists() and time.time() - t0 < 60:
        time.sleep(0.01)
    p.send_signal(signal.SIGINT)
    out, err = p.communicate(timeout=120)
    assert p.returncode in (0, 1), err
    raw = np.fromfile(tmp_path / ("c%d" % q), dtype=np.uint32)
    end = (q + 31) // 32
    assert raw.size == end + 10
    assert raw[end] == q
    n, j, off = int(raw[end + 1]), int(raw[end + 2]), int(raw[end + 3])
    assert raw[end + 9] == cl.checkpoint_checksum(raw[: end + 9].tobytes())
    digits = cl.unpack_bits(raw[:end], q, n)
    assert cl.digits_res64(digits, q, n, off) == exact.res64(q, j - 1)
    r = run(cli, str(q), cwd=str(tmp_path))
    assert r.returncode == 0, r.stderr
    assert "Continuing M%d @ iteration %d" % (q, j) in r.stdout
    line = (tmp_path / "results.txt").read_text().strip().split("\n")[-1]
    final = exact.res64(q, q - 2)  # 132049 is a Mersenne prime exponent: residue 0
    if final == 0:
        assert line.startswith("M( %d )P, offset = " % q)
    else:
        assert line.startswith("M( %d )C, 0x%016x" % (q, final))


@pytest.mark.gpu
def test_cli_selftest(cli, tmp_path):
    r = run(cli, "-r", "0", cwd=str(tmp_path))
    assert r.returncode == 0, r.stdout[-2000:]
    assert r.stdout.count("This residue is correct.") == 20


# ------------------------------------------------- recovery and round-off --
def run_until(cmd, cwd, pattern, timeout=300, env=None):
    """Runs cmd, sends SIGINT once a stdout line contains `pattern`, and
    returns (returncode, stdout, stderr)."""
    import signal
    import threading
    p = subprocess.Popen(cmd, cwd=str(cwd), stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True,
                         env=env)
    out, err = [], []
    t = threading.Thread(target=lambda: err.extend(p.stderr), daemon=True)
    t.start()
    sent = False
    for line in p.stdout:
        out.append(line)
        if not sent and pattern in line:
            p.send_signal(signal.SIGINT)
            sent = True
    rc = p.wait(timeout=timeout)
    t.join(timeout=10)
    return rc, "".join(out), "".join(err)


def final_line(tmp_path):
    return (tmp_path / "results.txt").read_text().strip().split("\n")[-1]


@pytest.mark.gpu
def test_cli_roundoff_test_before_a_fresh_test(cli, tmp_path):
    """RoundoffTest=1: 1000 careful iterations with the error read after
    each one (CUDALucas.cu:2589-2648), then the test continues."""
    (tmp_path / "CUDALucas.ini").write_text(INI + "RoundoffTest=1\n")
    r = run(cli, "86243", cwd=str(tmp_path))
    assert r.returncode == 0, r.stderr
    assert "Running careful round off test for 1000 iterations." in r.stdout
    assert "<= 0.25 (max error = " in r.stdout and "continuing test." in r.stdout
    assert final_line(tmp_path).startswith("M( 86243 )P, offset = ")


@pytest.mark.gpu
def test_cli_injected_step_failure_restarts_from_last_report(cli, tmp_path):
    """A failed ll_step (injected on the host, no device fault) is handled as
    the reference handles a CUDA error in the LL loop (CUDALucas.cu:2938-2950):
    restart from the last good state; the result is unchanged."""
    (tmp_path / "CUDALucas.ini").write_text(INI)
    env = dict(os.environ, LLUCAS_INJECT_FAILURES="55000:2")
    r = subprocess.run([cli, "216091"], cwd=str(tmp_path), capture_output=True, text=True, timeout=300, env=env)
    assert r.returncode == 0, r.stderr
    assert r.stdout.count("Resetting device and restarting from last checkpoint.") == 2
    assert "injected failure" in r.stderr
    assert "Continuing M216091 @ iteration 50001" in r.stdout
    assert final_line(tmp_path).startswith("M( 216091 )P, offset = ")


@pytest.mark.gpu
def test_cli_roundoff_policy_retry_longer_fft_and_reset(cli, tmp_path):
    """ErrorLimit 1 (0.00875 at ErrorIterations 100): the 4K length's real
    roundoff for M86243 (21 bits per word) exceeds it, the 8K length's does
    not.  The policy of CUDALucas.cu:3043-3097 retries from the last
    checkpoint, moves to the next length until the next checkpoint, goes
    back ("Resettng fft.") and repeats; the test still completes."""
    (tmp_path / "CUDALucas.ini").write_text(INI.replace("ErrorLimit=40", "ErrorLimit=1"))
    r = run(cli, "-f", "4K", "86243", cwd=str(tmp_path))
    assert r.returncode == 0, r.stdout[-3000:] + r.stderr
    out = r.stdout
    assert "Round off error at iteration = " in out
    assert "Restarting from last checkpoint to see if the error is repeatable." in out
    assert "The error persists.\nTrying a larger fft until the next checkpoint." in out
    assert "Resettng fft." in out
    assert final_line(tmp_path).startswith("M( 86243 )P, offset = ")


@pytest.mark.gpu
def test_cli_roundoff_policy_gives_up(cli, tmp_path):
    """ErrorLimit 0: every length exceeds it, so after the retry and the
    longer length the policy gives up (CUDALucas.cu:3060-3064)."""
    (tmp_path / "CUDALucas.ini").write_text(INI.replace("ErrorLimit=40", "ErrorLimit=0"))
    r = run(cli, "-f", "4K", "86243", cwd=str(tmp_path))
    assert r.returncode == 2
    assert "The error won't go away. I give up." in r.stdout
    assert not (tmp_path / "results.txt").exists()


@pytest.mark.gpu
def test_cli_resume_at_another_length_and_from_the_backup(cli, tmp_path):
    """Checkpoints written at 12K resume at 14K (the packed residue does not
    depend on the length, CUDALucas.cu:1366-1372); a corrupt c<q> falls back
    to t<q>, the previous checkpoint (CUDALucas.cu:1765-1792)."""
    (tmp_path / "CUDALucas.ini").write_text(INI)
    q = 216091
    rc, out, err = run_until([cli, "-f", "12K", str(q)], tmp_path, "Iteration 30000 ")
    assert rc in (0, 1), err
    assert (tmp_path / ("c%d" % q)).exists() and (tmp_path / ("t%d" % q)).exists()
    raw = bytearray((tmp_path / ("c%d" % q)).read_bytes())
    raw[100] ^= 0xFF
    (tmp_path / ("c%d" % q)).write_bytes(bytes(raw))
    r = run(cli, "-f", "14K", str(q), cwd=str(tmp_path))
    assert r.returncode == 0, r.stderr
    assert "The checkpoint appears to be corrupt. Trying the backup file." in r.stderr
    assert "with fft length 14K" in r.stdout
    assert final_line(tmp_path).startswith("M( %d )P, offset = " % q)


REF = os.path.join(ROOT, "oracle", "_ref", "CUDALucas")
REF_INI = ("WorkFile=worktodo.txt\nResultsFile=results.txt\nSaveAllCheckpoints=0\nSaveFolder=savefiles\n"
           "DeviceNumber=0\nPrintDeviceInfo=0\nErrorIterations=100\nReportIterations=10000\n"
           "CheckpointIterations=10000\nPolite=0\nPoliteValue=50\nBigCarry=0\nErrorReset=85\nInteractive=0\n"
           "RoundoffTest=0\nThreads=256 128\nOutputHInterval=0\nSleep=0\nSleepValue=0\nErrorLimit=40\n")


@pytest.mark.gpu
@pytest.mark.skipif(not os.path.exists(REF), reason="reference binary not built (make -C oracle ref)")
def test_checkpoint_written_by_the_reference_resumes_in_llucas(cli, tmp_path):
    """CUDALucas itself writes c216091 (interrupted with SIGINT, which makes
    it write a checkpoint and exit); llucas continues from that file to the
    prime verdict."""
    (tmp_path / "CUDALucas.ini").write_text(REF_INI)
    q = 216091
    rc, out, err = run_until([REF, "-f", "12K", str(q)], tmp_path, "Iteration 40000 ")
    assert (tmp_path / ("c%d" % q)).exists(), out[-2000:] + err
    raw = (tmp_path / ("c%d" % q)).read_bytes()
    assert len(raw) == 4 * ((q + 31) // 32 + 10)
    r = run(cli, str(q), cwd=str(tmp_path))
    assert r.returncode == 0, r.stderr
    assert "Continuing M%d @ iteration " % q in r.stdout
    assert final_line(tmp_path).startswith("M( %d )P, offset = " % q)


@pytest.mark.gpu
@pytest.mark.skipif(not os.path.exists(REF), reason="reference binary not built (make -C oracle ref)")
def test_checkpoint_written_by_llucas_resumes_in_the_reference(cli, tmp_path):
    """llucas writes c216091; CUDALucas itself continues from that file to the
    prime verdict (the byte layout and CRC are the reference's)."""
    (tmp_path / "CUDALucas.ini").write_text(REF_INI)
    q = 216091
    rc, out, err = run_until([cli, "-f", "12K", str(q)], tmp_path, "Iteration 40000 ")
    assert rc in (0, 1), err
    assert (tmp_path / ("c%d" % q)).exists()
    r = subprocess.run([REF, str(q)], cwd=str(tmp_path), capture_output=True, text=True, timeout=300)
    assert "Continuing M%d @ iteration " % q in r.stdout, r.stdout[-2000:]
    assert "M( %d )P" % q in r.stdout, r.stdout[-2000:]


@pytest.mark.gpu
def test_cli_cufftbench_writes_the_gpu_tables_and_they_are_read(cli, tmp_path):
    """-cufftbench s e passes (CUDALucas.cu:2413-2587): times the supported
    lengths from s K to e K, writes `<gpu> fft.txt` in the reference's layout
    (kept lengths only) and `<gpu> shapes.txt`; a later run reads fft.txt
    (init_ffts, CUDALucas.cu:975-1021) and chooses from the kept lengths."""
    import cudalucas_b200 as cl
    (tmp_path / "CUDALucas.ini").write_text(INI)
    r = run(cli, "-cufftbench", "12", "20", "2", cwd=str(tmp_path))
    assert r.returncode == 0, r.stderr
    gpu = cl.device_name(0)
    fft = (tmp_path / ("%s fft.txt" % gpu)).read_text().split("\n")
    assert "  fft    max exp  ms/iter" in fft
    rows = [l.split() for l in fft if l[:5].strip().isdigit()]
    assert rows and all(12 <= int(k) <= 20 for k, _, _ in rows)
    assert ["16" == k for k, _, _ in rows].count(True) == 1      # a power of two is always kept
    shapes = (tmp_path / ("%s shapes.txt" % gpu)).read_text().split("\n")
    rows_s = [l.split() for l in shapes if l and l[0] != "#"]
    assert any(r[:1] == ["12"] for r in rows_s)
    # fft(K) width ms/iter kernels: the kernel variant is one the table may choose
    assert all(len(r) == 4 and int(r[3]) in (0, cl.native.LL_KERNELS_NO_CLUSTER, cl.native.LL_KERNELS_ALT_WIDE)
               for r in rows_s)
    kept = [int(k) for k, _, _ in rows]
    # the table merged as init_ffts merges fft.txt (built-in lengths below the first kept
    # one and above the last stay), then the length policy's choice for M216091
    cl.fft_table_merge([k * 1024 for k in kept])
    try:
        want = cl.choose_fft_length(216091) // 1024
    finally:
        cl.fft_table_merge([])
    assert want in kept or want < min(kept)
    (tmp_path / "CUDALucas.ini").write_text(INI.replace("ReportIterations=10000", "ReportIterations=100"))
    rc, out, err = run_until([cli, "216091"], tmp_path, "Iteration 200 ")
    assert "Starting M216091 fft length = %dK" % want in out, out[:500]


@pytest.mark.gpu
@pytest.mark.slow
def test_cli_long_selftest(cli, tmp_path):
    """-r 1: the 92-entry table of CUDALucas.cu:2684-2729, 10000 iterations
    each at the default length."""
    r = subprocess.run([cli, "-r", "1"], cwd=str(tmp_path), capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stdout[-2000:]
    assert r.stdout.count("This residue is correct.") == 92


@pytest.mark.gpu
def test_cli_polite_mode(cli, tmp_path):
    """-polite 25 reads the GPU state back every 25 iterations instead of every
    100 (CUDALucas.cu:1979); the result is unchanged."""
    (tmp_path / "CUDALucas.ini").write_text(INI)
    r = run(cli, "-polite", "25", "86243", cwd=str(tmp_path))
    assert r.returncode == 0, r.stderr
    assert final_line(tmp_path).startswith("M( 86243 )P, offset = ")
