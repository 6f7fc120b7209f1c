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
