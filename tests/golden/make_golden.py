"""Generates the committed golden fixtures under tests/golden/.

kat_res64.json: the CUDALucas self-test known-answer tables (exponent, Res64
of s_10000 from s0 = 4), read as text from the reference source
CUDALucas.cu:2673-2729 (tables `tests[20]` and `testl[92]`).

exact_res64.json: Res64 after k iterations for a spread of exponents and k,
computed with exact big-integer arithmetic (oracle/exact.py).

Run from the repository root:  python tests/golden/make_golden.py REFDIR
(REFDIR: the CUDALucas source tree; or set CUDALUCAS_SRC)
"""
import json
import os
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)


def extract_kats(refdir):
    path = os.path.join(refdir, "CUDALucas.cu")
    lines = open(path).read().split("\n")
    out = {}
    for name in ("tests", "testl"):
        start = next(i for i, l in enumerate(lines) if re.search(r"res_test\s+%s\[" % name, l))
        body = []
        i = start
        while True:
            body.append(lines[i])
            if "};" in lines[i]:
                break
            i += 1
        pairs = re.findall(r"\{\s*(\d+)\s*,\s*(0x[0-9a-fA-F]+)\s*\}", "\n".join(body))
        out[name] = {
            "source": "CUDALucas.cu:%d-%d" % (start + 1, i + 1),
            "iterations": 10000,
            "entries": [[int(p), r.lower()] for p, r in pairs],
        }
    assert len(out["tests"]["entries"]) == 20 and len(out["testl"]["entries"]) == 92
    return out


def exact_table():
    from oracle.exact import res64
    cases = []
    for p in (127, 521, 607, 1279, 2203, 4253, 9689, 9941, 11213, 19937, 21701, 23209, 44497):
        for k in (1, 2, 3, 10, 100, p - 2):
            if k <= p - 2:
                cases.append([p, k, "0x%016x" % res64(p, k)])
    for p in (86243, 132049, 216091, 1257787):
        for k in (1, 5, 50, 500):
            cases.append([p, k, "0x%016x" % res64(p, k)])
    return {"generator": "oracle/exact.py (exact big-integer LL)", "entries": cases}


if __name__ == "__main__":
    refdir = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("CUDALUCAS_SRC")
    if not refdir:
        sys.exit("usage: make_golden.py REFDIR (the CUDALucas source tree), or set CUDALUCAS_SRC")
    kats = extract_kats(refdir)
    with open(os.path.join(HERE, "kat_res64.json"), "w") as f:
        json.dump(kats, f, indent=1)
    with open(os.path.join(HERE, "exact_res64.json"), "w") as f:
        json.dump(exact_table(), f, indent=1)
    print("wrote", len(kats["tests"]["entries"]) + len(kats["testl"]["entries"]), "KATs")
