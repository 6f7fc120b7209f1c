"""Loaders for the committed golden fixtures in tests/golden/."""
import json
import os

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def kats(table=None):
    d = json.load(open(os.path.join(HERE, "kat_res64.json")))
    names = [table] if table else ["tests", "testl"]
    out = []
    for nm in names:
        out += [(p, int(r, 16)) for p, r in d[nm]["entries"]]
    return out


def exact_entries():
    d = json.load(open(os.path.join(HERE, "exact_res64.json")))
    return [(p, k, int(r, 16)) for p, k, r in d["entries"]]


def large_entries():
    path = os.path.join(HERE, "large_res64.json")
    if not os.path.exists(path):
        return []
    d = json.load(open(path))
    return [(p, k, int(r, 16)) for p, k, r in d["entries"]]


def reference_run_entries():
    """Res64 values printed by the reference binary itself on a B200."""
    out = []
    for name in ("ref_c1_res64.json", "ref_c2_res64.json", "ref_c3_res64.json"):
        d = json.load(open(os.path.join(HERE, name)))
        out += [(p, k, int(r, 16)) for p, k, r in d["entries"]]
    return out
