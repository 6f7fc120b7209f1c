"""GPU test of the engine's timing tool (the counterpart of -cufftbench /
-threadbench): every launch choice of a length is timed and the fastest is
written to a tuning table."""
import json

import pytest

from cudalucas_b200 import fftbench

pytestmark = pytest.mark.gpu


def test_all_shapes_of_a_short_length_are_timed(tmp_path):
    n = 12288
    cands = fftbench.candidate_shapes(n)
    # the cluster-resident step, the two-launch path of the same shape, and
    # the other row widths with the engine's kernels for them
    assert any(sh.get("cluster") for _, sh in cands)
    assert any(not sh.get("cluster") and sh["W"] == 256 for _, sh in cands)
    assert all(sh["wide_specialised"] or sh["W"] != 256 for _, sh in cands)
    table = tmp_path / "t.json"
    fftbench.main(["12K", "--iters", "50", "--all-shapes", "--table", str(table)])
    got = json.loads(table.read_text())
    best = got[str(n)]
    assert best["ms_per_iter"] > 0 and best["W"] in {sh["W"] for _, sh in cands}
