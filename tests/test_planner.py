"""The engine's planner (host only, via flagfftB200PlannerTree) builds the same
plan trees as the reference planner: against the committed fixture of the
reference planner's output, and against the reference planner binary itself
over a seeded random sweep when oracle/_ref/ref_planner has been built."""
import json
import random
import subprocess
from pathlib import Path

import pytest

from oracle import oracle as O

ROOT = Path(__file__).resolve().parent.parent
REF_BIN = ROOT / "oracle" / "_ref" / "ref_planner"


def strip(d):
    """Compare the fields both serialisers emit (tree shape and leaf parameters)."""
    d = {k: v for k, v in d.items() if k not in ("idx", "prime", "impl")}
    for k in ("row", "col", "fft_plan", "conv_plan"):
        if k in d:
            d[k] = strip(d[k])
    return d


def test_planner_matches_reference_fixture(ffb):
    path = ROOT / "tests" / "golden" / "ref_plans.json"
    rows = json.loads(path.read_text())
    assert len(rows) > 1500
    bad = []
    for r in rows:
        mine = ffb.planner_tree(r["n"], r["dtype"] == "complex128")
        if strip(mine) != strip(r["root"]):
            bad.append(r["n"])
    assert not bad, f"plan trees differ for {bad[:10]}"


@pytest.mark.skipif(not REF_BIN.exists(), reason="reference planner not built here")
def test_planner_matches_reference_binary_sweep(ffb):
    rnd = random.Random(7)
    ns = rnd.sample(range(2, 200000), 300) + [2 ** k for k in range(1, 25)]
    for smem, dt in ((0, "c"), (166912, "c"), (0, "z")):
        args = [f"{n}:{dt}" for n in ns]
        env = {"FFO_SMEM": str(smem or 232448)}
        out = subprocess.run([str(REF_BIN), *args], capture_output=True, text=True, check=True, env=env).stdout
        for line in out.strip().split("\n"):
            r = json.loads(line)
            mine = ffb.planner_tree(r["n"], dt == "z", smem)
            assert strip(mine) == strip(r["root"]), r["n"]


@pytest.mark.parametrize("n,kind", [(4096, "ct_leaf"), (1701, "ct_leaf"), (1009, "bluestein"),
                                    (10007, "bluestein"), (2 ** 24, "four_step"), (67, "rader"),
                                    (23, "bluestein"), (16384, "four_step")])
def test_baseline_plan_kinds(ffb, n, kind):
    assert ffb.planner_tree(n)["kind"] == kind


def test_planner_rejects_bad_lengths(ffb):
    with pytest.raises(ffb.FlagFFTError):
        ffb.planner_tree(0)
