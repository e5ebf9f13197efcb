"""Autotuner on the GPU: tuning writes a valid row of the reference's tune
table, and a plan created afterwards with that database runs the stored tree
and stays within the oracle bounds (relative L2 <= 5e-7 log2 N)."""
import json
import sqlite3

import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n", [4096, 1009])
def test_tune_writes_db_and_plan_uses_it(ffb, torch_cuda, tmp_path, monkeypatch, n):
    db = str(tmp_path / "tuned.sqlite")
    rep = ffb.tune(n, ffb.C2C, 64, ffb.FORWARD, db)
    assert rep["stored"] and rep["best_ms"] > 0 and len(rep["candidates"]) >= 2
    rows = sqlite3.connect(db).execute(
        "SELECT status, rank, fft_length, batch_bucket, dtype, direction, plan_json FROM tuned_measurements").fetchall()
    assert len(rows) == 1
    status, rank, length, bucket, dtype, direction, plan_json = rows[0]
    assert (status, rank, length, bucket, dtype, direction) == ("valid", 0, n, "9-64", "complex64", "forward")
    assert json.loads(plan_json)["root"] == rep["best"]
    monkeypatch.setenv("FLAGFFT_TUNE_DB", db)
    x = O.random_complex(n * 64, 7).reshape(64, n)
    a = torch_cuda.from_numpy(x).cuda()
    b = torch_cuda.empty_like(a)
    plan = ffb.plan1d(n, ffb.C2C, 64)
    try:
        assert plan.tree() == rep["best"]
        plan.execute(a, b, ffb.FORWARD)
        torch_cuda.cuda.synchronize()
    finally:
        plan.destroy()
    err = O.error_stats(b.cpu().numpy(), O.c2c(x.astype(np.complex128), -1))
    assert err["rel_l2"] <= O.north_star_bound(O.C2C, n)
