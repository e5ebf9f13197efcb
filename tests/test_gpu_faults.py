"""Failure handling on the host (nothing here faults, traps or hangs the GPU):

* a failing device allocator (FLAGFFT_FAULT_ALLOC=1, injected in the
  library's allocation wrapper) makes plan creation return
  FLAGFFT_ALLOC_FAILED with the handle left NULL, as the reference maps
  std::bad_alloc (src/exec/c_api_plan.cpp:240-244); the next plan succeeds;
* a corrupt tune-database row -- unparsable JSON, or a valid tree for another
  length -- is ignored and the planner's own tree is used, as the reference's
  lookup does (src/utils/plan_json.cpp:163-207, src/exec/c_api_plan.cpp:27-39);
* the device-side bounded waits of the TMA column kernels report no failure
  after a run.
"""
import ctypes
import json
import sqlite3

import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu


def test_failing_allocator_gives_alloc_failed(ffb, torch_cuda, monkeypatch):
    lib = ffb.LIB
    h = ctypes.c_void_p(0)
    monkeypatch.setenv("FLAGFFT_FAULT_ALLOC", "1")
    # a length no earlier test planned, so its tables are not in the shared cache
    rc = lib.flagfftPlan1d(ctypes.byref(h), 12347, ffb.C2C, 3)
    assert rc == 2 and not h.value  # FLAGFFT_ALLOC_FAILED, no handle
    rc = lib.flagfftPlan1d(ctypes.byref(h), 1 << 21, ffb.C2C, 2)  # multi-pass: a workspace allocation
    assert rc == 2 and not h.value
    monkeypatch.delenv("FLAGFFT_FAULT_ALLOC")
    x = O.random_complex(12347 * 3, 5).reshape(3, 12347)
    xd = torch_cuda.from_numpy(x).cuda()
    yd = torch_cuda.empty_like(xd)
    with ffb.plan1d(12347, ffb.C2C, 3) as p:
        p.execute(xd, yd, ffb.FORWARD)
        torch_cuda.cuda.synchronize()
    err = O.error_stats(yd.cpu().numpy(), O.c2c(x.astype(np.complex128), -1))
    assert err["rel_l2"] <= O.north_star_bound(O.C2C, 12347)


@pytest.mark.parametrize("corrupt", ["not json {", "wrong length"])
def test_corrupt_tune_row_falls_back_to_planner(ffb, torch_cuda, tmp_path, monkeypatch, corrupt):
    n, batch = 4096, 64
    db = str(tmp_path / "tuned.sqlite")
    ffb.tune(n, ffb.C2C, batch, ffb.FORWARD, db)  # a valid row under this key
    con = sqlite3.connect(db)
    if corrupt == "not json {":
        con.execute("UPDATE tuned_measurements SET plan_json=?", (corrupt,))
    else:
        row = json.loads(con.execute("SELECT plan_json FROM tuned_measurements").fetchone()[0])
        row["root"] = ffb.planner_tree(2048)  # a tree of another length
        con.execute("UPDATE tuned_measurements SET plan_json=?", (json.dumps(row),))
    con.commit()
    con.close()
    monkeypatch.setenv("FLAGFFT_TUNE_DB", db)
    x = O.random_complex(n * batch, 9).reshape(batch, n)
    xd = torch_cuda.from_numpy(x).cuda()
    yd = torch_cuda.empty_like(xd)
    with ffb.plan1d(n, ffb.C2C, batch) as p:
        assert p.tree() == ffb.planner_tree(n)
        p.execute(xd, yd, ffb.FORWARD)
        torch_cuda.cuda.synchronize()
    err = O.error_stats(yd.cpu().numpy(), O.c2c(x.astype(np.complex128), -1))
    assert err["rel_l2"] <= O.north_star_bound(O.C2C, n)


def test_tma_column_waits_never_gave_up(ffb, torch_cuda):
    n0 = n1 = 4096
    x = torch_cuda.randn(n0, n1, dtype=torch_cuda.complex64, device="cuda")
    y = torch_cuda.empty_like(x)
    with ffb.plan2d(n0, n1, ffb.C2C) as p:
        assert "tma-columns" in p.description()
        p.execute(x, y, ffb.FORWARD)
        torch_cuda.cuda.synchronize()
    assert ffb.device_wait_failures() == 0
