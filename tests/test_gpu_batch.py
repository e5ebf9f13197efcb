"""Batch plans (flagfftB200PlanBatch) on the GPU: transforms of uneven
lengths, packed group after group, run as persistent launches over a work
queue and replayed through a CUDA graph.  Every transform is checked against
the FP64 oracle with the same bounds as the single-length plans:
relative L2 <= 5e-7 log2 N (C2C) / 1e-15 log2 N (Z2Z)."""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu

# single-pass (Stockham, fused Bluestein, fused Rader), two-pass four-step and
# three-pass Bluestein lengths side by side, and 16384 (single precision: a
# row-kernel pass that launches on its own beside the persistent launches)
LENGTHS = [16, 2, 13, 67, 1009, 1701, 4096, 10007, 20020, 65536, 12289, 16384]
COUNTS = [5, 3, 4, 2, 3, 2, 2, 2, 1, 1, 1, 2]


def _check_groups(got, x, lengths, counts, direction, double):
    ftype = O.Z2Z if double else O.C2C
    off = 0
    for n, c in zip(lengths, counts):
        xs = x[off:off + n * c].reshape(c, n).astype(np.complex128)
        ref = O.c2c(xs, direction)
        err = O.error_stats(got[off:off + n * c].reshape(c, n), ref)
        assert err["finite"] and err["rel_l2"] <= O.north_star_bound(ftype, n), (n, c, direction, err)
        off += n * c


def _run(ffb, torch, plan, x, direction):
    a = torch.from_numpy(x).cuda()
    b = torch.empty_like(a)
    plan.execute(a, b, direction)
    torch.cuda.synchronize()
    return a, b


@pytest.mark.parametrize("double", [False, True], ids=["C2C", "Z2Z"])
def test_batch_uneven_lengths(ffb, torch_cuda, double):
    torch = torch_cuda
    ftype = ffb.Z2Z if double else ffb.C2C
    total = sum(n * c for n, c in zip(LENGTHS, COUNTS))
    x = O.random_complex(total, O.accuracy_seed(O.Z2Z if double else O.C2C, total, 1, 3), double)
    plan = ffb.plan_batch(LENGTHS, COUNTS, ftype)
    try:
        assert plan.launch_count(-1) >= 1
        for direction in (-1, 1):
            a, b = _run(ffb, torch, plan, x, direction)
            first = b.cpu().numpy()
            _check_groups(first, x, LENGTHS, COUNTS, direction, double)
            # second Exec on the same buffers replays the captured graph
            b.zero_()
            plan.execute(a, b, direction)
            torch.cuda.synchronize()
            np.testing.assert_array_equal(b.cpu().numpy(), first)
        # in place
        a = torch.from_numpy(x).cuda()
        plan.execute(a, a, -1)
        torch.cuda.synchronize()
        _check_groups(a.cpu().numpy(), x, LENGTHS, COUNTS, -1, double)
    finally:
        plan.destroy()


def test_batch_matches_single_plans(ffb, torch_cuda):
    """Each group of a batch gives the same result as its own plan1d plan
    (the same lowering, run from the work queue instead of its own launch)."""
    torch = torch_cuda
    lengths, counts = [1009, 4096, 10007], [3, 2, 2]
    total = sum(n * c for n, c in zip(lengths, counts))
    x = O.random_complex(total, 77)
    plan = ffb.plan_batch(lengths, counts, ffb.C2C)
    try:
        _, b = _run(ffb, torch, plan, x, -1)
        got = b.cpu().numpy()
    finally:
        plan.destroy()
    off = 0
    for n, c in zip(lengths, counts):
        p = ffb.plan1d(n, ffb.C2C, c)
        try:
            _, y = _run(ffb, torch, p, x[off:off + n * c].reshape(c, n), -1)
        finally:
            p.destroy()
        np.testing.assert_allclose(got[off:off + n * c].reshape(c, n), y.cpu().numpy(), rtol=0, atol=1e-4)
        off += n * c


def test_batch_without_graphs(ffb, torch_cuda, monkeypatch):
    """FLAGFFT_BATCH_GRAPH=0 (read at plan time) launches the phases directly."""
    monkeypatch.setenv("FLAGFFT_BATCH_GRAPH", "0")
    lengths, counts = [64, 10007, 243], [4, 1, 3]
    total = sum(n * c for n, c in zip(lengths, counts))
    x = O.random_complex(total, 91)
    plan = ffb.plan_batch(lengths, counts, ffb.C2C)
    try:
        assert "direct" in plan.description()
        _, b = _run(ffb, torch_cuda, plan, x, 1)
        _check_groups(b.cpu().numpy(), x, lengths, counts, 1, False)
    finally:
        plan.destroy()
