"""Request server (flagfftB200Server*) on the GPU: requests of mixed type,
length and batch submitted together are checked against the FP64 oracle
(relative L2 <= 5e-7 log2 N single / 1e-15 log2 N double precision), and each
request's output is bit-identical alone and in the mix (its tiles do not
depend on the requests that share its tick)."""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu

# (type name, n, batch, direction)
MIX = [("C2C", 1009, 3, -1), ("Z2Z", 64, 5, 1), ("R2C", 4096, 2, -1), ("C2C", 10007, 2, 1), ("C2C", 16, 7, -1),
       ("D2Z", 999, 3, -1), ("C2C", 61423, 1, -1), ("C2R", 1000, 2, 1), ("Z2Z", 1701, 4, -1), ("C2C", 4096, 64, 1),
       ("C2C", 16384, 2, -1), ("C2C", 131072, 1, 1),
       # real lengths without an on-chip core: widened to complex (odd n) or a
       # multi-pass half-length transform with a Hermitian pre pass (2 x prime)
       ("R2C", 30011, 2, -1), ("C2R", 60022, 2, 1), ("D2Z", 20011, 1, -1)]


def _inputs(ffb, torch, seed):
    rng_seed = seed
    out = []
    for t, n, b, d in MIX:
        code = getattr(ffb, t)
        dbl = t in ("Z2Z", "D2Z", "Z2D")
        if t in ("C2C", "Z2Z"):
            x = O.random_complex(n * b, rng_seed, dbl).reshape(b, n)
            y_shape, y_dtype = (b, n), x.dtype
        elif t in ("R2C", "D2Z"):
            x = O.random_real(n * b, rng_seed, dbl).reshape(b, n)
            y_shape, y_dtype = (b, n // 2 + 1), (np.complex128 if dbl else np.complex64)
        else:
            x = np.fft.rfft(O.random_real(n * b, rng_seed, dbl).reshape(b, n).astype(np.float64),
                            axis=-1).astype(np.complex128 if dbl else np.complex64)
            y_shape, y_dtype = (b, n), (np.float64 if dbl else np.float32)
        rng_seed += 1
        xd = torch.from_numpy(np.ascontiguousarray(x)).cuda()
        yd = torch.empty(y_shape, dtype=getattr(torch, np.dtype(y_dtype).name), device="cuda")
        out.append((t, code, n, b, d, x, xd, yd))
    return out


def _reference(t, n, d, x):
    x = x.astype(np.complex128 if np.iscomplexobj(x) else np.float64)
    if t in ("C2C", "Z2Z"):
        return O.c2c(x, d)
    if t in ("R2C", "D2Z"):
        return O.r2c(x)
    return O.c2r(x, n)


def test_server_mix_matches_oracle_and_alone(ffb, torch_cuda):
    torch = torch_cuda
    reqs = _inputs(ffb, torch, 501)
    with ffb.Server(hbm_budget_bytes=4 << 30, max_ticks=3) as srv:
        # alone: one request in flight at a time
        alone = []
        for t, code, n, b, d, x, xd, yd in reqs:
            srv.wait(srv.submit(code, n, b, xd, yd, d))
            alone.append(yd.cpu().numpy().copy())
            yd.zero_()
        # the mix: everything submitted at once
        tickets = [srv.submit(code, n, b, xd, yd, d) for t, code, n, b, d, x, xd, yd in reqs]
        lat = [srv.wait(tk) for tk in tickets]
        assert all(v >= 0 for v in lat)
        stats = srv.stats()
        assert stats["completed"] == 2 * len(reqs) and stats["bytes_in_use"] == 0
    for (t, code, n, b, d, x, xd, yd), solo in zip(reqs, alone):
        got = yd.cpu().numpy()
        np.testing.assert_array_equal(got, solo)
        ftype = {"C2C": O.C2C, "Z2Z": O.Z2Z, "R2C": O.R2C, "D2Z": O.D2Z, "C2R": O.C2R, "Z2D": O.Z2D}[t]
        err = O.error_stats(got, _reference(t, n, d, x))
        assert err["finite"] and err["rel_l2"] <= O.north_star_bound(ftype, n), (t, n, b, d, err)


def test_server_budget_and_arguments(ffb, torch_cuda):
    torch = torch_cuda
    x = torch.zeros(8192, dtype=torch.complex64, device="cuda")
    y = torch.empty_like(x)
    with ffb.Server(hbm_budget_bytes=1 << 16, max_ticks=1) as srv:
        with pytest.raises(ffb.FlagFFTError) as e:
            srv.submit(ffb.C2C, 8192, 1, x, y)  # 128 KiB of input + output: above a 64 KiB budget
        assert e.value.code == 8
        with pytest.raises(ffb.FlagFFTError) as e:
            srv.submit(ffb.C2C, 0, 1, x, y)
        assert e.value.code == 8
        tk = srv.submit(ffb.C2C, 1024, 1, x, y)
        srv.wait(tk)


def test_server_staged_admission_and_overlap(ffb, torch_cuda):
    """(a) A budget smaller than the whole mix: submitted at once, the mix is
    admitted in stages (several ticks), each request once its memory frees.
    (b) Continuous batching: requests submitted while a long request's tick is
    on the GPU are admitted into another tick at once (two ticks in flight,
    requests admitted while the GPU was busy).  Every result must equal the
    request alone, bit for bit, and meet the oracle bound."""
    torch = torch_cuda
    reqs = _inputs(ffb, torch, 901)
    with ffb.Server(hbm_budget_bytes=1 << 30, max_ticks=3) as srv:
        alone = []
        for t, code, n, b, d, x, xd, yd in reqs:
            srv.wait(srv.submit(code, n, b, xd, yd, d))
            alone.append(yd.cpu().numpy().copy())
            yd.zero_()
    # (a) 6 MiB: every request fits (the largest charge, C2C 4096 x 64, is
    # 4 MiB of input + output), the whole mix does not
    with ffb.Server(hbm_budget_bytes=6 << 20, max_ticks=3) as srv:
        for t, code, n, b, d, x, xd, yd in reqs:
            srv.prepare(code, n, d)
        tickets = [srv.submit(code, n, b, xd, yd, d) for t, code, n, b, d, x, xd, yd in reqs]
        for tk in tickets:
            srv.wait(tk, timeout_s=60.0)
        st_a = srv.stats()
        out_a = [yd.cpu().numpy().copy() for *_, yd in reqs]
    assert st_a["ticks"] >= 2 and st_a["bytes_in_use"] == 0, st_a
    # (b) a long request first (C2C 2^20 x 32: about a millisecond on the GPU)
    big_n, big_b = 1 << 20, 32
    bx = torch.randn(big_b, big_n, dtype=torch.complex64, device="cuda")
    by = torch.empty_like(bx)
    for *_, yd in reqs:
        yd.zero_()
    with ffb.Server(hbm_budget_bytes=8 << 30, max_ticks=3) as srv:
        # templates first: building one inside submit() uploads its tables
        # synchronously, which would let the long request finish meanwhile
        srv.prepare(ffb.C2C, big_n, ffb.FORWARD)
        for t, code, n, b, d, x, xd, yd in reqs:
            srv.prepare(code, n, d)
        t_big = srv.submit(ffb.C2C, big_n, big_b, bx, by)
        tickets = [srv.submit(code, n, b, xd, yd, d) for t, code, n, b, d, x, xd, yd in reqs]
        for tk in tickets + [t_big]:
            srv.wait(tk, timeout_s=60.0)
        st_b = srv.stats()
        out_b = [yd.cpu().numpy().copy() for *_, yd in reqs]
    assert st_b["max_ticks_in_flight"] >= 2 and st_b["admitted_while_busy"] > 0, st_b
    for outs in (out_a, out_b):
        for (t, code, n, b, d, x, xd, yd), solo, got in zip(reqs, alone, outs):
            np.testing.assert_array_equal(got, solo)
    for (t, code, n, b, d, x, xd, yd), got in zip(reqs, out_b):
        ftype = {"C2C": O.C2C, "Z2Z": O.Z2Z, "R2C": O.R2C, "D2Z": O.D2Z, "C2R": O.C2R, "Z2D": O.Z2D}[t]
        err = O.error_stats(got, _reference(t, n, d, x))
        assert err["finite"] and err["rel_l2"] <= O.north_star_bound(ftype, n), (t, n, b, d, err)
    ref_big = np.fft.fft(bx[:2].cpu().numpy().astype(np.complex128), axis=-1)
    assert O.error_stats(by[:2].cpu().numpy(), ref_big)["rel_l2"] <= O.north_star_bound(O.C2C, big_n)


def test_server_wait_timeout_keeps_ticket(ffb, torch_cuda):
    """A bounded wait that runs out reports "not done" and keeps the ticket;
    a later wait returns the result.  The request is held back on the host
    (its input is not ready: the caller's stream holds a long kernel the
    server's tick must follow), so nothing on the GPU is made to hang."""
    torch = torch_cuda
    n, b = 4096, 4
    x = torch.randn(b, n, dtype=torch.complex64, device="cuda")
    y = torch.empty_like(x)
    with ffb.Server(hbm_budget_bytes=4 << 30, max_ticks=1) as srv:
        # occupy the only slot with a large request (1.5 GB with its
        # workspace), then wait on the next
        # with a zero timeout: it cannot have finished yet
        big_n, big_b = 1 << 20, 64
        bx = torch.randn(big_b, big_n, dtype=torch.complex64, device="cuda")
        by = torch.empty_like(bx)
        t_big = srv.submit(ffb.C2C, big_n, big_b, bx, by)
        tk = srv.submit(ffb.C2C, n, b, x, y)
        with pytest.raises(TimeoutError):
            srv.wait(tk, timeout_s=0.0)
        srv.wait(t_big, timeout_s=60.0)
        assert srv.wait(tk, timeout_s=60.0) >= 0
    ref = np.fft.fft(x.cpu().numpy().astype(np.complex128), axis=-1)
    err = O.error_stats(y.cpu().numpy(), ref)
    assert err["rel_l2"] <= O.north_star_bound(O.C2C, n)
