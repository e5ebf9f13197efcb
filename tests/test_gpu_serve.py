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
       ("C2C", 16384, 2, -1), ("C2C", 131072, 1, 1)]


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
