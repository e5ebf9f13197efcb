"""GPU parity: libflagfft.so through the flagfft.h C ABI against the FP64
oracle on the reference test harness's seeded inputs.

Bounds (written per test): relative L2 vs the FP64 oracle
    <= 5e-7 * log2 N   (C2C, R2C, C2R)      <= 1e-15 * log2 N   (Z2Z, D2Z, Z2D)
and, per batch, the reference's own frozen limits C * u * work(N)
(ctest/flagfft_test.h:274-320).  "No worse than the reference": the error is
also compared with the oracle's float-arithmetic restatement of the reference
algorithm on the same input (an estimate of the reference's FP32 Exec output).
"""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu

CT = [16, 64, 81, 243, 256, 361, 512, 2048, 4096, 8192, 16384]
BS = [23, 67, 997, 1009]
EXTRA = [2, 3, 5, 7, 11, 13, 17, 19, 6, 10, 12, 15, 1701, 2023, 10007, 20020, 65536, 30030]
# four-step plans whose passes are fused Bluestein / Rader cores (the four-step
# twiddle applied in their stores), and a Rader prime whose p - 1 has a prime
# factor above 19 (2099: p - 1 = 2 x 1049, run through a Bluestein core)
COMPOSITE = [11573, 19549, 32980, 61423, 2099]
# single-precision Bluestein lengths whose n1 x n2 four-step convolution runs
# in one CTA per transform, one per shape (9..13 x 2048, 13 / 15 / 16 x 1024)
ONE_PASS = [8213, 9221, 10243, 11279, 12301, 6491, 6659, 7688]


def _ref_plan(plans, n, double):
    return plans.get(f"{n}:{'z' if double else 'c'}") or plans.get(f"{n}:c") or O.default_plan(n)


@pytest.fixture(scope="module")
def plans():
    O.build()
    return O.ref_plans()


def _run_c2c(ffb, torch, x, direction, double):
    n = x.shape[-1]
    batch = x.shape[0]
    dev_in = torch.from_numpy(x).cuda()
    dev_out = torch.empty_like(dev_in)
    plan = ffb.plan1d(n, ffb.Z2Z if double else ffb.C2C, batch)
    try:
        plan.execute(dev_in, dev_out, direction)
        torch.cuda.synchronize()
        return dev_out.cpu().numpy()
    finally:
        plan.destroy()


def _check(err, ftype, n, est=None):
    bound = O.north_star_bound(ftype, n)
    lim_l2, lim_inf = O.accuracy_limits(ftype, n)
    assert err["finite"]
    assert err["rel_l2"] <= bound, (n, err, bound)
    assert err["rel_l2"] <= lim_l2 and err["rel_linf"] <= lim_inf, (n, err, lim_l2, lim_inf)
    if est is not None:
        # no worse than the reference algorithm in the same precision (with slack for rounding noise)
        assert err["rel_l2"] <= 1.5 * est["rel_l2"] + 1e-8, (n, err, est)


@pytest.mark.parametrize("double", [False, True], ids=["C2C", "Z2Z"])
@pytest.mark.parametrize("n", CT + BS + EXTRA + COMPOSITE)
def test_c2c_z2z_vs_oracle(ffb, torch_cuda, plans, n, double):
    torch = torch_cuda
    batch = 4 if n <= 20020 else 2
    if n in COMPOSITE:
        batch = 2
    ftype = O.Z2Z if double else O.C2C
    x = O.random_complex(n * batch, O.accuracy_seed(ftype, n, batch), double).reshape(batch, n)
    plan = _ref_plan(plans, n, double)
    for direction in (-1, 1):
        got = _run_c2c(ffb, torch, x, direction, double)
        ref = O.c2c(x.astype(np.complex128), direction, plan)
        est = None if double or n > 20020 else O.error_stats(O.c2c(x, direction, plan, precision="f32"), ref)
        _check(O.error_stats(got, ref), ftype, n, est)


@pytest.mark.parametrize("n", ONE_PASS)
def test_bluestein_one_pass_vs_oracle(ffb, torch_cuda, plans, n):
    torch = torch_cuda
    batch = 3
    plan_ours = ffb.plan1d(n, ffb.C2C, batch)
    try:
        assert "bluestein-four-step" in plan_ours.description()
    finally:
        plan_ours.destroy()
    x = O.random_complex(n * batch, O.accuracy_seed(O.C2C, n, batch), False).reshape(batch, n)
    plan = _ref_plan(plans, n, False)
    for direction in (-1, 1):
        got = _run_c2c(ffb, torch, x, direction, False)
        ref = O.c2c(x.astype(np.complex128), direction, plan)
        est = O.error_stats(O.c2c(x, direction, plan, precision="f32"), ref)
        _check(O.error_stats(got, ref), O.C2C, n, est)


@pytest.mark.parametrize("double", [False, True], ids=["C2C", "Z2Z"])
@pytest.mark.parametrize("n,batch", [(131072, 1), (65536, 3), (32768, 2)])
def test_four_step_tiles_vs_oracle(ffb, torch_cuda, plans, n, batch, double):
    """Four-steps whose strided passes run on the tile kernels (partial last
    tiles included)."""
    torch = torch_cuda
    ftype = O.Z2Z if double else O.C2C
    x = O.random_complex(n * batch, O.accuracy_seed(ftype, n, batch), double).reshape(batch, n)
    for direction in (-1, 1):
        got = _run_c2c(ffb, torch, x, direction, double)
        ref = O.c2c(x.astype(np.complex128), direction)
        _check(O.error_stats(got, ref), ftype, n)


@pytest.mark.parametrize("double", [False, True], ids=["C2C", "Z2Z"])
@pytest.mark.parametrize("shape", [(2048, 40), (4096, 24), (1024, 50), (1701, 20)])
def test_2d_column_tiles_vs_oracle(ffb, torch_cuda, shape, double):
    """2-D transforms whose column pass runs on the tile kernels, with a
    partial last tile of columns."""
    torch = torch_cuda
    n0, n1 = shape
    x = O.random_complex(n0 * n1, 4321 + n0 + n1, double).reshape(1, n0, n1)
    dev_in = torch.from_numpy(x).cuda()
    dev_out = torch.empty_like(dev_in)
    p = ffb.plan_many([n0, n1], None, 1, n0 * n1, None, 1, n0 * n1, ffb.Z2Z if double else ffb.C2C, 1)
    try:
        assert "tiles" in p.description()
        for d in (-1, 1):
            p.execute(dev_in, dev_out, d)
            torch.cuda.synchronize()
            ref = O.fft2(x.astype(np.complex128), "c2c", d)
            _check(O.error_stats(dev_out.cpu().numpy().reshape(1, -1), ref.reshape(1, -1)),
                   O.Z2Z if double else O.C2C, n0 * n1)
    finally:
        p.destroy()


@pytest.mark.parametrize("scale", [2.0 ** -20, 1.0, 2.0 ** 20])
def test_input_scales(ffb, torch_cuda, plans, scale):
    """ctest/flagfft_test.h:457: inputs scaled by 2^-20, 1, 2^20."""
    n, batch = 1009, 4
    x = (O.random_complex(n * batch, O.accuracy_seed(O.C2C, n, batch, 1)) * np.float32(scale)).reshape(batch, n)
    got = _run_c2c(ffb, torch_cuda, x, -1, False)
    _check(O.error_stats(got, O.c2c(x.astype(np.complex128), -1, plans["1009:c"])), O.C2C, n)


@pytest.mark.parametrize("double", [False, True], ids=["R2C_C2R", "D2Z_Z2D"])
# 40022 / 65534: n/2 = 20011 (prime) and 32767 = 7 * 31 * 151 run as a complex
# transform of n/2 points of any lowering plus the Hermitian post / pre pass;
# 201 = 3 * 67 and 40027 (prime, odd) widen to a full complex transform
@pytest.mark.parametrize("n", [2, 3, 15, 16, 64, 100, 101, 134, 256, 2018, 4096, 8192, 16384, 1701, 9000, 40022, 65534,
                               201, 40027, 131072, 262144])
def test_real_vs_oracle(ffb, torch_cuda, n, double):
    torch = torch_cuda
    batch = 4
    fwd, inv = (O.D2Z, O.Z2D) if double else (O.R2C, O.C2R)
    x = O.random_real(n * batch, O.accuracy_seed(fwd, n, batch), double).reshape(batch, n)
    half = n // 2 + 1
    dev_in = torch.from_numpy(x).cuda()
    dev_out = torch.empty((batch, half), dtype=torch.complex128 if double else torch.complex64, device="cuda")
    p = ffb.plan1d(n, fwd, batch)
    p.execute(dev_in, dev_out)
    torch.cuda.synchronize()
    got = dev_out.cpu().numpy()
    p.destroy()
    ref = O.r2c(x.astype(np.float64))
    _check(O.error_stats(got, ref), fwd, n)
    # inverse on the oracle spectrum with garbage in Im(DC) / Im(Nyquist) (ignored by C2R)
    spec = ref.astype(np.complex128 if double else np.complex64)
    spec[:, 0] += 3j
    if n % 2 == 0:
        spec[:, -1] -= 2j
    dev_spec = torch.from_numpy(spec).cuda()
    dev_real = torch.empty((batch, n), dtype=torch.float64 if double else torch.float32, device="cuda")
    q = ffb.plan1d(n, inv, batch)
    q.execute(dev_spec, dev_real)
    torch.cuda.synchronize()
    got2 = dev_real.cpu().numpy()
    q.destroy()
    _check(O.error_stats(got2, O.c2r(spec.astype(np.complex128), n)), inv, n)


@pytest.mark.parametrize("n", [16, 64, 1701, 4096])
def test_r2c_c2r_in_place_padded(ffb, torch_cuda, n):
    """In-place real transforms use padded rows of 2(n/2+1) reals (src/exec/raw_nodes.cpp:425-429)."""
    torch = torch_cuda
    batch = 3
    half = n // 2 + 1
    x = O.random_real(n * batch, 99).reshape(batch, n)
    buf = torch.zeros((batch, 2 * half), dtype=torch.float32, device="cuda")
    buf[:, :n] = torch.from_numpy(x).cuda()
    p = ffb.plan1d(n, ffb.R2C, batch)
    p.execute(buf, buf)
    torch.cuda.synchronize()
    spec = buf.cpu().numpy().view(np.complex64)
    p.destroy()
    _check(O.error_stats(spec, O.r2c(x.astype(np.float64))), O.R2C, n)
    q = ffb.plan1d(n, ffb.C2R, batch)
    q.execute(buf, buf)
    torch.cuda.synchronize()
    back = buf.cpu().numpy()[:, :n]
    q.destroy()
    _check(O.error_stats(back, n * x.astype(np.float64)), O.C2R, n)


@pytest.mark.parametrize("shape", [(16, 16), (64, 64), (128, 256), (256, 128), (23, 23), (997, 16), (16, 997),
                                   (67, 32)])
@pytest.mark.parametrize("batch", [1, 4])
def test_2d_vs_oracle(ffb, torch_cuda, shape, batch):
    """ctest/test_2d_correctness.cpp:14-31 sizes."""
    torch = torch_cuda
    n0, n1 = shape
    x = O.random_complex(n0 * n1 * batch, 1234 + n0 + n1).reshape(batch, n0, n1)
    dev_in = torch.from_numpy(x).cuda()
    dev_out = torch.empty_like(dev_in)
    dist = n0 * n1
    p = ffb.plan_many([n0, n1], None, 1, dist, None, 1, dist, ffb.C2C, batch)
    for d in (-1, 1):
        p.execute(dev_in, dev_out, d)
        torch.cuda.synchronize()
        ref = O.fft2(x.astype(np.complex128), "c2c", d)
        _check(O.error_stats(dev_out.cpu().numpy().reshape(batch, -1), ref.reshape(batch, -1)), O.C2C, n0 * n1)
    p.destroy()
    xr = O.random_real(n0 * n1 * batch, 77 + n0).reshape(batch, n0, n1)
    h1 = n1 // 2 + 1
    pr = ffb.plan_many([n0, n1], None, 1, dist, None, 1, n0 * h1, ffb.R2C, batch)
    spec = torch.empty((batch, n0, h1), dtype=torch.complex64, device="cuda")
    pr.execute(torch.from_numpy(xr).cuda(), spec)
    torch.cuda.synchronize()
    ref = O.fft2(xr.astype(np.float64), "r2c")
    _check(O.error_stats(spec.cpu().numpy().reshape(batch, -1), ref.reshape(batch, -1)), O.R2C, n0 * n1)
    pr.destroy()
    pc = ffb.plan_many([n0, n1], None, 1, n0 * h1, None, 1, dist, ffb.C2R, batch)
    back = torch.empty((batch, n0, n1), dtype=torch.float32, device="cuda")
    pc.execute(spec, back)
    torch.cuda.synchronize()
    _check(O.error_stats(back.cpu().numpy().reshape(batch, -1), (xr * n0 * n1).reshape(batch, -1)), O.C2R, n0 * n1)
    pc.destroy()


@pytest.mark.parametrize("policy", ["inplace", "multipass"])
@pytest.mark.parametrize("double", [False, True], ids=["C2C", "Z2Z"])
@pytest.mark.parametrize("n", [1009, 1701, 4096, 10007, 20020])
def test_lowering_policies(ffb, torch_cuda, plans, monkeypatch, policy, double, n):
    """Every lowering of a tree (one fused pass in place, or the multi-pass
    chain) meets the same bounds; FLAGFFT_ONCHIP_POLICY is read at plan time."""
    monkeypatch.setenv("FLAGFFT_ONCHIP_POLICY", policy)
    batch = 3
    ftype = O.Z2Z if double else O.C2C
    x = O.random_complex(n * batch, O.accuracy_seed(ftype, n, batch, 2), double).reshape(batch, n)
    plan = _ref_plan(plans, n, double)
    for direction in (-1, 1):
        got = _run_c2c(ffb, torch_cuda, x, direction, double)
        _check(O.error_stats(got, O.c2c(x.astype(np.complex128), direction, plan)), ftype, n)


# 1701 = 9 9 7 3 has two row-kernel forms: up to 2048 transforms a pass the
# wide one (one radix-7 butterfly per thread, 256 threads a row), above that
# the default (one radix-9 butterfly per thread, 192 threads).
@pytest.mark.parametrize("batch,double,threads", [(5, False, 256), (2048, False, 256), (2049, False, 192),
                                                  (3, True, 256), (3000, True, 192)])
def test_1701_row_forms(ffb, torch_cuda, batch, double, threads):
    n = 1701
    ftype = O.Z2Z if double else O.C2C
    x = O.random_complex(n * batch, O.accuracy_seed(ftype, n, batch), double).reshape(batch, n)
    with ffb.plan1d(n, ffb.Z2Z if double else ffb.C2C, batch) as p:
        assert f"threads={threads} " in p.description(), p.description()
    for direction in (-1, 1):
        got = _run_c2c(ffb, torch_cuda, x, direction, double)
        _check(O.error_stats(got, O.c2c(x.astype(np.complex128), direction)), ftype, n)
