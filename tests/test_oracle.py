"""The oracle (FP64 CPU restatement of the reference algorithms) pinned against
independent references: an O(n^2) long-double DFT, numpy's pocketfft, the
reference's own plan trees (golden fixture), and the behaviours the reference's
tests pin (zero in -> zero out, unnormalized round trip, Rader for N=67)."""
import json

import numpy as np
import pytest

from oracle import oracle as O


def _rand(shape, seed, cplx=True):
    r = np.random.default_rng(seed)
    x = r.uniform(-1, 1, shape)
    if cplx:
        x = x + 1j * r.uniform(-1, 1, shape)
    return x


@pytest.fixture(scope="module")
def plans():
    O.build()
    return O.ref_plans()


@pytest.mark.parametrize("n", [2, 3, 5, 7, 16, 23, 60, 64, 67, 81, 97, 128, 210, 243, 256, 361])
def test_oracle_matches_long_double_dft(plans, n):
    x = _rand((n,), n)
    plan = plans.get(f"{n}:c") or O.default_plan(n)
    for d in (-1, 1):
        got = O.c2c(x[None], d, plan)[0]
        ref = O.naive_dft(x, d)
        assert O.error_stats(got, ref)["rel_l2"] < 4e-15


@pytest.mark.parametrize("n", [512, 1009, 1701, 2048, 2023, 4096, 8192, 10007, 16384, 20020])
def test_oracle_matches_numpy(plans, n):
    x = _rand((3, n), n)
    plan = plans.get(f"{n}:c") or O.default_plan(n)
    assert O.error_stats(O.c2c(x, -1, plan), np.fft.fft(x))["rel_l2"] < 1e-14
    assert O.error_stats(O.c2c(x, 1, plan), np.fft.ifft(x) * n)["rel_l2"] < 1e-14


def test_every_plan_kind_is_exercised(plans):
    kinds = set()

    def walk(nd):
        kinds.add(nd["kind"])
        for k in ("row", "col", "fft_plan", "conv_plan"):
            if k in nd:
                walk(nd[k])

    for key in ("4096:c", "1009:c", "67:c", "16384:c", "10007:c"):
        walk(plans[key])
    assert {"ct_leaf", "four_step", "bluestein", "rader"} <= kinds


@pytest.mark.parametrize("n", [15, 16, 67, 100, 101, 1009, 2048])
def test_oracle_real_transforms(n):
    x = _rand((2, n), n + 7, cplx=False)
    assert O.error_stats(O.r2c(x), np.fft.rfft(x))["rel_l2"] < 1e-14
    h = np.fft.rfft(x)
    assert O.error_stats(O.c2r(h, n), np.fft.irfft(h, n) * n)["rel_l2"] < 1e-14


def test_c2r_ignores_imag_of_dc_and_nyquist():
    """compact_to_hermitian_full zeroes Im(X[0]) and Im(X[n/2]) (kernels.py:1185-1186)."""
    n = 16
    h = np.fft.rfft(_rand((1, n), 3, cplx=False))
    h2 = h.copy()
    h2[0, 0] += 5j
    h2[0, n // 2] -= 2j
    assert np.allclose(O.c2r(h, n), O.c2r(h2, n), atol=1e-14)


def test_zero_in_zero_out():
    """ctest/test_exec_c2r_ct_s.cpp:76-97: C2R of zeros is exactly zero."""
    z = np.zeros((2, 9), dtype=np.complex128)
    assert not np.any(O.c2r(z, 16))
    assert not np.any(O.c2c(np.zeros((1, 67), np.complex128), -1, O.default_plan(67)))


@pytest.mark.parametrize("n", [23, 997, 1009, 4096])
def test_roundtrip_is_n_times_input(plans, n):
    """ctest/test_exec_c2c_inv_bs_b.cpp:73-91: inverse(forward(x)) = n x."""
    x = _rand((2, n), 11)
    plan = plans[f"{n}:c"]
    y = O.c2c(O.c2c(x, -1, plan), 1, plan)
    assert O.error_stats(y, n * x)["rel_l2"] < 1e-14


def test_n67_reference_tree_is_rader(plans):
    """ctest/test_plan.cpp:47-54."""
    assert plans["67:c"]["kind"] == "rader"


@pytest.mark.parametrize("kind", ["c2c", "r2c"])
def test_oracle_2d(kind):
    if kind == "c2c":
        x = _rand((2, 12, 20), 5)
        assert O.error_stats(O.fft2(x, "c2c", -1), np.fft.fft2(x))["rel_l2"] < 1e-14
    else:
        x = _rand((2, 12, 20), 5, cplx=False)
        y = O.fft2(x, "r2c")
        assert O.error_stats(y, np.fft.rfft2(x))["rel_l2"] < 1e-14
        back = O.fft2(y, "c2r", 1, n1=20)
        assert O.error_stats(back, x * 240)["rel_l2"] < 1e-14


def test_f32_estimate_is_float_accurate(plans):
    x = _rand((4, 4096), 1).astype(np.complex64)
    err = O.error_stats(O.c2c(x, -1, plans["4096:c"], precision="f32"), np.fft.fft(x.astype(np.complex128)))
    assert 1e-8 < err["rel_l2"] < O.north_star_bound(O.C2C, 4096)


def test_stable_rng_stream():
    """splitmix64 (ctest/flagfft_test.h:390-411): first output of seed 0 is the
    published splitmix64 test value; scalar and vectorised streams agree."""
    r = O.StableRng(0)
    assert r.next_u64() == 0xE220A8397B1DCDAF
    seed = O.accuracy_seed(O.C2C, 4096, 256)
    r = O.StableRng(seed)
    a = np.array([r.signed_unit() for _ in range(64)])
    assert np.array_equal(a, O.signed_units(seed, 64))
    assert a.min() >= -1.0 and a.max() < 1.0


def test_accuracy_seed_formula():
    """ctest/flagfft_test.h:413-417."""
    assert O.accuracy_seed(0x29, 4096, 256) == (0x4654464654455354 ^ (0x29 << 48) ^ (4096 << 16) ^ 256)
    assert O.accuracy_seed(0x29, 16, 1, 1) == (0x4654464654455354 ^ (0x29 << 48) ^ (16 << 16) ^ 1 ^ 0x9E3779B97F4A7C15)


def test_error_stats_metric():
    ref = np.array([[3 + 4j, 0j]])
    val = np.array([[3 + 4j, 1 + 0j]])
    s = O.error_stats(val, ref)
    assert s["rel_l2"] == pytest.approx(1 / 5)
    assert s["rel_linf"] == pytest.approx(1 / 5)
    assert O.error_stats(ref * 0, ref * 0)["rel_l2"] == 0.0
