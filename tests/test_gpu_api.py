"""C API behaviour on the GPU (ctest/test_plan.cpp and the Exec argument checks
of src/exec/c_api_exec.cpp)."""
import ctypes

import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu


def test_create_destroy_all_types(ffb, torch_cuda):
    for t in (ffb.C2C, ffb.Z2Z, ffb.R2C, ffb.D2Z, ffb.C2R, ffb.Z2D):
        p = ffb.plan1d(256, t, 1)
        assert p.handle
        p.destroy()
        q = ffb.plan2d(64, 32, t)
        q.destroy()
    ffb.plan1d(128, ffb.C2C, 4).destroy()
    n = [64, 32]
    ffb.plan_many(n, None, 1, 64 * 32, None, 1, 64 * 32, ffb.C2C, 4).destroy()


def test_description_and_rader(ffb, torch_cuda):
    p = ffb.plan1d(67, ffb.C2C, 1)
    d = p.description()
    assert "Rader" in d and "rader-fused" in d
    assert p.tree()["kind"] == "rader"
    p.destroy()
    q = ffb.plan2d(67, 32, ffb.C2C)
    assert "Rader" in q.description()
    q.destroy()
    r = ffb.plan1d(67, ffb.R2C, 1)
    r.destroy()


def test_exec_argument_checks(ffb, torch_cuda):
    torch = torch_cuda
    p = ffb.plan1d(64, ffb.C2C, 1)
    buf = torch.zeros(64, dtype=torch.complex64, device="cuda")
    L = ffb.LIB
    assert L.flagfftExecC2C(p._h, None, ctypes.c_void_p(buf.data_ptr()), -1) == 4
    assert L.flagfftExecC2C(p._h, ctypes.c_void_p(buf.data_ptr()), ctypes.c_void_p(buf.data_ptr()), 0) == 4
    assert L.flagfftExecZ2Z(p._h, ctypes.c_void_p(buf.data_ptr()), ctypes.c_void_p(buf.data_ptr()), -1) == 3
    assert L.flagfftExecR2C(p._h, ctypes.c_void_p(buf.data_ptr()), ctypes.c_void_p(buf.data_ptr())) == 3
    p.destroy()


def test_zero_in_zero_out(ffb, torch_cuda):
    """ctest/test_exec_c2r_ct_s.cpp:76-97."""
    torch = torch_cuda
    for t, n in ((ffb.C2R, 256), (ffb.Z2D, 100)):
        double = t == ffb.Z2D
        p = ffb.plan1d(n, t, 2)
        inp = torch.zeros((2, n // 2 + 1), dtype=torch.complex128 if double else torch.complex64, device="cuda")
        out = torch.full((2, n), 7.0, dtype=torch.float64 if double else torch.float32, device="cuda")
        p.execute(inp, out)
        torch.cuda.synchronize()
        assert not torch.any(out != 0)
        p.destroy()


@pytest.mark.parametrize("n", [997, 1009, 4096])
def test_roundtrip_is_n_times_input(ffb, torch_cuda, n):
    """ctest/test_exec_c2c_inv_bs_b.cpp:73-91."""
    torch = torch_cuda
    x = O.random_complex(4 * n, 5).reshape(4, n)
    a = torch.from_numpy(x).cuda()
    b = torch.empty_like(a)
    p = ffb.plan1d(n, ffb.C2C, 4)
    p.execute(a, b, -1)
    p.execute(b, b, 1)
    torch.cuda.synchronize()
    lim = sum(O.accuracy_limits(O.C2C, n))
    assert O.error_stats(b.cpu().numpy(), n * x.astype(np.complex128))["rel_l2"] <= lim
    p.destroy()


def test_set_stream(ffb, torch_cuda):
    torch = torch_cuda
    s = torch.cuda.Stream()
    n = 4096
    x = O.random_complex(8 * n, 3).reshape(8, n)
    a = torch.from_numpy(x).cuda()
    b = torch.empty_like(a)
    p = ffb.plan1d(n, ffb.C2C, 8)
    p.set_stream(s)
    torch.cuda.synchronize()
    p.execute(a, b, -1)
    s.synchronize()
    ref = O.c2c(x.astype(np.complex128), -1)
    assert O.error_stats(b.cpu().numpy(), ref)["rel_l2"] < O.north_star_bound(O.C2C, n)
    p.destroy()
