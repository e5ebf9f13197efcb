"""flagfftB200ExecC2CNoAlloc: the transform that allocates nothing, for callers
that cannot call cudaMalloc (allocator-restricted or memory-exhausted code).
It must give the same result as the ordinary plan path (flagfftPlan1d +
flagfftExecC2C) on the same input, call after call, although every call
reuses one fixed workspace inside the library.

Tolerance: relative L2 difference between the two paths <= 5e-7 * log2 N, the
bound each path meets against the FP64 oracle.  This file is named to be
collected last, so a stop-at-first-failure run has run every other test
before it.
"""
import ctypes
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _plan_path(ffb, x, n, batch, direction):
    import torch
    out = torch.empty_like(x)
    p = ffb.plan1d(n, ffb.C2C, batch)
    try:
        p.exec_c2c(x, out, direction)
        torch.cuda.synchronize()
    finally:
        p.destroy()
    return out


# (1 << 17, 8) reaches the 512-point pass (radices 16, 16, 2)
@pytest.mark.parametrize("n,batch", [(8192, 8), (65536, 4), (1 << 17, 8), (1 << 20, 2), (1 << 22, 1)])
def test_no_alloc_matches_plan_path_twice(ffb, torch_cuda, n, batch):
    torch = torch_cuda
    fn = ffb.LIB.flagfftB200ExecC2CNoAlloc
    fn.restype = ctypes.c_int
    fn.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_void_p]
    bound = 5e-7 * math.log2(n)
    g = torch.Generator(device="cuda").manual_seed(n + batch)
    for call, direction in enumerate((ffb.FORWARD, ffb.INVERSE)):
        x = torch.view_as_complex(torch.rand((batch, n, 2), device="cuda", generator=g) * 2 - 1)
        y = torch.full_like(x, float("nan"))
        rc = fn(ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(y.data_ptr()), n, batch, direction, None)
        assert rc == 0, f"call {call}: status {rc}"
        torch.cuda.synchronize()
        ref = _plan_path(ffb, x, n, batch, direction)
        d = y.to(torch.complex128) - ref.to(torch.complex128)
        err = (torch.linalg.vector_norm(d, dim=-1) / torch.linalg.vector_norm(ref.to(torch.complex128), dim=-1)).max()
        assert torch.isfinite(y).all()
        assert err.item() <= bound, f"call {call}: rel L2 {err.item():.3e} > {bound:.3e}"


def test_no_alloc_rejects_oversize_and_bad_lengths(ffb, torch_cuda):
    torch = torch_cuda
    fn = ffb.LIB.flagfftB200ExecC2CNoAlloc
    fn.restype = ctypes.c_int
    fn.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_void_p]
    x = torch.zeros(16, dtype=torch.complex64, device="cuda")
    p = ctypes.c_void_p(x.data_ptr())
    assert fn(p, p, 1 << 22, 2, ffb.FORWARD, None) == 8        # batch * n above the fixed workspace
    assert fn(p, p, 1 << 23, 1, ffb.FORWARD, None) == 8        # n above the fixed workspace
    assert fn(p, p, 12288, 1, ffb.FORWARD, None) == 8          # not a power of two
    assert fn(p, p, 4096, 1, ffb.FORWARD, None) == 8           # below the four-step range
    assert fn(None, p, 8192, 1, ffb.FORWARD, None) == 4
    assert fn(p, p, 8192, 1, 0, None) == 4


def test_no_alloc_matches_fp64_oracle_2p20(ffb, torch_cuda):
    """2^20 x 4 against the FP64 oracle itself (relative L2 <= 5e-7 log2 N per
    transform), forward and inverse, on the reference harness's seeded input."""
    from oracle import oracle as O
    torch = torch_cuda
    fn = ffb.LIB.flagfftB200ExecC2CNoAlloc
    fn.restype = ctypes.c_int
    fn.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_void_p]
    n, batch = 1 << 20, 4
    x = O.random_complex(n * batch, O.accuracy_seed(O.C2C, n, batch)).reshape(batch, n)
    dx = torch.from_numpy(x).cuda()
    dy = torch.empty_like(dx)
    for direction in (ffb.FORWARD, ffb.INVERSE):
        rc = fn(ctypes.c_void_p(dx.data_ptr()), ctypes.c_void_p(dy.data_ptr()), n, batch, direction, None)
        assert rc == 0
        torch.cuda.synchronize()
        err = O.error_stats(dy.cpu().numpy(), O.c2c(x.astype(np.complex128), direction))
        assert err["finite"] and err["rel_l2"] <= O.north_star_bound(O.C2C, n), err
