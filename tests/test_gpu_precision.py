"""Precision mode (flagfftB200PrecisionC2C): radix-16 stages as split-bf16
DFT-matrix products on the tcgen05 tensor cores, measured against the FP64
oracle at N = 256, 4096 and 65536 (65536 = 256 x 256: two 256-point
tensor-core passes with the four-step twiddle and transposes between them in
fp32 on the GPU).

Bound: relative L2 <= 5e-7 log2 N per transform (the single-precision bound
the plan path meets).  The six-term split (every product down to 2^-24) must
meet it; the three-term split (the two-way split's three products) is
measured and must stay a correct transform (relative L2 < 1e-4) -- whether it
meets the bound is the ship-or-not question this mode answers, and the errors
are printed (pytest -s) for the record.
"""
import ctypes
import math

import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _pm(ffb, torch, x, direction, terms):
    fn = ffb.LIB.flagfftB200PrecisionC2C
    fn.restype = ctypes.c_int
    fn.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                   ctypes.c_void_p]
    y = torch.empty_like(x)
    rc = fn(ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(y.data_ptr()), x.shape[-1], x.shape[0], direction, terms,
            None)
    assert rc == 0, rc
    return y


def _per_row_rel_l2(got, ref):
    d = np.linalg.norm((got.astype(np.complex128) - ref), axis=-1)
    return float((d / np.linalg.norm(ref, axis=-1)).max())


@pytest.mark.parametrize("terms", [3, 6])
@pytest.mark.parametrize("n,batch", [(4096, 64), (256, 1000)])
def test_precision_mode_vs_oracle(ffb, torch_cuda, n, batch, terms):
    torch = torch_cuda
    x = O.random_complex(n * batch, O.accuracy_seed(O.C2C, n, batch, 7)).reshape(batch, n)
    xd = torch.from_numpy(x).cuda()
    for direction in (ffb.FORWARD, ffb.INVERSE):
        got = _pm(ffb, torch, xd, direction, terms)
        torch.cuda.synchronize()
        ref = O.c2c(x.astype(np.complex128), direction)
        err = _per_row_rel_l2(got.cpu().numpy(), ref)
        bound = 5e-7 * math.log2(n)
        print(f"precision mode n={n} terms={terms} dir={direction}: rel L2 {err:.3e} (bound {bound:.3e})")
        assert np.isfinite(err) and err < 1e-4
        if terms == 6:
            assert err <= bound, (n, terms, err, bound)


@pytest.mark.parametrize("terms", [3, 6])
def test_precision_mode_65536_four_step(ffb, torch_cuda, terms):
    torch = torch_cuda
    n, batch, n1 = 65536, 4, 256
    x = O.random_complex(n * batch, O.accuracy_seed(O.C2C, n, batch, 7)).reshape(batch, n)
    xd = torch.from_numpy(x).cuda()
    # x[j1 * 256 + j2]: columns j2 (over j1) -> 256-point transforms
    cols = xd.view(batch, n1, n1).transpose(1, 2).contiguous().view(batch * n1, n1)
    a = _pm(ffb, torch, cols, ffb.FORWARD, terms).view(batch, n1, n1)  # [b][j2][k1]
    j2 = torch.arange(n1, device="cuda", dtype=torch.float64).view(n1, 1)
    k1 = torch.arange(n1, device="cuda", dtype=torch.float64).view(1, n1)
    tw = torch.exp(-2j * math.pi * ((j2 * k1) % n) / n).to(torch.complex64)
    a = (a * tw).transpose(1, 2).contiguous().view(batch * n1, n1)  # rows k1 over j2
    b = _pm(ffb, torch, a, ffb.FORWARD, terms).view(batch, n1, n1)  # [b][k1][k2] = X[k1 + 256 k2]
    got = b.transpose(1, 2).contiguous().view(batch, n)
    torch.cuda.synchronize()
    err = _per_row_rel_l2(got.cpu().numpy(), O.c2c(x.astype(np.complex128), -1))
    bound = 5e-7 * math.log2(n)
    print(f"precision mode n={n} terms={terms}: rel L2 {err:.3e} (bound {bound:.3e})")
    assert np.isfinite(err) and err < 1e-4
    if terms == 6:
        assert err <= bound


def test_precision_mode_arguments_and_waits(ffb, torch_cuda):
    torch = torch_cuda
    fn = ffb.LIB.flagfftB200PrecisionC2C
    fn.restype = ctypes.c_int
    fn.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                   ctypes.c_void_p]
    x = torch.zeros(4096, dtype=torch.complex64, device="cuda")
    p = ctypes.c_void_p(x.data_ptr())
    assert fn(p, p, 1024, 1, -1, 3, None) == 14  # NOT_SUPPORTED length
    assert fn(p, p, 4096, 1, -1, 4, None) == 14  # NOT_SUPPORTED term count
    assert fn(p, p, 4096, 1, 0, 3, None) == 4
    assert fn(None, p, 4096, 1, -1, 3, None) == 4
    c = ctypes.c_longlong(-1)
    ffb.LIB.flagfftB200PrecisionWaitFailures.argtypes = [ctypes.POINTER(ctypes.c_longlong)]
    assert ffb.LIB.flagfftB200PrecisionWaitFailures(ctypes.byref(c)) == 0 and c.value == 0
