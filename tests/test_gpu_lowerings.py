"""Lowerings of plan trees that do not fit the on-chip or two-pass shapes,
against the FP64 oracle (relative L2 <= 5e-7 log2 N single / 1e-15 log2 N
double precision per transform, plus the reference suite's C * u * work(N)
limits):

* 2-D transforms with an axis too long for one CTA (src/exec/raw_nodes.cpp
  :549-610 runs any child per axis): rows, tiled transpose, the other axis
  as rows, transpose back -- C2C, Z2Z, R2C and C2R;
* Bluestein convolutions too long for a one-codelet column (large primes):
  the three-pass chain with a multi-stage column core;
* trees that nest a four-step in a four-step or in a Bluestein inside a
  four-step (30021 = 3 x Bluestein(10007, M = 20020 = 13 x 1540),
  30098 = 2 x four-step(15049)), and a four-step over a multi-pass Bluestein
  (2 x 1048573).
"""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _bounds(err, ftype, n):
    assert err["finite"]
    assert err["rel_l2"] <= O.north_star_bound(ftype, n), (n, err)
    lim_l2, lim_inf = O.accuracy_limits(ftype, n)
    assert err["rel_l2"] <= lim_l2 and err["rel_linf"] <= lim_inf, (n, err, lim_l2, lim_inf)


@pytest.mark.parametrize("shape,double", [((65536, 64), False), ((64, 65536), True), ((20011, 8), False),
                                          ((8, 20011), True), ((131072, 4), False)])
def test_2d_long_axis_c2c(ffb, torch_cuda, shape, double):
    torch = torch_cuda
    n0, n1 = shape
    ftype = O.Z2Z if double else O.C2C
    x = O.random_complex(n0 * n1, O.accuracy_seed(ftype, n0 * n1, 1), double).reshape(1, n0, n1)
    with ffb.plan2d(n0, n1, ffb.Z2Z if double else ffb.C2C) as p:
        assert "transpose" in p.description()
        for d in (ffb.FORWARD, ffb.INVERSE):
            xd = torch.from_numpy(x).cuda()
            yd = torch.empty_like(xd)
            p.execute(xd, yd, d)
            torch.cuda.synchronize()
            ref = O.fft2(x.astype(np.complex128), "c2c", d)
            _bounds(O.error_stats(yd.cpu().numpy().reshape(1, -1), ref.reshape(1, -1)), ftype, n0 * n1)


@pytest.mark.parametrize("shape", [(65536, 16), (20011, 8)])
def test_2d_long_column_real(ffb, torch_cuda, shape):
    torch = torch_cuda
    n0, n1 = shape
    h1 = n1 // 2 + 1
    x = O.random_real(n0 * n1, O.accuracy_seed(O.R2C, n0 * n1, 1)).reshape(1, n0, n1)
    with ffb.plan2d(n0, n1, ffb.R2C) as p:
        spec = torch.empty((1, n0, h1), dtype=torch.complex64, device="cuda")
        p.execute(torch.from_numpy(x).cuda(), spec)
        torch.cuda.synchronize()
    ref = O.fft2(x.astype(np.float64), "r2c")
    _bounds(O.error_stats(spec.cpu().numpy().reshape(1, -1), ref.reshape(1, -1)), O.R2C, n0 * n1)
    with ffb.plan2d(n0, n1, ffb.C2R) as q:
        back = torch.empty((1, n0, n1), dtype=torch.float32, device="cuda")
        q.execute(spec, back)
        torch.cuda.synchronize()
    refb = O.fft2(spec.cpu().numpy().astype(np.complex128), "c2r", n1=n1)
    _bounds(O.error_stats(back.cpu().numpy().reshape(1, -1), refb.reshape(1, -1)), O.C2R, n0 * n1)


@pytest.mark.parametrize("n,batch,double", [(1048573, 1, False), (131074, 2, True), (2097146, 1, False),
                                            (30021, 4, False), (30021, 4, True), (30098, 4, False),
                                            (30098, 4, True)])
def test_long_bluestein_and_nested_trees(ffb, torch_cuda, n, batch, double):
    torch = torch_cuda
    ftype = O.Z2Z if double else O.C2C
    x = O.random_complex(n * batch, O.accuracy_seed(ftype, n, batch), double).reshape(batch, n)
    with ffb.plan1d(n, ffb.Z2Z if double else ffb.C2C, batch) as p:
        for d in (ffb.FORWARD, ffb.INVERSE):
            xd = torch.from_numpy(x).cuda()
            yd = torch.empty_like(xd)
            p.execute(xd, yd, d)
            torch.cuda.synchronize()
            _bounds(O.error_stats(yd.cpu().numpy(), O.c2c(x.astype(np.complex128), d)), ftype, n)


# The one-pass Bluestein in its pair form ($FLAGFFT_BLUESTEIN_PAIR=1, read at
# plan time): the N1 x 2048 convolution rows split over a two-CTA cluster
# exchanging through distributed shared memory, N1 = 8 (8009), 10 (10007,
# 8501) and 12 (11003); batch 300 is more transforms than pairs resident at
# once, so pairs walk several transforms.
@pytest.mark.parametrize("n,batch,double", [(8009, 3, True), (10007, 300, True), (8501, 2, True),
                                            (11003, 5, True), (10007, 300, False), (11003, 5, False)])
def test_bluestein_pair(ffb, torch_cuda, monkeypatch, n, batch, double):
    torch = torch_cuda
    monkeypatch.setenv("FLAGFFT_BLUESTEIN_PAIR", "1")
    ftype = O.Z2Z if double else O.C2C
    x = O.random_complex(n * batch, O.accuracy_seed(ftype, n, batch), double).reshape(batch, n)
    with ffb.plan1d(n, ffb.Z2Z if double else ffb.C2C, batch) as p:
        assert "bluestein-four-step-pair" in p.description()
        for d in (ffb.FORWARD, ffb.INVERSE):
            xd = torch.from_numpy(x).cuda()
            yd = torch.empty_like(xd)
            p.execute(xd, yd, d)
            torch.cuda.synchronize()
            _bounds(O.error_stats(yd.cpu().numpy(), O.c2c(x.astype(np.complex128), d)), ftype, n)


# The plan tree's own lowerings (FLAGFFT_TREE_LOWERING=1, read at plan time):
# the reference's generic four-step over a multi-pass child (60022 = 2 x
# Bluestein(30011), M = 60021 = 19 x 3159) and its Rader chain over a
# multi-pass p - 1 transform (65537: 256 x 256; 40961: 128 x 320), in place
# and out of place.
@pytest.mark.parametrize("n,batch,double,marker", [(60022, 3, False, "transpose"), (65537, 2, False, "rader-gather"),
                                                   (40961, 2, True, "rader-gather"), (65537, 1, True, "rader-gather")])
def test_tree_lowering(ffb, torch_cuda, monkeypatch, n, batch, double, marker):
    monkeypatch.setenv("FLAGFFT_TREE_LOWERING", "1")
    torch = torch_cuda
    ftype = O.Z2Z if double else O.C2C
    x = O.random_complex(n * batch, O.accuracy_seed(ftype, n, batch, 3), double).reshape(batch, n)
    with ffb.plan1d(n, ffb.Z2Z if double else ffb.C2C, batch) as p:
        assert marker in p.description(), p.description()
        for d in (ffb.FORWARD, ffb.INVERSE):
            ref = np.stack([O.c2c(r, d) for r in x.astype(np.complex128)])
            xd = torch.from_numpy(x).cuda()
            yd = torch.empty_like(xd)
            p.execute(xd, yd, d)
            p.execute(xd, xd, d)  # in place
            torch.cuda.synchronize()
            _bounds(O.error_stats(yd.cpu().numpy(), ref), ftype, n)
            np.testing.assert_array_equal(xd.cpu().numpy(), yd.cpu().numpy())
