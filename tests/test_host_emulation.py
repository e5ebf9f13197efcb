"""CPU checks of the engine's index arithmetic through its host-emulation
build (the kernel and lowering sources compiled with FFB_HOST_EMULATION; the
kernels run sequentially on the CPU and the TMA box copies are done by hand,
refusing the ones the hardware would refuse for alignment).  Results are
compared with the FP64 oracle.  These tests prove nothing about GPU timing or
memory ordering; they catch layout, stride, ring-slot and table mistakes
before a kernel reaches a GPU."""
import numpy as np
import pytest

import hostcheck as H
from oracle import oracle as O

C2C, R2C, C2R, Z2Z, D2Z, Z2D = 0x29, 0x2A, 0x2C, 0x69, 0x6A, 0x6C


def _rel(a, b):
    a = np.asarray(a, np.complex128).reshape(-1)
    b = np.asarray(b, np.complex128).reshape(-1)
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def _bound(n, double):
    return (1e-15 if double else 5e-7) * max(1.0, np.log2(n)) * 4


def _describe(plan):
    h = plan()
    try:
        return H.describe(h)
    finally:
        H.lib().flagfftDestroy(h)


# (n0, n1, double): the column pass is a TMA column pass of length n0 whose
# groups fill every ring slot (n1 / transforms-per-group > 3)
@pytest.mark.parametrize("n0,n1,double", [(1024, 40, False), (2048, 24, False), (4096, 12, False),
                                          (1536, 20, False), (1024, 20, True), (2048, 10, True),
                                          (1536, 12, True)])
def test_tma_column_pass_2d(n0, n1, double):
    x = O.random_complex(n0 * n1, O.accuracy_seed(C2C, n0, n1), double=True).reshape(n0, n1)
    d = _describe(lambda: H.plan2d(n0, n1, Z2Z if double else C2C))
    assert "tma-columns" in d, d
    for direction, kind in ((-1, "c2c_fwd"), (1, "c2c_inv")):
        ref = O.fft2(x, "c2c", direction)
        got = H.fft2(x, kind, double=double)
        assert _rel(got, ref) < _bound(n0 * n1, double), (kind, _rel(got, ref))


@pytest.mark.parametrize("n,batch,double", [(1 << 20, 1, False), (1 << 20, 2, True)])
def test_tma_column_four_step_c2c(n, batch, double):
    x = O.random_complex(n * batch, O.accuracy_seed(C2C, n, batch), double=True).reshape(batch, n)
    d = _describe(lambda: H.plan1d(n, Z2Z if double else C2C, batch))
    assert "tma-columns" in d, d
    got = H.c2c(x, -1, double)
    ref = np.stack([O.c2c(r, -1) for r in x])
    assert _rel(got, ref) < _bound(n, double)


# a 1536-point column pass in double precision (the 3 * 2^20 real transform)
# and a power-of-two real transform, forward and back
@pytest.mark.parametrize("n,batch,double", [(3 << 19, 2, True), (1 << 21, 1, False)])
def test_tma_column_real_round_trip(n, batch, double):
    x = O.random_normal(n * batch, O.accuracy_seed(R2C, n, batch), double=True).reshape(batch, n)
    spec = H.r2c(x, double)
    ref = np.stack([O.r2c(r) for r in x])
    assert _rel(spec, ref) < _bound(n, double)
    back = H.c2r(ref, n, double)
    assert _rel(back, x * n) < _bound(n, double)


def _server_run(reqs):
    """Submits every (type code, n, batch, direction, input) to one server of
    the host-emulation build and returns the outputs."""
    import ctypes
    L = H.lib()
    vp, i = ctypes.c_void_p, ctypes.c_int
    L.flagfftB200ServerCreate.argtypes = [ctypes.POINTER(vp), ctypes.c_longlong, i]
    L.flagfftB200ServerSubmit.argtypes = [vp, i, i, i, i, vp, vp, ctypes.POINTER(ctypes.c_longlong)]
    L.flagfftB200ServerWait.argtypes = [vp, ctypes.c_longlong, ctypes.POINTER(ctypes.c_double)]
    L.flagfftB200ServerDestroy.argtypes = [vp]
    srv = vp()
    assert L.flagfftB200ServerCreate(ctypes.byref(srv), 1 << 30, 2) == 0
    outs, tickets = [], []
    try:
        for code, n, b, d, x in reqs:
            dbl = code in (Z2Z, D2Z, Z2D)
            if code in (R2C, D2Z):
                y = np.empty((b, n // 2 + 1), np.complex128 if dbl else np.complex64)
            elif code in (C2R, Z2D):
                y = np.empty((b, n), np.float64 if dbl else np.float32)
            else:
                y = np.empty((b, n), np.complex128 if dbl else np.complex64)
            tk = ctypes.c_longlong()
            assert L.flagfftB200ServerSubmit(srv, code, n, b, d, H._p(x), H._p(y), ctypes.byref(tk)) == 0
            outs.append(y)
            tickets.append(tk.value)
        for tk in tickets:
            lat = ctypes.c_double()
            assert L.flagfftB200ServerWait(srv, tk, ctypes.byref(lat)) == 0
    finally:
        L.flagfftB200ServerDestroy(srv)
    return outs


def test_server_real_lengths_without_an_on_chip_core():
    """Real requests whose lowering has widen / take or Hermitian pre / post
    passes around a multi-pass complex transform: every pass runs at the
    request's batch."""
    n_odd, n_even, n_dbl = 30011, 60022, 20011
    x1 = O.random_real(2 * n_odd, 11).reshape(2, n_odd).astype(np.float32)
    x2 = np.fft.rfft(O.random_real(3 * n_even, 12).reshape(3, n_even).astype(np.float64), axis=-1).astype(np.complex64)
    x3 = O.random_real(n_dbl, 13, True).reshape(1, n_dbl).astype(np.float64)
    outs = _server_run([(R2C, n_odd, 2, -1, x1), (C2R, n_even, 3, 1, x2), (D2Z, n_dbl, 1, -1, x3)])
    assert _rel(outs[0], np.stack([O.r2c(r.astype(np.float64)) for r in x1])) < _bound(n_odd, False)
    ref2 = np.stack([O.c2r(r.astype(np.complex128), n_even) for r in x2])
    assert _rel(outs[1], ref2) < _bound(n_even, False)
    assert _rel(outs[2], np.stack([O.r2c(r) for r in x3])) < _bound(n_dbl, True)


# The plan tree's own lowerings (FLAGFFT_TREE_LOWERING=1): a four-step over a
# multi-pass Bluestein child (60022 = 2 x 30011) and Rader chains over
# multi-pass p - 1 transforms (65537: 256 x 256; 40961: 128 x 320).
@pytest.mark.parametrize("n,batch,double,marker", [(60022, 3, False, "transpose"), (65537, 2, False, "rader-gather"),
                                                   (40961, 1, True, "rader-gather")])
def test_tree_lowering(monkeypatch, n, batch, double, marker):
    monkeypatch.setenv("FLAGFFT_TREE_LOWERING", "1")
    x = O.random_complex(n * batch, O.accuracy_seed(C2C, n, batch), double=True).reshape(batch, n)
    d = _describe(lambda: H.plan1d(n, Z2Z if double else C2C, batch))
    assert marker in d, d
    for direction in (-1, 1):
        got = H.c2c(x, direction, double)
        ref = np.stack([O.c2c(r, direction) for r in x])
        assert _rel(got, ref) < _bound(n, double), (direction, _rel(got, ref))


# The one-pass Bluestein's pair form (FLAGFFT_BLUESTEIN_PAIR=1): the two
# CTAs of the cluster emulated phase by phase, each writing half of its
# columns' rows into the other's buffer; N1 = 8, 10 and 12 rows of 2048.
@pytest.mark.parametrize("n,batch,double", [(8009, 2, True), (10007, 2, True), (11003, 1, True), (10007, 2, False)])
def test_bluestein_pair(monkeypatch, n, batch, double):
    monkeypatch.setenv("FLAGFFT_BLUESTEIN_PAIR", "1")
    x = O.random_complex(n * batch, O.accuracy_seed(C2C, n, batch), double=True).reshape(batch, n)
    d = _describe(lambda: H.plan1d(n, Z2Z if double else C2C, batch))
    assert "bluestein-four-step-pair" in d, d
    for direction in (-1, 1):
        got = H.c2c(x, direction, double)
        ref = np.stack([O.c2c(r, direction) for r in x])
        assert _rel(got, ref) < _bound(n, double), (direction, _rel(got, ref))


# 1701's two row-kernel forms: 256 threads a row up to 2048 transforms a
# pass (every radix-9 and radix-7 stage one round), 192 above.
@pytest.mark.parametrize("double", [False, True])
def test_1701_row_forms(double):
    n, batch = 1701, 3
    code = Z2Z if double else C2C
    assert "threads=256 " in _describe(lambda: H.plan1d(n, code, batch))
    assert "threads=192 " in _describe(lambda: H.plan1d(n, code, 2049))
    x = O.random_complex(n * batch, O.accuracy_seed(code, n, batch), double=True).reshape(batch, n)
    for direction in (-1, 1):
        got = H.c2c(x, direction, double)
        ref = np.stack([O.c2c(r, direction) for r in x])
        assert _rel(got, ref) < _bound(n, double), (direction, _rel(got, ref))


def test_server_multi_pass_lengths():
    """Server templates lower their four-step and Bluestein-chain passes in
    the persistent kernel's form (no strided tile / TMA column kernels):
    complex lengths above one CTA, both precisions."""
    reqs = []
    for code, n, b, d, seed in [(C2C, 65536, 2, -1, 21), (C2C, 131072, 1, 1, 22), (Z2Z, 20011, 1, -1, 23),
                                (Z2Z, 32768, 2, 1, 24)]:
        dbl = code == Z2Z
        x = O.random_complex(n * b, seed, double=True).reshape(b, n).astype(np.complex128 if dbl else np.complex64)
        reqs.append((code, n, b, d, x))
    outs = _server_run(reqs)
    for (code, n, b, d, x), y in zip(reqs, outs):
        ref = np.stack([O.c2c(r.astype(np.complex128), d) for r in x])
        assert _rel(y, ref) < _bound(n, code == Z2Z), (code, n, _rel(y, ref))


def test_server_1701_wide_items():
    """1701 requests (their wide 256-thread form) in one persistent launch
    with lengths of other thread counts, both precisions and directions."""
    reqs = []
    for code, n, b, d, seed in [(C2C, 1701, 3, -1, 41), (C2C, 4096, 2, 1, 42), (Z2Z, 1701, 2, 1, 43),
                                (C2C, 1009, 1, -1, 44), (Z2Z, 1701, 1, -1, 45)]:
        dbl = code == Z2Z
        x = O.random_complex(n * b, seed, double=True).reshape(b, n).astype(np.complex128 if dbl else np.complex64)
        reqs.append((code, n, b, d, x))
    outs = _server_run(reqs)
    for (code, n, b, d, x), y in zip(reqs, outs):
        ref = np.stack([O.c2c(r.astype(np.complex128), d) for r in x])
        assert _rel(y, ref) < _bound(n, code == Z2Z), (code, n, _rel(y, ref))


def test_server_real_on_chip_items():
    """Real requests whose transform fits one CTA: the persistent launch runs
    their pack / Hermitian post (R2C) and pre / unpack (C2R) tiles."""
    n1, n2, n3 = 4096, 1000, 998
    x1 = O.random_real(3 * n1, 31).reshape(3, n1).astype(np.float32)
    x2 = np.fft.rfft(O.random_real(2 * n2, 32).reshape(2, n2).astype(np.float64), axis=-1).astype(np.complex64)
    x3 = O.random_real(4 * n3, 33, True).reshape(4, n3).astype(np.float64)
    x4 = np.fft.rfft(O.random_real(2 * n3, 34).reshape(2, n3).astype(np.float64), axis=-1).astype(np.complex128)
    outs = _server_run([(R2C, n1, 3, -1, x1), (C2R, n2, 2, 1, x2), (D2Z, n3, 4, -1, x3), (Z2D, n3, 2, 1, x4)])
    assert _rel(outs[0], np.stack([O.r2c(r.astype(np.float64)) for r in x1])) < _bound(n1, False)
    assert _rel(outs[1], np.stack([O.c2r(r.astype(np.complex128), n2) for r in x2])) < _bound(n2, False)
    assert _rel(outs[2], np.stack([O.r2c(r) for r in x3])) < _bound(n3, True)
    assert _rel(outs[3], np.stack([O.c2r(r, n3) for r in x4])) < _bound(n3, True)
