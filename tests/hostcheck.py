"""Test helper: drives the host-emulation build of the engine
(flagfft_b200/_build/hostcheck/libflagfft_hostcheck.so -- the same kernel and
lowering sources compiled with FFB_HOST_EMULATION, kernels run sequentially on
the CPU) through the flagfft.h C ABI with host arrays.  It checks the engine's
index arithmetic, lowering and tables without a GPU; it is not the product
path and proves nothing about GPU execution."""
import ctypes

import numpy as np

_LIB = None


def lib():
    global _LIB
    if _LIB is None:
        from flagfft_b200 import build as B
        path = B.build_hostcheck()
        L = ctypes.CDLL(str(path))
        PH = ctypes.POINTER(ctypes.c_void_p)
        i, vp = ctypes.c_int, ctypes.c_void_p
        L.flagfftPlan1d.argtypes = [PH, i, i, i]
        L.flagfftPlan2d.argtypes = [PH, i, i, i]
        L.flagfftPlanMany.argtypes = [PH, i, ctypes.POINTER(i), ctypes.POINTER(i), i, i, ctypes.POINTER(i), i, i, i, i]
        for f in ("flagfftExecC2C", "flagfftExecZ2Z"):
            getattr(L, f).argtypes = [vp, vp, vp, i]
        for f in ("flagfftExecR2C", "flagfftExecD2Z", "flagfftExecC2R", "flagfftExecZ2D"):
            getattr(L, f).argtypes = [vp, vp, vp]
        L.flagfftDestroy.argtypes = [vp]
        L.flagfftGetPlanDescription.argtypes = [vp]
        L.flagfftGetPlanDescription.restype = ctypes.c_char_p
        _LIB = L
    return _LIB


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def plan1d(n, ftype, batch):
    h = ctypes.c_void_p()
    rc = lib().flagfftPlan1d(ctypes.byref(h), n, ftype, batch)
    assert rc == 0, rc
    return h


def plan2d(n0, n1, ftype):
    h = ctypes.c_void_p()
    rc = lib().flagfftPlan2d(ctypes.byref(h), n0, n1, ftype)
    assert rc == 0, rc
    return h


def describe(h):
    return lib().flagfftGetPlanDescription(h).decode()


def c2c(x, direction, double=False):
    """x: (batch, n) complex; returns the engine's transform."""
    n = x.shape[-1]
    xin = np.ascontiguousarray(x, dtype=np.complex128 if double else np.complex64)
    out = np.empty_like(xin)
    h = plan1d(n, 0x69 if double else 0x29, xin.shape[0])
    fn = lib().flagfftExecZ2Z if double else lib().flagfftExecC2C
    assert fn(h, _p(xin), _p(out), direction) == 0
    lib().flagfftDestroy(h)
    return out


def r2c(x, double=False):
    n = x.shape[-1]
    xin = np.ascontiguousarray(x, dtype=np.float64 if double else np.float32)
    out = np.empty((xin.shape[0], n // 2 + 1), dtype=np.complex128 if double else np.complex64)
    h = plan1d(n, 0x6A if double else 0x2A, xin.shape[0])
    fn = lib().flagfftExecD2Z if double else lib().flagfftExecR2C
    assert fn(h, _p(xin), _p(out)) == 0
    lib().flagfftDestroy(h)
    return out


def c2r(x, n, double=False):
    xin = np.ascontiguousarray(x, dtype=np.complex128 if double else np.complex64)
    out = np.empty((xin.shape[0], n), dtype=np.float64 if double else np.float32)
    h = plan1d(n, 0x6C if double else 0x2C, xin.shape[0])
    fn = lib().flagfftExecZ2D if double else lib().flagfftExecC2R
    assert fn(h, _p(xin), _p(out)) == 0
    lib().flagfftDestroy(h)
    return out


def fft2(x, kind, n1=None, double=False):
    if kind == "c2c_fwd" or kind == "c2c_inv":
        n0, n1 = x.shape
        xin = np.ascontiguousarray(x, dtype=np.complex128 if double else np.complex64)
        out = np.empty_like(xin)
        h = plan2d(n0, n1, 0x69 if double else 0x29)
        fn = lib().flagfftExecZ2Z if double else lib().flagfftExecC2C
        assert fn(h, _p(xin), _p(out), -1 if kind == "c2c_fwd" else 1) == 0
    elif kind == "r2c":
        n0, n1 = x.shape
        xin = np.ascontiguousarray(x, dtype=np.float64 if double else np.float32)
        out = np.empty((n0, n1 // 2 + 1), dtype=np.complex128 if double else np.complex64)
        h = plan2d(n0, n1, 0x6A if double else 0x2A)
        fn = lib().flagfftExecD2Z if double else lib().flagfftExecR2C
        assert fn(h, _p(xin), _p(out)) == 0
    else:
        n0 = x.shape[0]
        xin = np.ascontiguousarray(x, dtype=np.complex128 if double else np.complex64)
        out = np.empty((n0, n1), dtype=np.float64 if double else np.float32)
        h = plan2d(n0, n1, 0x6C if double else 0x2C)
        fn = lib().flagfftExecZ2D if double else lib().flagfftExecC2R
        assert fn(h, _p(xin), _p(out)) == 0
    lib().flagfftDestroy(h)
    return out
