"""flagfft_b200 -- Python binding of libflagfft.so, the sm_100a FFT engine behind
the flagfft.h C ABI.

The binding mirrors the C API one to one (``plan1d`` / ``plan2d`` / ``plan3d`` /
``plan_many`` -> ``flagfftPlan*``, ``Plan.exec_*`` -> ``flagfftExec*``,
``Plan.set_stream`` / ``Plan.destroy`` / ``Plan.description``), takes device
pointers as integers or CUDA torch tensors, and raises ``FlagFFTError`` with the
C status code on any non-success result.  There is no fallback: the shared
library is loaded on first use (so that ``python -m flagfft_b200.build`` works
on a fresh tree) and, if it is missing, that first use raises ImportError.
"""
from __future__ import annotations

import ctypes
import json
import os
from pathlib import Path

__all__ = [
    "FlagFFTError", "Plan", "plan1d", "plan2d", "plan3d", "plan_many", "plan_batch", "Server", "tune", "tune_candidates", "planner_tree", "library_path",
    "C2C", "Z2Z", "R2C", "D2Z", "C2R", "Z2D", "FORWARD", "INVERSE", "STATUS",
]

_PKG = Path(__file__).resolve().parent
_LIB_PATH = Path(os.environ.get("FLAGFFT_B200_LIB", _PKG / "libflagfft.so"))

C2C, Z2Z, R2C, D2Z, C2R, Z2D = 0x29, 0x69, 0x2A, 0x6A, 0x2C, 0x6C
FORWARD, INVERSE = -1, 1
STATUS = {
    0: "FLAGFFT_SUCCESS", 1: "FLAGFFT_INVALID_PLAN", 2: "FLAGFFT_ALLOC_FAILED", 3: "FLAGFFT_INVALID_TYPE",
    4: "FLAGFFT_INVALID_VALUE", 5: "FLAGFFT_INTERNAL_ERROR", 6: "FLAGFFT_EXEC_FAILED", 7: "FLAGFFT_SETUP_FAILED",
    8: "FLAGFFT_INVALID_SIZE", 9: "FLAGFFT_UNALIGNED_DATA", 10: "FLAGFFT_INCOMPLETE_PARAMETER_LIST",
    11: "FLAGFFT_INVALID_DEVICE", 12: "FLAGFFT_PARSE_ERROR", 13: "FLAGFFT_NO_WORKSPACE", 14: "FLAGFFT_NOT_SUPPORTED",
}
TYPE_NAMES = {C2C: "C2C", Z2Z: "Z2Z", R2C: "R2C", D2Z: "D2Z", C2R: "C2R", Z2D: "Z2D"}


class FlagFFTError(RuntimeError):
    def __init__(self, code: int, what: str):
        self.code = code
        super().__init__(f"{what}: {STATUS.get(code, code)}")


def library_path() -> Path:
    return _LIB_PATH


def _load():
    if not _LIB_PATH.exists():
        raise ImportError(f"libflagfft.so not built at {_LIB_PATH}; run `python -m flagfft_b200.build`")
    lib = ctypes.CDLL(str(_LIB_PATH))
    H = ctypes.c_void_p
    PH = ctypes.POINTER(ctypes.c_void_p)
    i, vp, cp = ctypes.c_int, ctypes.c_void_p, ctypes.c_char_p
    ip = ctypes.POINTER(ctypes.c_int)
    sigs = {
        "flagfftPlan1d": (i, [PH, i, i, i]),
        "flagfftPlan2d": (i, [PH, i, i, i]),
        "flagfftPlan3d": (i, [PH, i, i, i, i]),
        "flagfftPlanMany": (i, [PH, i, ip, ip, i, i, ip, i, i, i, i]),
        "flagfftExecC2C": (i, [H, vp, vp, i]),
        "flagfftExecZ2Z": (i, [H, vp, vp, i]),
        "flagfftExecR2C": (i, [H, vp, vp]),
        "flagfftExecD2Z": (i, [H, vp, vp]),
        "flagfftExecC2R": (i, [H, vp, vp]),
        "flagfftExecZ2D": (i, [H, vp, vp]),
        "flagfftSetStream": (i, [H, vp]),
        "flagfftDestroy": (i, [H]),
        "flagfftGetPlanDescription": (cp, [H]),
        "flagfftB200Version": (cp, []),
        "flagfftB200PlannerTree": (i, [i, i, ctypes.c_longlong, cp, i]),
        "flagfftB200PlanJson": (cp, [H]),
        "flagfftB200LaunchCount": (i, [H, i]),
        "flagfftB200PlanBatch": (i, [PH, i, ip, ip, i]),
        "flagfftB200ServerCreate": (i, [PH, ctypes.c_longlong, i]),
        "flagfftB200ServerPrepare": (i, [H, i, i, i]),
        "flagfftB200ServerSubmit": (i, [H, i, i, i, i, vp, vp, ctypes.POINTER(ctypes.c_longlong)]),
        "flagfftB200ServerWait": (i, [H, ctypes.c_longlong, ctypes.POINTER(ctypes.c_double)]),
        "flagfftB200ServerStats": (i, [H, ctypes.POINTER(ctypes.c_longlong), ctypes.POINTER(ctypes.c_longlong),
                                       ctypes.POINTER(ctypes.c_longlong)]),
        "flagfftB200ServerWaitFor": (i, [H, ctypes.c_longlong, ctypes.c_double, ctypes.POINTER(ctypes.c_double),
                                         ctypes.POINTER(i)]),
        "flagfftB200ServerOverlap": (i, [H, ctypes.POINTER(ctypes.c_longlong), ctypes.POINTER(ctypes.c_longlong)]),
        "flagfftB200ServerDestroy": (i, [H]),
        "flagfftB200DeviceWaitFailures": (i, [ctypes.POINTER(ctypes.c_longlong)]),
        "flagfftB200Tune": (i, [i, i, i, i, cp, cp, i, ctypes.POINTER(ctypes.c_double)]),
        "flagfftB200TuneCandidates": (i, [i, i, cp, i]),
    }
    for name, (res, args) in sigs.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


_LIB = None


def _lib():
    global _LIB
    if _LIB is None:
        _LIB = _load()
    return _LIB


def __getattr__(name):
    if name == "LIB":
        return _lib()
    raise AttributeError(f"module {__name__!r} has no attribute {name!r}")


def _check(code: int, what: str) -> None:
    if code != 0:
        raise FlagFFTError(code, what)


def _ptr(x) -> int:
    """Device address of a CUDA tensor, or an integer address as given."""
    if x is None:
        return 0
    if isinstance(x, int):
        return x
    if hasattr(x, "data_ptr"):
        if hasattr(x, "is_cuda") and not x.is_cuda:
            raise ValueError("flagfft_b200 executes on device memory; got a host tensor")
        return x.data_ptr()
    raise TypeError(f"cannot take a device pointer of {type(x).__name__}")


def _stream_handle(stream) -> int:
    if stream is None:
        return 0
    if isinstance(stream, int):
        return stream
    return int(getattr(stream, "cuda_stream", stream))


class Plan:
    """A flagfftHandle.  Destroyed explicitly with destroy() or on garbage collection."""

    def __init__(self, handle: int, ftype: int, shape: tuple[int, ...], batch: int):
        self._h = ctypes.c_void_p(handle)
        self.type = ftype
        self.shape = shape
        self.batch = batch

    @property
    def handle(self) -> int:
        return self._h.value or 0

    def _exec(self, fn: str, idata, odata, *extra) -> None:
        _check(getattr(_lib(), fn)(self._h, ctypes.c_void_p(_ptr(idata)), ctypes.c_void_p(_ptr(odata)), *extra), fn)

    def exec_c2c(self, idata, odata, direction: int) -> None:
        self._exec("flagfftExecC2C", idata, odata, direction)

    def exec_z2z(self, idata, odata, direction: int) -> None:
        self._exec("flagfftExecZ2Z", idata, odata, direction)

    def exec_r2c(self, idata, odata) -> None:
        self._exec("flagfftExecR2C", idata, odata)

    def exec_d2z(self, idata, odata) -> None:
        self._exec("flagfftExecD2Z", idata, odata)

    def exec_c2r(self, idata, odata) -> None:
        self._exec("flagfftExecC2R", idata, odata)

    def exec_z2d(self, idata, odata) -> None:
        self._exec("flagfftExecZ2D", idata, odata)

    def execute(self, idata, odata, direction: int = FORWARD) -> None:
        """Dispatch on the plan's type (direction only matters for C2C / Z2Z)."""
        t = self.type
        if t == C2C:
            self.exec_c2c(idata, odata, direction)
        elif t == Z2Z:
            self.exec_z2z(idata, odata, direction)
        elif t == R2C:
            self.exec_r2c(idata, odata)
        elif t == D2Z:
            self.exec_d2z(idata, odata)
        elif t == C2R:
            self.exec_c2r(idata, odata)
        else:
            self.exec_z2d(idata, odata)

    def set_stream(self, stream) -> None:
        _check(_lib().flagfftSetStream(self._h, ctypes.c_void_p(_stream_handle(stream))), "flagfftSetStream")

    def description(self) -> str:
        s = _lib().flagfftGetPlanDescription(self._h)
        if s is None:
            raise FlagFFTError(1, "flagfftGetPlanDescription")
        return s.decode()

    def tree(self) -> dict:
        s = _lib().flagfftB200PlanJson(self._h)
        if s is None:
            raise FlagFFTError(1, "flagfftB200PlanJson")
        return json.loads(s.decode())

    def launch_count(self, direction: int = FORWARD) -> int:
        return int(_lib().flagfftB200LaunchCount(self._h, direction))

    def destroy(self) -> None:
        if self._h.value:
            _check(_lib().flagfftDestroy(self._h), "flagfftDestroy")
            self._h = ctypes.c_void_p(0)

    def __del__(self):
        try:
            if self._h.value:
                _lib().flagfftDestroy(self._h)
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.destroy()


def plan1d(nx: int, ftype: int, batch: int = 1) -> Plan:
    h = ctypes.c_void_p(0)
    _check(_lib().flagfftPlan1d(ctypes.byref(h), nx, ftype, batch), "flagfftPlan1d")
    return Plan(h.value, ftype, (nx,), batch)


def plan2d(nx: int, ny: int, ftype: int) -> Plan:
    h = ctypes.c_void_p(0)
    _check(_lib().flagfftPlan2d(ctypes.byref(h), nx, ny, ftype), "flagfftPlan2d")
    return Plan(h.value, ftype, (nx, ny), 1)


def plan3d(nx: int, ny: int, nz: int, ftype: int) -> Plan:
    h = ctypes.c_void_p(0)
    _check(_lib().flagfftPlan3d(ctypes.byref(h), nx, ny, nz, ftype), "flagfftPlan3d")
    return Plan(h.value, ftype, (nx, ny, nz), 1)


def plan_many(n, inembed, istride: int, idist: int, onembed, ostride: int, odist: int, ftype: int,
              batch: int) -> Plan:
    rank = len(n)
    arr = lambda v: None if v is None else (ctypes.c_int * rank)(*v)  # noqa: E731
    h = ctypes.c_void_p(0)
    _check(_lib().flagfftPlanMany(ctypes.byref(h), rank, arr(n), arr(inembed), istride, idist, arr(onembed), ostride,
                               odist, ftype, batch), "flagfftPlanMany")
    return Plan(h.value, ftype, tuple(n), batch)


def plan_batch(lengths, counts, ftype: int = C2C) -> Plan:
    """Batch plan (flagfftB200PlanBatch): counts[g] transforms of length
    lengths[g], packed group after group; execute() runs all of them."""
    lengths, counts = list(lengths), list(counts)
    if len(lengths) != len(counts) or not lengths:
        raise ValueError("lengths and counts must be non-empty and of equal length")
    g = len(lengths)
    h = ctypes.c_void_p(0)
    _check(_lib().flagfftB200PlanBatch(ctypes.byref(h), g, (ctypes.c_int * g)(*lengths), (ctypes.c_int * g)(*counts),
                                       ftype), "flagfftB200PlanBatch")
    total = sum(l * c for l, c in zip(lengths, counts))
    return Plan(h.value, ftype, (total,), 1)


class Server:
    """Request server (flagfftB200ServerCreate): continuous batching of
    transforms of mixed type, length and batch on device buffers."""

    def __init__(self, hbm_budget_bytes: int = 40 << 30, max_ticks: int = 4):
        h = ctypes.c_void_p(0)
        _check(_lib().flagfftB200ServerCreate(ctypes.byref(h), hbm_budget_bytes, max_ticks), "flagfftB200ServerCreate")
        self._h = h

    def prepare(self, ftype: int, n: int, direction: int = FORWARD) -> None:
        _check(_lib().flagfftB200ServerPrepare(self._h, ftype, n, direction), "flagfftB200ServerPrepare")

    def submit(self, ftype: int, n: int, batch: int, idata, odata, direction: int = FORWARD) -> int:
        t = ctypes.c_longlong(0)
        _check(_lib().flagfftB200ServerSubmit(self._h, ftype, n, batch, direction, ctypes.c_void_p(_ptr(idata)),
                                              ctypes.c_void_p(_ptr(odata)), ctypes.byref(t)), "flagfftB200ServerSubmit")
        return t.value

    def wait(self, ticket: int, timeout_s: float | None = None) -> float:
        """Blocks until the request finished (at most timeout_s seconds when
        given: TimeoutError then, and the ticket stays valid); returns its
        latency in ms."""
        ms = ctypes.c_double(0)
        if timeout_s is None:
            _check(_lib().flagfftB200ServerWait(self._h, ticket, ctypes.byref(ms)), "flagfftB200ServerWait")
            return ms.value
        done = ctypes.c_int(0)
        _check(_lib().flagfftB200ServerWaitFor(self._h, ticket, timeout_s * 1e3, ctypes.byref(ms), ctypes.byref(done)),
               "flagfftB200ServerWaitFor")
        if not done.value:
            raise TimeoutError(f"request {ticket} not finished after {timeout_s} s")
        return ms.value

    def stats(self) -> dict:
        c, t, u = ctypes.c_longlong(), ctypes.c_longlong(), ctypes.c_longlong()
        _check(_lib().flagfftB200ServerStats(self._h, ctypes.byref(c), ctypes.byref(t), ctypes.byref(u)),
               "flagfftB200ServerStats")
        m, a = ctypes.c_longlong(), ctypes.c_longlong()
        _check(_lib().flagfftB200ServerOverlap(self._h, ctypes.byref(m), ctypes.byref(a)), "flagfftB200ServerOverlap")
        return {"completed": c.value, "ticks": t.value, "bytes_in_use": u.value, "max_ticks_in_flight": m.value,
                "admitted_while_busy": a.value}

    def close(self) -> None:
        if self._h:
            _lib().flagfftB200ServerDestroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def tune(n: int, ftype: int = C2C, batch: int = 1, direction: int = FORWARD, db_path: str | None = None) -> dict:
    """Autotune one request shape (flagfftB200Tune) and store the fastest tree
    in the tune database; returns the report (every candidate's time)."""
    buf = ctypes.create_string_buffer(1 << 20)
    ms = ctypes.c_double(0)
    _check(_lib().flagfftB200Tune(n, ftype, batch, direction, db_path.encode() if db_path else None, buf, len(buf),
                                  ctypes.byref(ms)), "flagfftB200Tune")
    return json.loads(buf.value.decode())


def tune_candidates(n: int, is_double: bool = False) -> list:
    """The autotuner's candidate trees for a length (host only)."""
    need = _lib().flagfftB200TuneCandidates(n, int(is_double), None, 0)
    if need < 0:
        raise FlagFFTError(4, f"no candidates for length {n}")
    buf = ctypes.create_string_buffer(need + 1)
    _lib().flagfftB200TuneCandidates(n, int(is_double), buf, need + 1)
    return json.loads(buf.value.decode())


def planner_tree(n: int, is_double: bool = False, smem_bytes: int = 0) -> dict:
    """Plan tree for a 1-D complex length, host only (no GPU)."""
    need = _lib().flagfftB200PlannerTree(n, int(is_double), smem_bytes, None, 0)
    if need < 0:
        raise FlagFFTError(4, f"planner rejected length {n}")
    buf = ctypes.create_string_buffer(need + 1)
    _lib().flagfftB200PlannerTree(n, int(is_double), smem_bytes, buf, need + 1)
    return json.loads(buf.value.decode())


def device_wait_failures() -> int:
    """Bounded device-side waits that gave up on the current device (a copy
    that never landed); 0 in normal operation."""
    v = ctypes.c_longlong(0)
    _check(_lib().flagfftB200DeviceWaitFailures(ctypes.byref(v)), "flagfftB200DeviceWaitFailures")
    return v.value


def version() -> str:
    return _lib().flagfftB200Version().decode()
