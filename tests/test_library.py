"""libflagfft.so loads, exports every entry point include/*.h declares, and
validates arguments exactly as the reference C API does -- all host-side
checks that return before any device work (src/exec/c_api_plan.cpp:274-336,
src/exec/c_api_exec.cpp)."""
import ctypes
import re
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent


def declared_symbols():
    names = set()
    for h in (ROOT / "include").glob("*.h"):
        for m in re.finditer(r"FLAGFFT_API\s+[\w\s\*]+?\b(flagfft\w+)\s*\(", h.read_text()):
            names.add(m.group(1))
    return names


def test_header_declares_reference_entry_points():
    ref = {"flagfftPlan1d", "flagfftPlan2d", "flagfftPlan3d", "flagfftPlanMany", "flagfftExecC2C",
           "flagfftExecZ2Z", "flagfftExecR2C", "flagfftExecD2Z", "flagfftExecC2R", "flagfftExecZ2D",
           "flagfftSetStream", "flagfftDestroy", "flagfftGetPlanDescription"}
    assert ref <= declared_symbols()


def test_library_exports_every_declared_symbol(ffb):
    lib = ctypes.CDLL(str(ffb.library_path()))
    missing = [s for s in sorted(declared_symbols()) if not hasattr(lib, s)]
    assert not missing


def test_enum_values_match_reference(ffb):
    """cuFFT-valued type codes (include/flagfft.h:28-35)."""
    assert (ffb.R2C, ffb.C2R, ffb.C2C, ffb.D2Z, ffb.Z2D, ffb.Z2Z) == (0x2A, 0x2C, 0x29, 0x6A, 0x6C, 0x69)
    assert ffb.STATUS[14] == "FLAGFFT_NOT_SUPPORTED"


def _plan_many(ffb, rank, n, istride=1, idist=None, ostride=1, odist=None, ftype=0x29, batch=1):
    h = ctypes.c_void_p(123)
    arr = (ctypes.c_int * rank)(*n)
    tot = 1
    for v in n:
        tot *= v
    rc = ffb.LIB.flagfftPlanMany(ctypes.byref(h), rank, arr, None, istride, idist or tot, None, ostride,
                                 odist or tot, ftype, batch)
    return rc, h.value


def test_invalid_arguments_before_device(ffb):
    h = ctypes.c_void_p(1)
    assert ffb.LIB.flagfftPlan1d(None, 256, ffb.C2C, 1) == 4               # INVALID_VALUE
    assert ffb.LIB.flagfftPlan1d(ctypes.byref(h), 0, ffb.C2C, 1) == 8      # INVALID_SIZE
    assert h.value is None
    assert ffb.LIB.flagfftPlan1d(ctypes.byref(h), 16, ffb.C2C, 0) == 4     # batch <= 0
    assert ffb.LIB.flagfftPlan1d(ctypes.byref(h), 16, 0x11, 1) == 3        # INVALID_TYPE
    assert ffb.LIB.flagfftPlan2d(ctypes.byref(h), 0, 32, ffb.C2C) == 8
    assert ffb.LIB.flagfftPlan3d(ctypes.byref(h), 0, 16, 8, ffb.C2C) == 8
    assert ffb.LIB.flagfftPlan3d(None, 32, 16, 8, ffb.C2C) == 4


def test_unsupported_layouts(ffb):
    # 3-D and strided / padded 2-D are NOT_SUPPORTED (ctest/test_plan.cpp:104-169)
    for t in (0x29, 0x69, 0x2A, 0x6A, 0x2C, 0x6C):
        h = ctypes.c_void_p(5)
        assert ffb.LIB.flagfftPlan3d(ctypes.byref(h), 32, 16, 8, t) == 14
        assert h.value is None
    assert _plan_many(ffb, 2, [64, 32], istride=2)[0] == 14
    assert _plan_many(ffb, 2, [64, 32], idist=64 * 32 + 16)[0] == 14
    assert _plan_many(ffb, 2, [64, 32], odist=64 * 32 + 16)[0] == 14
    assert _plan_many(ffb, 1, [64], istride=2)[0] == 14


def test_exec_on_null_plan(ffb):
    assert ffb.LIB.flagfftExecC2C(None, None, None, -1) == 1
    assert ffb.LIB.flagfftDestroy(None) == 1
    assert ffb.LIB.flagfftSetStream(None, None) == 1
    assert ffb.LIB.flagfftGetPlanDescription(None) is None
    assert ffb.LIB.flagfftB200LaunchCount(None, -1) == -1


def test_version_string(ffb):
    assert "sm_100a" in ffb.version()


def test_batch_plan_argument_checks(ffb):
    """flagfftB200PlanBatch rejects bad arguments before touching a device."""
    import ctypes as C
    h = C.c_void_p(7)
    ints = lambda *v: (C.c_int * len(v))(*v)  # noqa: E731
    L = ffb.LIB
    assert L.flagfftB200PlanBatch(None, 1, ints(16), ints(1), ffb.C2C) == 4
    assert L.flagfftB200PlanBatch(C.byref(h), 0, ints(16), ints(1), ffb.C2C) == 4 and h.value is None
    assert L.flagfftB200PlanBatch(C.byref(h), 1, None, ints(1), ffb.C2C) == 4
    assert L.flagfftB200PlanBatch(C.byref(h), 1, ints(16), ints(1), ffb.R2C) == 3
    assert L.flagfftB200PlanBatch(C.byref(h), 2, ints(16, 0), ints(1, 1), ffb.C2C) == 8
    assert L.flagfftB200PlanBatch(C.byref(h), 2, ints(16, 32), ints(1, 0), ffb.Z2Z) == 4


def test_tune_candidates_host_only(ffb):
    """The autotuner's candidates: the default tree first, distinct, every
    one a tree of the requested length."""
    for n, dbl in ((4096, False), (1009, False), (30030, True), (67, False)):
        cands = ffb.tune_candidates(n, dbl)
        assert cands and cands[0] == ffb.planner_tree(n, dbl)
        keys = [repr(c) for c in cands]
        assert len(set(keys)) == len(keys)
        assert all(c["length"] == n for c in cands)
