"""ORACLE -- test infrastructure only.

Only tests/, ``__graft_entry__.smoke()`` and bench.py's ``cpu_baseline`` leg may
import this module, and only as the checker.  The product (``flagfft_b200`` and
``libflagfft.so``) never imports, links or calls anything under ``oracle/``.

Python side of the oracle:

* ``c2c / r2c / c2r / fft2`` -- ctypes calls into ``libffo.so`` (``ffo.c``), the
  CPU restatement of the reference's Exec algorithms, in FP64 (``precision=
  "f64"``, the oracle proper) or with the reference's float tables and float
  arithmetic (``precision="f32"``, an estimate of the reference's own FP32
  output).
* ``StableRng`` / ``accuracy_seed`` / input generators -- restate the
  reference test harness's deterministic inputs (ctest/flagfft_test.h:390-455).
* ``error_stats`` / ``accuracy_limits`` -- restate its normwise error metric
  and limits (ctest/flagfft_test.h:222-320).
* ``default_plan`` -- a simple valid plan tree for any length, used when a
  test does not supply the reference planner's own tree (the FP64 result does
  not depend on the tree; only the f32 estimate does).
"""
from __future__ import annotations

import ctypes
import json
import math
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
_LIB = None

C2C, Z2Z, R2C, D2Z, C2R, Z2D = 0x29, 0x69, 0x2A, 0x6A, 0x2C, 0x6C
SUPPORTED_RADICES = (19, 17, 16, 15, 13, 12, 11, 10, 9, 8, 7, 6, 5, 4, 3, 2)


def build() -> Path:
    """Compile libffo.so with the Makefile beside this file (idempotent)."""
    subprocess.run(["make", "-s", "-C", str(HERE), "all"], check=True)
    return HERE / "libffo.so"


def lib():
    global _LIB
    if _LIB is None:
        path = HERE / "libffo.so"
        if not path.exists():
            build()
        _LIB = ctypes.CDLL(str(path))
        i64, vp, ci = ctypes.c_int64, ctypes.c_void_p, ctypes.c_int
        for sfx in ("_d", "_f", "_l"):
            getattr(_LIB, "ffo_c2c" + sfx).argtypes = [vp, vp, vp, i64, i64, i64, ci]
            getattr(_LIB, "ffo_r2c" + sfx).argtypes = [vp, vp, vp, i64, i64, i64]
            getattr(_LIB, "ffo_c2r" + sfx).argtypes = [vp, vp, vp, i64, i64, i64]
            getattr(_LIB, "ffo_2d" + sfx).argtypes = [ci, vp, vp, i64, i64, vp, vp, i64, ci]
        _LIB.ffo_naive_dft.argtypes = [vp, vp, i64, ci]
    return _LIB


# ----------------------------------------------------------------------------
# plan trees (reference JSON node shape, src/utils/plan_json.cpp:18-57)
# ----------------------------------------------------------------------------

def plan_code(node: dict) -> np.ndarray:
    """Flatten a plan-tree dict into the int64 preorder code ffo.c parses."""
    out: list[int] = []

    def rec(nd):
        kind = nd["kind"]
        if kind == "ct_leaf":
            out.extend([0, nd["length"], len(nd["factors"]), *nd["factors"]])
        elif kind == "four_step":
            out.extend([1, nd["length"], nd["n1"], nd["n2"]])
            rec(nd["row"])
            rec(nd["col"])
        elif kind == "bluestein":
            out.extend([2, nd["length"], nd["conv_length"]])
            rec(nd["fft_plan"])
        elif kind == "rader":
            out.extend([3, nd["length"], nd["root"]])
            rec(nd["conv_plan"])
        elif kind == "direct_dft":
            out.extend([4, nd["length"]])
        else:
            raise ValueError(f"unknown plan node kind {kind}")

    rec(node)
    return np.asarray(out, dtype=np.int64)


def _smooth_factors(n: int) -> list[int] | None:
    f, r = [], n
    while r > 1:
        for x in SUPPORTED_RADICES:
            if r % x == 0:
                f.append(x)
                r //= x
                break
        else:
            return None
    return f


def _is_prime(n: int) -> bool:
    if n < 2:
        return False
    if n % 2 == 0:
        return n == 2
    d = 3
    while d * d <= n:
        if n % d == 0:
            return False
        d += 2
    return True


def primitive_root(p: int) -> int:
    """Smallest primitive root mod p (src/plan/rader_utils.cpp:55-76)."""
    if p == 2:
        return 1
    phi, fac, t, d = p - 1, [], p - 1, 2
    while d * d <= t:
        if t % d == 0:
            fac.append(d)
            while t % d == 0:
                t //= d
        d += 1
    if t > 1:
        fac.append(t)
    for g in range(2, p):
        if all(pow(g, phi // q, p) != 1 for q in fac):
            return g
    raise ValueError("no primitive root")


def default_plan(n: int) -> dict:
    """A valid plan tree for any n: leaf up to 4096, balanced four-step above,
    Bluestein for lengths with a prime factor above 19."""
    f = _smooth_factors(n)
    if f is not None and n <= 4096:
        return {"kind": "ct_leaf", "length": n, "factors": f}
    if f is not None:
        best = None
        for n1 in range(2, int(math.isqrt(n)) + 1):
            if n % n1 == 0:
                best = n1
        if best is None:
            return {"kind": "ct_leaf", "length": n, "factors": f}
        return {"kind": "four_step", "length": n, "n1": best, "n2": n // best,
                "row": default_plan(best), "col": default_plan(n // best)}
    if n <= 64:
        return {"kind": "direct_dft", "length": n}
    m = 1
    while m < 2 * n - 1:
        m <<= 1
    return {"kind": "bluestein", "length": n, "conv_length": m, "fft_plan": default_plan(m)}


# ----------------------------------------------------------------------------
# transforms
# ----------------------------------------------------------------------------

def _ptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.c_void_p)


_PRECISIONS = {"f64": ("_d", np.float64, np.complex128), "f32": ("_f", np.float32, np.complex64),
               "f80": ("_l", np.longdouble, np.clongdouble)}


def _real_dtype(precision: str):
    return _PRECISIONS[precision][1]


def _cplx_dtype(precision: str):
    return _PRECISIONS[precision][2]


def _fn(name: str, precision: str):
    return getattr(lib(), name + _PRECISIONS[precision][0])


def c2c(x: np.ndarray, direction: int, plan: dict | None = None, precision: str = "f64") -> np.ndarray:
    """Batched C2C over the last axis (unnormalized inverse)."""
    x = np.asarray(x)
    n = x.shape[-1]
    plan = plan or default_plan(n)
    rd = _real_dtype(precision)
    cd = _cplx_dtype(precision)
    xin = np.ascontiguousarray(x.reshape(-1, n), dtype=cd)
    out = np.empty_like(xin)
    code = plan_code(plan)
    fn = _fn("ffo_c2c", precision)
    rc = fn(_ptr(code), _ptr(xin.view(rd)), _ptr(out.view(rd)), xin.shape[0], n, n, int(direction))
    if rc != 0:
        raise ValueError("oracle rejected the plan tree")
    return out.reshape(x.shape)


def r2c(x: np.ndarray, plan: dict | None = None, precision: str = "f64") -> np.ndarray:
    x = np.asarray(x)
    n = x.shape[-1]
    plan = plan or default_plan(n)
    rd = _real_dtype(precision)
    cd = _cplx_dtype(precision)
    xin = np.ascontiguousarray(x.reshape(-1, n), dtype=rd)
    half = n // 2 + 1
    out = np.empty((xin.shape[0], half), dtype=cd)
    code = plan_code(plan)
    fn = _fn("ffo_r2c", precision)
    if fn(_ptr(code), _ptr(xin), _ptr(out.view(rd)), xin.shape[0], n, half) != 0:
        raise ValueError("oracle rejected the plan tree")
    return out.reshape(*x.shape[:-1], half)


def c2r(x: np.ndarray, n: int, plan: dict | None = None, precision: str = "f64") -> np.ndarray:
    x = np.asarray(x)
    half = n // 2 + 1
    assert x.shape[-1] == half
    plan = plan or default_plan(n)
    rd = _real_dtype(precision)
    cd = _cplx_dtype(precision)
    xin = np.ascontiguousarray(x.reshape(-1, half), dtype=cd)
    out = np.empty((xin.shape[0], n), dtype=rd)
    code = plan_code(plan)
    fn = _fn("ffo_c2r", precision)
    if fn(_ptr(code), _ptr(xin.view(rd)), _ptr(out), xin.shape[0], half, n) != 0:
        raise ValueError("oracle rejected the plan tree")
    return out.reshape(*x.shape[:-1], n)


def fft2(x: np.ndarray, kind: str, direction: int = -1, n1: int | None = None,
         row_plan: dict | None = None, col_plan: dict | None = None, precision: str = "f64") -> np.ndarray:
    """2-D RTRT over the last two axes. kind: 'c2c', 'r2c' or 'c2r' (for c2r pass n1)."""
    x = np.asarray(x)
    n0 = x.shape[-2]
    if kind == "c2r":
        assert n1 is not None
    else:
        n1 = x.shape[-1]
    h1 = n1 // 2 + 1
    row_plan = row_plan or default_plan(n1)
    col_plan = col_plan or default_plan(n0)
    rd = _real_dtype(precision)
    cd = _cplx_dtype(precision)
    k = {"c2c": 0, "r2c": 1, "c2r": 2}[kind]
    if k == 1:
        xin = np.ascontiguousarray(x.reshape(-1, n0, n1), dtype=rd)
        out = np.empty((xin.shape[0], n0, h1), dtype=cd)
        outshape = (*x.shape[:-2], n0, h1)
    elif k == 2:
        xin = np.ascontiguousarray(x.reshape(-1, n0, h1), dtype=cd)
        out = np.empty((xin.shape[0], n0, n1), dtype=rd)
        outshape = (*x.shape[:-2], n0, n1)
    else:
        xin = np.ascontiguousarray(x.reshape(-1, n0, n1), dtype=cd)
        out = np.empty_like(xin)
        outshape = x.shape
    rc_, cc_ = plan_code(row_plan), plan_code(col_plan)
    fn = _fn("ffo_2d", precision)
    if fn(k, _ptr(rc_), _ptr(cc_), n0, n1, _ptr(xin), _ptr(out), xin.shape[0], int(direction)) != 0:
        raise ValueError("oracle rejected the plan tree")
    return out.reshape(outshape)


def naive_dft(x: np.ndarray, direction: int) -> np.ndarray:
    """O(n^2) long-double DFT of one 1-D complex vector."""
    xin = np.ascontiguousarray(x, dtype=np.complex128)
    out = np.empty_like(xin)
    lib().ffo_naive_dft(_ptr(xin.view(np.float64)), _ptr(out.view(np.float64)), xin.shape[-1], int(direction))
    return out


# ----------------------------------------------------------------------------
# deterministic inputs (ctest/flagfft_test.h:390-455)
# ----------------------------------------------------------------------------

_M64 = (1 << 64) - 1


class StableRng:
    """splitmix64 stream; signed_unit() = uniform [-1, 1) from 53 mantissa bits."""

    def __init__(self, seed: int):
        self.state = seed & _M64

    def next_u64(self) -> int:
        self.state = (self.state + 0x9E3779B97F4A7C15) & _M64
        v = self.state
        v = ((v ^ (v >> 30)) * 0xBF58476D1CE4E5B9) & _M64
        v = ((v ^ (v >> 27)) * 0x94D049BB133111EB) & _M64
        return v ^ (v >> 31)

    def signed_unit(self) -> float:
        return ((self.next_u64() >> 11) * (1.0 / 9007199254740992.0)) * 2.0 - 1.0


def signed_units(seed: int, count: int) -> np.ndarray:
    """Vectorised StableRng(seed).signed_unit() x count (identical stream)."""
    idx = np.arange(1, count + 1, dtype=np.uint64)
    with np.errstate(over="ignore"):
        s = np.uint64(seed & _M64) + idx * np.uint64(0x9E3779B97F4A7C15)
        v = s
        v = (v ^ (v >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        v = (v ^ (v >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        v = v ^ (v >> np.uint64(31))
    bits = (v >> np.uint64(11)).astype(np.float64)
    return bits * (1.0 / 9007199254740992.0) * 2.0 - 1.0


def accuracy_seed(ftype: int, n: int, batch: int, variant: int = 0) -> int:
    """ctest/flagfft_test.h:413-417."""
    return (0x4654464654455354 ^ (ftype << 48) ^ (n << 16) ^ batch ^ ((variant * 0x9E3779B97F4A7C15) & _M64)) & _M64


def random_complex(count: int, seed: int, double: bool = False) -> np.ndarray:
    """Interleaved re/im draws from one stream (random_complex / random_double_complex)."""
    u = signed_units(seed, 2 * count)
    z = u[0::2] + 1j * u[1::2]
    return z.astype(np.complex128 if double else np.complex64)


def random_real(count: int, seed: int, double: bool = False) -> np.ndarray:
    u = signed_units(seed, count)
    return u.astype(np.float64 if double else np.float32)


def random_normal(count: int, seed: int, double: bool = False) -> np.ndarray:
    """N(0,1) by Box-Muller on the same splitmix64 stream (pairs of draws)."""
    m = (count + 1) // 2
    u = signed_units(seed, 2 * m)
    u1 = (u[0::2] + 1.0) * 0.5
    u2 = (u[1::2] + 1.0) * 0.5
    u1 = np.where(u1 <= 0.0, 2.0 ** -53, u1)
    r = np.sqrt(-2.0 * np.log(u1))
    z = np.concatenate([r * np.cos(2 * np.pi * u2), r * np.sin(2 * np.pi * u2)])[:count]
    return z.astype(np.float64 if double else np.float32)


# ----------------------------------------------------------------------------
# error metric and limits (ctest/flagfft_test.h:222-320)
# ----------------------------------------------------------------------------

def error_stats(value: np.ndarray, reference: np.ndarray) -> dict:
    """Per-batch normwise relative L2 / Linf (rows = last axis), worst over batches."""
    v = np.asarray(value).astype(np.complex128 if np.iscomplexobj(value) else np.float64)
    r = np.asarray(reference).astype(np.complex128 if np.iscomplexobj(reference) else np.float64)
    n = r.shape[-1]
    v = v.reshape(-1, n)
    r = r.reshape(-1, n)
    diff = np.abs(v - r)
    ref = np.abs(r)
    finite = bool(np.all(np.isfinite(diff)) and np.all(np.isfinite(ref)))
    err_sq = np.sum(diff * diff, axis=1)
    ref_sq = np.sum(ref * ref, axis=1)
    with np.errstate(divide="ignore", invalid="ignore"):
        rel_l2 = np.where(ref_sq == 0, np.where(err_sq == 0, 0.0, np.inf), np.sqrt(err_sq / ref_sq))
        emax, rmax = diff.max(axis=1), ref.max(axis=1)
        rel_linf = np.where(rmax == 0, np.where(emax == 0, 0.0, np.inf), emax / rmax)
    return {"rel_l2": float(rel_l2.max()), "rel_linf": float(rel_linf.max()),
            "max_abs": float(diff.max()) if diff.size else 0.0, "finite": finite}


def work_factor(n: int) -> float:
    if n <= 64:
        return float(n)
    return 3.0 * math.ceil(math.log2(2 * n - 1)) + 3.0


_CONSTANTS = {"complex": (1.2419386546059821, 1.9343969087678796),
              "real_forward": (1.234681000407627, 1.8260558195934091),
              "real_inverse": (0.97722970418819066, 1.372182697342486)}


def accuracy_limits(ftype: int, n: int) -> tuple[float, float]:
    """C(class) * u(dtype) * work(N): the reference's frozen limits vs cuFFT."""
    cls = {C2C: "complex", Z2Z: "complex", R2C: "real_forward", D2Z: "real_forward",
           C2R: "real_inverse", Z2D: "real_inverse"}[ftype]
    u = (np.finfo(np.float64).eps if ftype in (Z2Z, D2Z, Z2D) else np.finfo(np.float32).eps) / 2.0
    c2, ci = _CONSTANTS[cls]
    s = u * work_factor(n)
    return c2 * s, ci * s


def north_star_bound(ftype: int, n: int) -> float:
    """Relative-L2 bound vs the FP64 oracle: 5e-7*log2N (FP32 types), 1e-15*log2N (FP64)."""
    lg = math.log2(max(n, 2))
    return (1e-15 if ftype in (Z2Z, D2Z, Z2D) else 5e-7) * lg


def ref_plans() -> dict:
    """Reference planner trees committed under tests/golden (key 'N:c' / 'N:z')."""
    path = HERE.parent / "tests" / "golden" / "ref_plans.json"
    with open(path) as fh:
        rows = json.load(fh)
    return {f"{r['n']}:{'z' if r['dtype'] == 'complex128' else 'c'}": r["root"] for r in rows}
