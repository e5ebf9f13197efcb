"""Command line compatible with the reference's ``flagfft-cli``.

    python -m flagfft_b200.cli bench [--rank R] [--shape AxB[,CxD...]] [--api c2c|z2z|r2c|d2z|c2r|z2d]
                                     [--batch N] [--direction forward|inverse]
                                     [--placement out-of-place|in-place] [--warmup N] [--iters N]
                                     [--json] [--print-path]
    python -m flagfft_b200.cli tune [autotune options]

``bench`` follows src/cli_tools/bench/runner.cpp:224-303 and report.cpp:12-67:
the same options and defaults, the same argument checks, inputs
sin(0.173 (i + 1)) over the whole allocation (Im of DC / Nyquist zeroed for
inverse real transforms), padded real rows of 2 (n/2 + 1) scalars, plans made
with flagfftPlan1d / flagfftPlanMany (rank 2, tight batches) /
flagfftPlan3d, W warm-up pairs, then I timed iterations that alternate which
of the two libraries runs first, each call timed by its own CUDA events on
one stream.  The comparison library is cuFFT (through torch.fft, into a
preallocated output).  Output: the same table, or the same JSON report
({"status", "command", "cases": [{api, shape, rank, batch, direction,
placement, timing: {flagfft_median_ms, flagfft_p90_ms, ref_median_ms,
ref_p90_ms, speedup, warmup, iters}, plan_description?}]}).

``tune`` runs this package's autotuner (the reference's tune command is a
placeholder, src/cli_tools/tune/tune.cpp:7-9).
"""
from __future__ import annotations

import json
import sys
from dataclasses import dataclass, field

APIS = ("c2c", "z2z", "r2c", "d2z", "c2r", "z2d")
EXIT_OK, EXIT_FAILED, EXIT_USAGE = 0, 1, 2

USAGE = """usage: python -m flagfft_b200.cli <bench|tune> [options]

bench options:
  --rank R                  1, 2 or 3 (default: 1)
  --shape S[,S...]          dimensions joined by 'x', several shapes comma-separated (default: 16)
  --api A                   c2c, z2z, r2c, d2z, c2r, z2d (default: c2c)
  --batch N                 transforms per call (default: 1)
  --direction D             forward or inverse (default: forward)
  --placement P             out-of-place or in-place (default: out-of-place)
  --warmup N                Warmup iterations (default: 10)
  --iters N                 Timed iterations (default: 100)
  --json                    Output JSON report
  --print-path              Include plan description in output
"""


class CliError(Exception):
    def __init__(self, message: str, code: int = EXIT_FAILED):
        super().__init__(message)
        self.code = code


@dataclass
class Case:
    api: str = "c2c"
    shape: list = field(default_factory=lambda: [16])
    batch: int = 1
    direction: int = -1
    placement: str = "out-of-place"
    rank: int = 1

    def to_json(self) -> dict:
        return {"api": self.api, "shape": list(self.shape), "rank": self.rank, "batch": self.batch,
                "direction": "inverse" if self.direction == 1 else "forward", "placement": self.placement}


def _positive(name: str, value: str, allow_zero: bool = False) -> int:
    try:
        v = int(value)
    except ValueError:
        raise CliError(f"invalid value for {name}")
    if (allow_zero and v < 0) or (not allow_zero and v <= 0):
        raise CliError(f"{name} must be {'non-negative' if allow_zero else 'positive'}")
    return v


def _shape(value: str) -> list:
    dims = [_positive("--shape", p) for p in value.lower().split("x") if p]
    if not dims:
        raise CliError(f"invalid --shape: {value}")
    return dims


def _direction(value: str) -> int:
    if value in ("forward", "fwd", "fft"):
        return -1
    if value in ("inverse", "inv", "ifft"):
        return 1
    raise CliError(f"invalid --direction: {value}")


def parse_bench_args(argv: list) -> dict:
    """The reference's option set and checks (src/cli_tools/flagfft-cli/main.cpp:46-133)."""
    proto = Case()
    shapes, warmup, iters, as_json, print_path = [], 10, 100, False, False
    i = 0

    def need(name):
        nonlocal i
        i += 1
        if i >= len(argv):
            raise CliError(f"{name} requires a value")
        return argv[i]

    while i < len(argv):
        a = argv[i]
        if a == "--rank":
            v = need(a)
            if v not in ("1", "2", "3"):
                raise CliError(f"invalid --rank: {v} (expected 1, 2, or 3)")
            proto.rank = int(v)
        elif a == "--shape":
            shapes += [_shape(p) for p in need(a).split(",") if p]
        elif a == "--api":
            v = need(a).lower()
            if v not in APIS:
                raise CliError(f"invalid --api: {v}")
            proto.api = v
        elif a == "--batch":
            proto.batch = _positive(a, need(a))
        elif a == "--direction":
            proto.direction = _direction(need(a))
        elif a == "--placement":
            v = need(a)
            if v not in ("out-of-place", "in-place", "outofplace", "inplace"):
                raise CliError(f"invalid --placement: {v}")
            proto.placement = "in-place" if v in ("in-place", "inplace") else "out-of-place"
        elif a == "--warmup":
            warmup = _positive(a, need(a), allow_zero=True)
        elif a == "--iters":
            iters = _positive(a, need(a))
        elif a == "--json":
            as_json = True
        elif a == "--print-path":
            print_path = True
        else:
            raise CliError(f"unknown argument: {a}")
        i += 1
    cases = []
    for sh in shapes or [list(proto.shape)]:
        cases.append(Case(proto.api, sh, proto.batch, proto.direction, proto.placement, proto.rank))
    for c in cases:
        if c.rank == 2 and c.api not in ("c2c", "z2z"):
            raise CliError("rank 2 currently supports only c2c and z2z")
        if c.rank > 2 and c.batch != 1:
            raise CliError("--batch is only supported with --rank 1 or complex --rank 2")
        if len(c.shape) != c.rank:
            raise CliError("--shape dimension count does not match --rank")
        if c.api in ("r2c", "d2z") and c.direction != -1:
            raise CliError(f"{c.api} only supports forward direction")
        if c.api in ("c2r", "z2d") and c.direction != 1:
            raise CliError(f"{c.api} only supports inverse direction")
    return {"cases": cases, "warmup": warmup, "iters": iters, "json": as_json, "print_path": print_path}


def percentile(times: list, fraction: float) -> float:
    """src/cli_tools/bench/runner.cpp:18-22: the sorted sample at index
    min(n - 1, floor(fraction n))."""
    s = sorted(times)
    return s[min(len(s) - 1, int(fraction * len(s)))]


def format_json(cases: list, results: list, warmup: int, iters: int) -> dict:
    out = []
    for c, r in zip(cases, results):
        e = c.to_json()
        e["timing"] = {"flagfft_median_ms": r["flagfft_median_ms"], "flagfft_p90_ms": r["flagfft_p90_ms"],
                       "ref_median_ms": r["ref_median_ms"], "ref_p90_ms": r["ref_p90_ms"], "speedup": r["speedup"],
                       "warmup": warmup, "iters": iters}
        if r.get("plan_description"):
            e["plan_description"] = r["plan_description"]
        out.append(e)
    return {"status": "passed", "command": "bench", "cases": out}


def format_table(cases: list, results: list, warmup: int, iters: int) -> str:
    lines = [f"{'shape':<12}{'api':<8}{'batch':<7}{'direction':<11}{'placement':<14}{'warmup':<8}{'iters':<7}"
             f"{'flagfft_median_ms':<17}{'ref_median_ms':<14}speedup"]
    for c, r in zip(cases, results):
        shape = "x".join(str(d) for d in c.shape)
        lines.append(f"{shape:<12}{c.api:<8}{c.batch:<7}{'inverse' if c.direction == 1 else 'forward':<11}"
                     f"{c.placement:<14}{warmup:<8}{iters:<7}{r['flagfft_median_ms']:<17.4f}"
                     f"{r['ref_median_ms']:<14.4f}{r['speedup']:.2f}x")
    return "\n".join(lines) + "\n"


def run_case(c: Case, warmup: int, iters: int, print_path: bool) -> dict:
    """One case as runner.cpp:224-303 runs it (needs a GPU)."""
    import math

    import torch

    import flagfft_b200 as ffb
    if not torch.cuda.is_available():
        raise CliError("bench needs a CUDA device")
    dev = torch.device("cuda")
    n = c.shape[-1]
    outer = c.batch * math.prod(c.shape[:-1])
    half = n // 2 + 1
    padded = 2 * half
    double = c.api in ("z2z", "d2z", "z2d")
    scalar = torch.float64 if double else torch.float32
    cplx = torch.complex128 if double else torch.complex64
    complex_api, real_fwd, real_inv = c.api in ("c2c", "z2z"), c.api in ("r2c", "d2z"), c.api in ("c2r", "z2d")
    in_scalars = n if real_fwd else (padded if real_inv else 2 * n)
    out_scalars = padded if real_fwd else (n if real_inv else 2 * n)
    inplace = c.placement == "in-place"
    if inplace:
        in_scalars = out_scalars = 2 * n if complex_api else padded
    count = outer * max(in_scalars, out_scalars)

    def seeded():
        v = torch.sin(torch.arange(1, count + 1, dtype=torch.float64) * 0.173).to(scalar)
        if real_inv:
            rows = v[:outer * padded].view(outer, padded)
            rows[:, 1] = 0
            if n % 2 == 0:
                rows[:, n + 1] = 0
        return v.to(dev)

    ff_in, ref_in = seeded(), seeded()
    ff_out = ff_in if inplace else torch.empty(count, dtype=scalar, device=dev)
    code = getattr(ffb, c.api.upper())
    if c.rank == 1:
        plan = ffb.plan1d(n, code, c.batch)
    elif c.rank == 2:
        dist = c.shape[0] * c.shape[1]
        plan = ffb.plan_many(c.shape, None, 1, dist, None, 1, dist, code, c.batch)
    else:
        plan = ffb.plan3d(c.shape[0], c.shape[1], c.shape[2], code)
    stream = torch.cuda.Stream(device=dev)
    plan.set_stream(stream)

    # cuFFT on the same shapes (row views of the reference buffer)
    dims = tuple(range(-c.rank, 0))
    if complex_api:
        ref_x = torch.view_as_complex(ref_in[:outer * 2 * n].view(c.batch, *c.shape, 2))
        ref_y = torch.empty_like(ref_x)
        fn = torch.fft.fftn if c.direction == -1 else torch.fft.ifftn
        call_ref = lambda: fn(ref_x, dim=dims, norm="backward" if c.direction == -1 else "forward", out=ref_y)  # noqa: E731
    elif real_fwd:
        ref_x = ref_in[:outer * n].view(c.batch, *c.shape) if not inplace else \
            ref_in.view(outer, padded)[:, :n].reshape(c.batch, *c.shape)
        ref_y = torch.empty((c.batch, *c.shape[:-1], half), dtype=cplx, device=dev)
        call_ref = lambda: torch.fft.rfftn(ref_x, dim=dims, out=ref_y)  # noqa: E731
    else:
        ref_x = torch.view_as_complex(ref_in[:outer * padded].view(c.batch, *c.shape[:-1], half, 2))
        ref_y = torch.empty((c.batch, *c.shape), dtype=scalar, device=dev)
        call_ref = lambda: torch.fft.irfftn(ref_x, s=c.shape, dim=dims, norm="forward", out=ref_y)  # noqa: E731

    def call_ff():
        plan.execute(ff_in, ff_out, c.direction)

    def timed(fn):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        fn()
        e1.record(stream)
        e1.synchronize()
        return e0.elapsed_time(e1)

    with torch.cuda.stream(stream):
        for _ in range(warmup):
            call_ff()
            call_ref()
        torch.cuda.synchronize()
        ff_t, ref_t = [], []
        for i in range(iters):
            if i % 2 == 0:
                ref_t.append(timed(call_ref))
                ff_t.append(timed(call_ff))
            else:
                ff_t.append(timed(call_ff))
                ref_t.append(timed(call_ref))
    med_ff, med_ref = percentile(ff_t, 0.5), percentile(ref_t, 0.5)
    r = {"flagfft_median_ms": med_ff, "flagfft_p90_ms": percentile(ff_t, 0.9), "ref_median_ms": med_ref,
         "ref_p90_ms": percentile(ref_t, 0.9), "speedup": med_ref / med_ff if med_ff > 0 else 0.0}
    if print_path:
        r["plan_description"] = plan.description()
    plan.destroy()
    return r


def main(argv: list | None = None) -> int:
    argv = list(sys.argv[1:] if argv is None else argv)
    if not argv or argv[0] in ("-h", "--help"):
        print(USAGE)
        return EXIT_OK
    cmd, rest = argv[0], argv[1:]
    try:
        if cmd == "tune":
            from flagfft_b200 import autotune
            return autotune.main(rest)
        if cmd != "bench":
            raise CliError(f"unknown command: {cmd}", EXIT_USAGE)
        if rest and rest[0] in ("-h", "--help"):
            print(USAGE)
            return EXIT_OK
        args = parse_bench_args(rest)
        results = [run_case(c, args["warmup"], args["iters"], args["print_path"]) for c in args["cases"]]
        if args["json"]:
            print(json.dumps(format_json(args["cases"], results, args["warmup"], args["iters"]), indent=2))
        else:
            sys.stdout.write(format_table(args["cases"], results, args["warmup"], args["iters"]))
            if args["print_path"]:
                for r in results:
                    print(r.get("plan_description", ""))
        return EXIT_OK
    except CliError as e:
        print(f"error: {e}", file=sys.stderr)
        return e.code


if __name__ == "__main__":
    sys.exit(main())
