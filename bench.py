#!/usr/bin/env python
"""Benchmark of the flagfft.h Exec hot path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--workload NAME]

Default workload ("arbitrary_1d"): the arbitrary-length 1-D configuration --
C2C (complex64) N = 1701, 1009, 10007 at batch 1024 and Z2Z (complex128) at the
same lengths at batch 256, forward, out of place.  One step executes all six
plans once.  Inputs are seeded iid uniform[-1, 1) re/im (synthetic; no
dataset).  Each step touches ~312 MB (inputs + outputs), more than the 126 MB
L2, so consecutive uses of a buffer come from HBM.

Metric: GFLOP/s at 5 N log2 N per complex transform, whole job (all ranks).
The JSON line also carries, per N, the device time, GFLOP/s and GB/s against
the algorithmic bytes (passes x batch x (N_in e_in + N_out e_out), passes = 1
when one transform fits on chip), the roofline of the dominant kernel, the
end-to-end figure through the public API with host buffers, cuFFT (torch.fft)
on the same problems as a comparator, and the CPU baseline.

Multi-GPU (torchrun): every rank runs the same per-GPU workload on its own
GPU (independent transforms: no collective on the data path, weak scaling);
timing is the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent

WORKLOADS = {
    # (type, N, batch)
    "arbitrary_1d": [("C2C", 1701, 1024), ("C2C", 1009, 1024), ("C2C", 10007, 1024),
                     ("Z2Z", 1701, 256), ("Z2Z", 1009, 256), ("Z2Z", 10007, 256)],
    "plain_c2c_4096": [("C2C", 4096, 256)],
    "real_large": [("R2C", 1 << 24, 4), ("D2Z", 3 << 20, 2)],
}
WORKLOAD_DESC = {
    "arbitrary_1d": "C2C N=1701,1009,10007 x1024 + Z2Z same N x256, forward, out-of-place",
    "plain_c2c_4096": "C2C N=4096 x256, forward, out-of-place",
    "real_large": "R2C N=2^24 x4 + D2Z N=3*2^20 x2, out-of-place",
}


def parse_args():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=sorted(WORKLOADS), default="arbitrary_1d")
    ap.add_argument("--cpu-seconds", type=float, default=12.0, help="budget of the CPU baseline sample")
    ap.add_argument("--no-cufft", action="store_true")
    ap.add_argument("--problem", default=None, metavar="TYPE:N:BATCH",
                    help="run one problem instead of a named workload (profiling captures), e.g. C2C:10007:1024")
    args = ap.parse_args()
    if args.problem:
        t, n, b = args.problem.split(":")
        if t not in ("C2C", "Z2Z", "R2C", "D2Z", "C2R", "Z2D"):
            ap.error(f"unknown transform type {t}")
        WORKLOADS["problem"] = [(t, int(n), int(b))]
        WORKLOAD_DESC["problem"] = f"{t} N={n} x{b}, forward, out-of-place"
        args.workload = "problem"
    return args


# ---------------------------------------------------------------------------
# helpers
# ---------------------------------------------------------------------------

def elem_bytes(t: str) -> tuple[int, int]:
    """(input element bytes, output element bytes)."""
    return {"C2C": (8, 8), "Z2Z": (16, 16), "R2C": (4, 8), "D2Z": (8, 16), "C2R": (8, 4), "Z2D": (16, 8)}[t]


def flops(t: str, n: int, batch: int) -> float:
    """5 N log2 N per transform (real transforms quoted at the same 5 N log2 N)."""
    return 5.0 * n * math.log2(n) * batch


def measured_peaks() -> dict:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return {"hbm_gbs": float(d["hbm_gbs"]), "source": "measured (MEASURED_PEAKS.json)"}
    return {"hbm_gbs": 6650.0, "source": "fallback 6.65 TB/s"}


class ClockSampler:
    """nvidia-smi SM clock / throttle-reason samples while the timed region runs."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.dev = device_index
        self.proc = None
        self.lines: list[str] = []
        self.thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.dev}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except (OSError, FileNotFoundError):
            self.proc = None
            return

        def reader():
            for line in self.proc.stdout:
                self.lines.append(line.strip())

        self.thread = threading.Thread(target=reader, daemon=True)
        self.thread.start()

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.15)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        if self.thread:
            self.thread.join(timeout=2)
        sm, smax, reasons, power = [], [], set(), []
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
                power.append(float(parts[3]))
            except ValueError:
                continue
            for name, flag in zip(names, parts[5:9]):
                if flag.lower() == "active":
                    reasons.add(name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(smax), "reasons": sorted(reasons),
                "samples": len(sm), "power_w_max": max(power) if power else None}


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------

def run_ours(args, rank: int, world: int, local_rank: int):
    import numpy as np
    import torch

    import flagfft_b200 as ffb

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    problems = WORKLOADS[args.workload]
    stream = torch.cuda.Stream(device=dev)

    cdt = {"C2C": torch.complex64, "Z2Z": torch.complex128, "R2C": torch.float32, "D2Z": torch.float64,
           "C2R": torch.complex64, "Z2D": torch.complex128}
    odt = {"C2C": torch.complex64, "Z2Z": torch.complex128, "R2C": torch.complex64, "D2Z": torch.complex128,
           "C2R": torch.float32, "Z2D": torch.float64}
    tcode = {"C2C": ffb.C2C, "Z2Z": ffb.Z2Z, "R2C": ffb.R2C, "D2Z": ffb.D2Z, "C2R": ffb.C2R, "Z2D": ffb.Z2D}

    gen = torch.Generator(device=dev)
    gen.manual_seed(0x46544646 + rank)
    items = []
    for (t, n, b) in problems:
        in_n = n // 2 + 1 if t in ("C2R", "Z2D") else n
        out_n = n // 2 + 1 if t in ("R2C", "D2Z") else n
        dt = cdt[t]
        if dt.is_complex:
            real = torch.float32 if dt == torch.complex64 else torch.float64
            x = torch.view_as_complex((torch.rand((b, in_n, 2), generator=gen, device=dev, dtype=real) * 2 - 1)
                                      .contiguous())
        else:
            x = torch.rand((b, in_n), generator=gen, device=dev, dtype=dt) * 2 - 1
        y = torch.empty((b, out_n), dtype=odt[t], device=dev)
        plan = ffb.plan1d(n, tcode[t], b)
        plan.set_stream(stream)
        ib, ob = elem_bytes(t)
        onchip = plan.launch_count(-1 if t not in ("C2R", "Z2D") else 1) == 1
        items.append({"t": t, "n": n, "b": b, "x": x, "y": y, "plan": plan, "in_n": in_n, "out_n": out_n,
                      "alg_bytes": (1 if onchip else 2) * b * (in_n * ib + out_n * ob),
                      "launches": plan.launch_count(1 if t in ("C2R", "Z2D") else -1)})

    def step():
        for it in items:
            it["plan"].execute(it["x"], it["y"], -1)

    # correctness spot check against cuFFT (torch.fft) on the first problem, untimed
    check = None
    it0 = items[0]
    if it0["t"] in ("C2C", "Z2Z"):
        with torch.cuda.stream(stream):
            it0["plan"].execute(it0["x"], it0["y"], -1)
        stream.synchronize()
        ref = torch.fft.fft(it0["x"].to(torch.complex128), dim=-1)
        err = (torch.linalg.vector_norm(it0["y"].to(torch.complex128) - ref, dim=-1) /
               torch.linalg.vector_norm(ref, dim=-1)).max().item()
        check = {"problem": f"{it0['t']} N={it0['n']}", "max_rel_l2_vs_cufft_fp64": err}

    def barrier():
        if world > 1:
            import torch.distributed as dist
            dist.barrier()

    with torch.cuda.stream(stream):
        for _ in range(args.warmup):
            step()
    torch.cuda.synchronize()

    # ---- whole-step timing
    sampler = ClockSampler(torch.cuda.current_device())
    sampler.start()
    barrier()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    with torch.cuda.stream(stream):
        for _ in range(args.steps):
            step()
    e1.record(stream)
    torch.cuda.synchronize()
    barrier()
    clocks = sampler.stop()
    total_ms = e0.elapsed_time(e1)

    # ---- per-problem timing (same stream, events around each exec)
    per = []
    reps = max(3, args.steps)
    for it in items:
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
        torch.cuda.synchronize()
        ev[0].record(stream)
        with torch.cuda.stream(stream):
            for _ in range(reps):
                it["plan"].execute(it["x"], it["y"], -1)
        ev[1].record(stream)
        torch.cuda.synchronize()
        ms = ev[0].elapsed_time(ev[1]) / reps
        it["ms"] = ms
        per.append(it)

    # ---- cuFFT comparator (torch.fft, same problems, same stream)
    cufft = None
    if not args.no_cufft:
        cufft = {}
        for it in items:
            fn = {"C2C": torch.fft.fft, "Z2Z": torch.fft.fft, "R2C": torch.fft.rfft, "D2Z": torch.fft.rfft}.get(it["t"])
            if fn is None:
                continue
            with torch.cuda.stream(stream):
                for _ in range(3):
                    fn(it["x"], dim=-1)
                ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
                torch.cuda.synchronize()
                ev[0].record(stream)
                for _ in range(reps):
                    fn(it["x"], dim=-1)
                ev[1].record(stream)
            torch.cuda.synchronize()
            ms = ev[0].elapsed_time(ev[1]) / reps
            cufft[f"{it['t']}_{it['n']}"] = {"ms": ms, "gflops": flops(it["t"], it["n"], it["b"]) / ms / 1e6}

    # ---- end-to-end through the public API with host buffers
    e2e = run_e2e(args, items, stream, torch)

    # ---- max over ranks
    if world > 1:
        import torch.distributed as dist
        tt = torch.tensor([total_ms, e2e["ms_per_step"]], device=dev, dtype=torch.float64)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        total_ms, e2e_ms = tt.tolist()
        e2e["ms_per_step"] = e2e_ms
    for it in items:
        it["plan"].destroy()
    return {"total_ms": total_ms, "per": per, "clocks": clocks, "check": check, "cufft": cufft, "e2e": e2e}


def run_e2e(args, items, stream, torch):
    """Same step through the public API with host buffers: per step the inputs
    are copied from pinned host memory and the results read back."""
    hosts = []
    for it in items:
        hin = torch.empty(it["x"].shape, dtype=it["x"].dtype, pin_memory=True)
        hin.copy_(it["x"].cpu())
        hout = torch.empty(it["y"].shape, dtype=it["y"].dtype, pin_memory=True)
        hosts.append((hin, hout))
    h2d = sum(h[0].numel() * h[0].element_size() for h in hosts)
    d2h = sum(h[1].numel() * h[1].element_size() for h in hosts)

    def step():
        with torch.cuda.stream(stream):
            for it, (hin, hout) in zip(items, hosts):
                it["x"].copy_(hin, non_blocking=True)
                it["plan"].execute(it["x"], it["y"], -1)
                hout.copy_(it["y"], non_blocking=True)

    for _ in range(max(1, args.warmup // 2)):
        step()
    torch.cuda.synchronize()
    steps = max(3, args.steps // 4)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        step()
    e1.record(stream)
    torch.cuda.synchronize()
    return {"ms_per_step": e0.elapsed_time(e1) / steps, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
            "steps": steps}


# ---------------------------------------------------------------------------
# CPU baseline / reference arm: the oracle port of the reference algorithm
# ---------------------------------------------------------------------------

def _cpu_sample_problem(job):
    """One bounded CPU job: (type, n, rows).  Returns (seconds, flop)."""
    t, n, rows = job
    import numpy as np
    sys.path.insert(0, str(ROOT))
    from oracle import oracle as O
    O.build()
    plans = O.ref_plans()
    double = t == "Z2Z"
    plan = plans.get(f"{n}:{'z' if double else 'c'}") or O.default_plan(n)
    x = O.random_complex(n * rows, n + rows, double).reshape(rows, n).astype(np.complex128)
    t0 = time.perf_counter()
    O.c2c(x, -1, plan, precision="f64" if double else "f32")
    return time.perf_counter() - t0, flops(t, n, rows)


def cpu_baseline(problems, budget_s: float, threads: int) -> dict:
    """Times the oracle (a CPU port of the reference's Exec algorithms, float
    arithmetic for C2C and double for Z2Z) on a bounded sample of the workload:
    a few rows of each problem, run as one process per core."""
    import multiprocessing as mp

    jobs = []
    for (t, n, b) in problems:
        if t not in ("C2C", "Z2Z"):
            continue
        rows = 2 if n > 5000 else 4
        jobs += [(t, n, rows)] * threads
    ctx = mp.get_context("spawn")
    t0 = time.perf_counter()
    done_flop, busy = 0.0, 0.0
    with ctx.Pool(threads) as pool:
        for sec, fl in pool.imap_unordered(_cpu_sample_problem, jobs):
            done_flop += fl
            busy += sec
            if time.perf_counter() - t0 > budget_s:
                break
    wall = time.perf_counter() - t0
    return {"value": done_flop / wall / 1e9, "unit": "GFLOP/s", "cores": threads, "kind": "port",
            "sample": f"{len(jobs)} jobs of 2-4 rows of each problem of the workload, oracle port (reference "
                      f"algorithm restated in C; float for C2C, double for Z2Z), {threads} processes, "
                      f"{wall:.1f}s wall"}


def run_reference(args, rank: int, world: int):
    if rank != 0:
        return 0
    problems = WORKLOADS[args.workload]
    threads = os.cpu_count() or 1
    vals = []
    for _ in range(args.warmup):
        pass
    for _ in range(max(1, min(args.steps, 3))):
        vals.append(cpu_baseline(problems, min(args.cpu_seconds, 20.0), threads))
    v = statistics.median(x["value"] for x in vals)
    total_flop = sum(flops(t, n, b) for (t, n, b) in problems)
    ms = total_flop / (v * 1e9) * 1e3 if v > 0 else None
    line = {
        "impl": "reference", "metric": "gflops_5nlog2n", "value": v, "unit": "GFLOP/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "c64+c128", "data": "synthetic",
        "config": {"workload": args.workload, "problems": WORKLOAD_DESC[args.workload]},
        "cpu_baseline": {**vals[-1], "value": v},
        "e2e": {"value": v, "unit": "GFLOP/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": "reference arm = the oracle's CPU port of the reference's Exec algorithms on the host cores "
                "(the reference's own Triton-JIT Exec cannot be built: its libtriton_jit submodule and "
                "Triton TLE extension are absent)",
    }
    print(json.dumps(line))
    return 0


# ---------------------------------------------------------------------------

def main():
    args = parse_args()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return run_reference(args, rank, world)

    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local_rank))
    res = run_ours(args, rank, world, local_rank)
    problems = WORKLOADS[args.workload]
    step_flop = sum(flops(t, n, b) for (t, n, b) in problems)
    ms_step = res["total_ms"] / args.steps
    value = step_flop * world / (ms_step * 1e-3) / 1e9
    peaks = measured_peaks()

    per_n = []
    dominant = None
    for it in res["per"]:
        gbs = it["alg_bytes"] / (it["ms"] * 1e-3) / 1e9
        row = {"type": it["t"], "N": it["n"], "batch": it["b"], "ms": it["ms"],
               "gflops": flops(it["t"], it["n"], it["b"]) / it["ms"] / 1e6, "alg_GBs": gbs,
               "hbm_frac": gbs / peaks["hbm_gbs"], "launches": it["launches"], "alg_bytes": it["alg_bytes"]}
        per_n.append(row)
        if dominant is None or row["ms"] > dominant["ms"]:
            dominant = row
    launches_per_step = sum(it["launches"] for it in res["per"])

    if rank == 0:
        e2e_ms = res["e2e"]["ms_per_step"]
        line = {
            "metric": "gflops_5nlog2n", "value": value, "unit": "GFLOP/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "c64+c128" if args.workload == "arbitrary_1d" else "mixed",
            "data": "synthetic (seeded uniform[-1,1) re/im)",
            "config": {"workload": args.workload, "problems": WORKLOAD_DESC[args.workload],
                       "l2": "per-step footprint above the 126 MB L2 (inputs+outputs)",
                       "parallelism": f"replicas over batch, {world} GPU"},
            "per_n": per_n,
            "roofline": {"bound": "hbm", "kernel": f"{dominant['type']} N={dominant['N']}",
                         "achieved": dominant["alg_GBs"], "peak": peaks["hbm_gbs"], "unit": "GB/s",
                         "frac": dominant["hbm_frac"], "traffic": None, "peak_source": peaks["source"],
                         "alg_bytes_per_launch": dominant["alg_bytes"] / max(1, dominant["launches"])},
            "e2e": {"value": step_flop * world / (e2e_ms * 1e-3) / 1e9, "unit": "GFLOP/s",
                    "h2d_bytes_per_step": res["e2e"]["h2d_bytes_per_step"],
                    "d2h_bytes_per_step": res["e2e"]["d2h_bytes_per_step"], "ms_per_step": e2e_ms},
            "gpu_launches": launches_per_step * args.steps,
            "clocks": res["clocks"],
            "check": res["check"],
            "cufft": res["cufft"],
        }
        if world == 1:
            line["cpu_baseline"] = cpu_baseline(problems, args.cpu_seconds, os.cpu_count() or 1)
        print(json.dumps(line))
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
