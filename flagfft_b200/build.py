"""Builds libflagfft.so in-tree (flagfft_b200/libflagfft.so) with nvcc for sm_100a.

    python -m flagfft_b200.build [--force] [--jobs N]

Objects go to flagfft_b200/_build/; a source is recompiled when it, or a
header its nvcc dependency file lists, is newer than its object (any header
of csrc/ and include/ when there is no dependency file yet).
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
BUILD = PKG / "_build"
LIB = PKG / "libflagfft.so"
INCLUDE = PKG.parent / "include"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_COMMON = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
               f"-I{INCLUDE}", f"-I{CSRC}"]


def nvcc() -> str:
    exe = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(exe).exists():
        raise RuntimeError("nvcc not found: the CUDA toolkit is required to build libflagfft.so")
    return exe


def _sources() -> list[Path]:
    return sorted(list(CSRC.glob("*.cu")) + list(CSRC.glob("*.cpp")))


def _headers_mtime() -> float:
    hs = list(CSRC.glob("*.cuh")) + list(CSRC.glob("*.hpp")) + list(CSRC.glob("*.inc")) + list(INCLUDE.glob("*.h"))
    return max((h.stat().st_mtime for h in hs), default=0.0)


def _deps(obj: Path) -> list[Path] | None:
    """Headers an object was built from (its nvcc -MD file), or None."""
    d = obj.with_suffix(".d")
    if not d.exists():
        return None
    text = d.read_text().replace("\\\n", " ")
    parts = text.split(":", 1)
    if len(parts) != 2:
        return None
    return [Path(t) for t in parts[1].split() if t]


def _stale(src: Path, obj: Path) -> bool:
    """An object is rebuilt when it is missing or older than its source or
    any header its dependency file lists (every header in csrc/ and include/
    when it has none)."""
    if not obj.exists():
        return True
    t = obj.stat().st_mtime
    deps = _deps(obj)
    if deps is None:
        return t < max(src.stat().st_mtime, _headers_mtime())
    return any((not d.exists()) or d.stat().st_mtime > t for d in [src, *deps])


def _compile(src: Path, obj: Path, verbose: bool) -> None:
    cmd = [nvcc(), *NVCC_COMMON, *ARCH, "-MD", "-MF", str(obj.with_suffix(".d")), "-c", str(src), "-o", str(obj)]
    if src.suffix == ".cu":
        cmd.insert(1, "-Xptxas=-warn-spills")
    else:
        cmd[1:1] = ["-x", "cu"]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)


def build(force: bool = False, jobs: int | None = None, verbose: bool = False) -> Path:
    BUILD.mkdir(exist_ok=True)
    todo = []
    objs = []
    for src in _sources():
        obj = BUILD / (src.stem + src.suffix.replace(".", "_") + ".o")
        objs.append(obj)
        if force or _stale(src, obj):
            todo.append((src, obj))
    jobs = jobs or min(8, os.cpu_count() or 1)
    if todo:
        with cf.ThreadPoolExecutor(max_workers=jobs) as ex:
            futs = [ex.submit(_compile, s, o, verbose) for s, o in todo]
            for f in futs:
                f.result()
    if todo or not LIB.exists() or LIB.stat().st_mtime < max(o.stat().st_mtime for o in objs):
        tmp = LIB.with_suffix(".so.tmp")
        cmd = [nvcc(), "-shared", *ARCH, "-o", str(tmp), *map(str, objs), "-ldl", "-lpthread"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
        os.replace(tmp, LIB)
    return LIB


HOSTCHECK_DIR = BUILD / "hostcheck"
HOSTCHECK_LIB = HOSTCHECK_DIR / "libflagfft_hostcheck.so"


def build_hostcheck(force: bool = False, jobs: int | None = None, verbose: bool = False) -> Path:
    """Host-emulation build of the same sources (-DFFB_HOST_EMULATION): the
    kernels run sequentially on the CPU and "device" memory is host memory.
    Test infrastructure only -- loaded by tests, never by the package."""
    HOSTCHECK_DIR.mkdir(parents=True, exist_ok=True)
    todo, objs = [], []
    for src in _sources():
        obj = HOSTCHECK_DIR / (src.stem + src.suffix.replace(".", "_") + ".o")
        objs.append(obj)
        if force or _stale(src, obj):
            todo.append((src, obj))

    def comp(src, obj):
        common = [f for f in NVCC_COMMON if f != "-O3"]
        cmd = [nvcc(), "-x", "cu", *common, "-O2", "-DFFB_HOST_EMULATION", *ARCH, "-MD", "-MF",
               str(obj.with_suffix(".d")), "-c", str(src), "-o", str(obj)]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)

    if todo:
        with cf.ThreadPoolExecutor(max_workers=jobs or min(8, os.cpu_count() or 1)) as ex:
            for f in [ex.submit(comp, s, o) for s, o in todo]:
                f.result()
    if todo or not HOSTCHECK_LIB.exists():
        cmd = [nvcc(), "-shared", *ARCH, "-o", str(HOSTCHECK_LIB), *map(str, objs), "-ldl", "-lpthread"]
        subprocess.run(cmd, check=True)
    return HOSTCHECK_LIB


def main(argv: list[str] | None = None) -> int:
    ap = argparse.ArgumentParser(description=__doc__)
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--jobs", type=int, default=None)
    ap.add_argument("-v", "--verbose", action="store_true")
    ap.add_argument("--hostcheck", action="store_true", help="also build the host-emulation test library")
    args = ap.parse_args(argv)
    path = build(args.force, args.jobs, args.verbose)
    print(path)
    if args.hostcheck:
        print(build_hostcheck(args.force, args.jobs, args.verbose))
    return 0


if __name__ == "__main__":
    sys.exit(main())
