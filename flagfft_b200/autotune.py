"""Autotuner command: times the candidate trees of each requested length on
this GPU and writes the fastest into the tune database plan creation reads.

    python -m flagfft_b200.autotune --lengths 1009,4096 --batch 256 [--type C2C|Z2Z]
                                    [--direction -1|1|both] [--db PATH]

Without --db the rows go to $FLAGFFT_TUNE_DB, else
<executable dir>/.flagfft/tuned_plans.sqlite (the same rule as the lookup).
"""
from __future__ import annotations

import argparse
import json
import sys

import flagfft_b200 as ffb


def main(argv: list[str] | None = None) -> int:
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--lengths", required=True, help="comma-separated transform lengths")
    ap.add_argument("--batch", type=int, default=1)
    ap.add_argument("--type", choices=["C2C", "Z2Z"], default="C2C")
    ap.add_argument("--direction", choices=["-1", "1", "both"], default="both")
    ap.add_argument("--db", default=None)
    args = ap.parse_args(argv)
    dirs = [-1, 1] if args.direction == "both" else [int(args.direction)]
    for n in (int(v) for v in args.lengths.split(",") if v):
        for d in dirs:
            rep = ffb.tune(n, getattr(ffb, args.type), args.batch, d, args.db)
            print(json.dumps({"n": n, "direction": d, "best_ms": rep["best_ms"], "default_ms": rep["default_ms"],
                              "stored": rep["stored"], "best_kind": rep["best"].get("kind")}))
    return 0


if __name__ == "__main__":
    sys.exit(main())
