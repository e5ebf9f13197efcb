"""Regenerates ref_plans.json: the reference planner's trees for a fixed set of
lengths, produced by oracle/_ref/ref_planner (the reference's own src/plan
sources, built by `make -C oracle ref` where the reference tree exists).

    python tests/golden/make_ref_plans.py

Lengths: every n in 1..1100, the reference test-suite sizes, the sizes the
benchmark configurations use, and 250 seeded random lengths in (1100, 70000],
for complex64; a subset again for complex128.
"""
import json
import random
import subprocess
from pathlib import Path

HERE = Path(__file__).resolve().parent
BIN = HERE.parent.parent / "oracle" / "_ref" / "ref_planner"

NAMED = [16, 64, 81, 243, 256, 361, 512, 2048, 4096, 8192, 16384, 23, 67, 997, 1009, 1701, 10007, 20020,
         2 ** 24, 2 ** 23, 3 * 2 ** 20, 3 * 2 ** 19, 1536, 2047, 4099, 65536, 65521, 30030, 32768]


def lengths():
    rnd = random.Random(20261203)
    c = sorted(set(list(range(1, 1101)) + NAMED + rnd.sample(range(1101, 70001), 250)))
    z = sorted(set(NAMED + list(range(1, 300)) + rnd.sample(range(300, 20000), 60)))
    return c, z


def main():
    c, z = lengths()
    args = [f"{n}:c" for n in c] + [f"{n}:z" for n in z]
    rows = []
    for i in range(0, len(args), 400):
        out = subprocess.run([str(BIN), *args[i:i + 400]], capture_output=True, text=True, check=True).stdout
        rows += [json.loads(line) for line in out.strip().split("\n")]
    with open(HERE / "ref_plans.json", "w") as fh:
        json.dump(rows, fh, separators=(",", ":"))
        fh.write("\n")
    print(len(rows), "plans")


if __name__ == "__main__":
    main()
