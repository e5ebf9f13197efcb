"""Seeded synthetic workloads of the benchmark configurations.

* ``uneven_lengths`` -- the batched uneven-length set: transform lengths drawn
  log-uniform in [16, 65536], 40% snapped to a power of two, 30% to the
  nearest 7-smooth number, 30% to the next prime.
* ``serving_trace`` -- the serving mix: Poisson arrivals, C2C / R2C / Z2Z
  requests (60 / 30 / 10 %) with lengths drawn from that set and batch 1..64.

Both are deterministic for a seed (numpy's PCG64), so the benchmark and the
tests draw the same transforms.  No dataset is involved.
"""
from __future__ import annotations

import math


def uneven_lengths(count: int = 10000, seed: int = 0x55AB, lo: int = 16, hi: int = 65536) -> list[int]:
    """Lengths log-uniform in [lo, hi]: 40% snapped to a power of two, 30% to
    the nearest 7-smooth number, 30% to the next prime (seeded)."""
    import numpy as np
    rng = np.random.default_rng(seed)
    smooth = sorted({2 ** a * 3 ** b * 5 ** c * 7 ** d for a in range(17) for b in range(11) for c in range(8)
                     for d in range(7) if lo <= 2 ** a * 3 ** b * 5 ** c * 7 ** d <= hi})
    sieve = np.ones(2 * hi + 1, dtype=bool)
    sieve[:2] = False
    for i in range(2, int((2 * hi) ** 0.5) + 1):
        if sieve[i]:
            sieve[i * i::i] = False
    primes = np.nonzero(sieve)[0]
    out = []
    for u, kind in zip(rng.uniform(math.log(lo), math.log(hi), count), rng.uniform(0, 1, count)):
        x = math.exp(u)
        if kind < 0.4:
            n = 2 ** int(round(math.log2(x)))
        elif kind < 0.7:
            i = int(np.searchsorted(smooth, x))
            cands = [smooth[j] for j in (i - 1, i) if 0 <= j < len(smooth)]
            n = min(cands, key=lambda v: abs(v - x))
        else:
            n = int(primes[np.searchsorted(primes, x)])
            if n > hi:
                n = int(primes[np.searchsorted(primes, hi) - 1])
        out.append(int(min(max(n, lo), hi)))
    return out


def length_groups(lengths: list[int]) -> tuple[list[int], list[int]]:
    """Distinct lengths (ascending) and how many transforms each has."""
    groups: dict[int, int] = {}
    for n in lengths:
        groups[n] = groups.get(n, 0) + 1
    glen = sorted(groups)
    return glen, [groups[n] for n in glen]


def serving_trace(rate: float, seconds: float, seed: int = 0x5E4E) -> list[tuple[float, str, int, int]]:
    """(arrival time s, type, n, batch) of a Poisson stream: C2C / R2C / Z2Z
    60 / 30 / 10 %, lengths drawn from the uneven_lengths() set, batch
    uniform 1..64.  Real requests keep even lengths."""
    import numpy as np
    rng = np.random.default_rng(seed)
    count = int(rate * seconds * 1.05) + 16
    gaps = rng.exponential(1.0 / rate, count)
    times = np.cumsum(gaps)
    times = times[times < seconds]
    pool = uneven_lengths()
    lengths = [pool[i] for i in rng.integers(0, len(pool), len(times))]
    kinds = rng.uniform(0, 1, len(times))
    batches = rng.integers(1, 65, len(times))
    out = []
    for t, n, k, b in zip(times, lengths, kinds, batches):
        ty = "C2C" if k < 0.6 else "R2C" if k < 0.9 else "Z2Z"
        if ty == "R2C" and n % 2:
            n += 1
        out.append((float(t), ty, int(n), int(b)))
    return out
