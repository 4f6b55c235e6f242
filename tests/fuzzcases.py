"""Seeded random small POA inputs for differential tests (test infrastructure).

Each case is a template of 30-700 bases and 1-14 reads copied from it with
substitutions, insertions and deletions at 0-25 % (some runs of N, some lower
case), run under one option set that the CPU restatement in oracle/ covers.
"""
from __future__ import annotations

import numpy as np

OPTION_SETS = [
    [],
    ["-B"],
    ["-r", "1"],
    ["-r", "2"],
    ["-B", "-r", "1"],
    ["-f", "0"],
    ["-M", "3", "-X", "5", "-O", "6", "-E", "1", "-b", "20", "-f", "10"],
    ["-M", "1", "-X", "2", "-O", "3", "-E", "1", "-B"],
]


def _mutate(rng, t: bytes, rate: float) -> bytes:
    out = bytearray()
    for c in t:
        u = rng.random()
        if u < rate * 0.5:  # substitution
            out.append(b"ACGT"[(b"ACGT".index(c) + 1 + int(rng.integers(3))) % 4] if c in b"ACGT" else c)
        elif u < rate * 0.75:  # deletion
            continue
        elif u < rate:  # insertion of 1-4 bases, then the base
            out += bytes(rng.choice(list(b"ACGT"), size=int(rng.integers(1, 5))).astype(np.uint8))
            out.append(c)
        else:
            out.append(c)
    return bytes(out)


def case(seed: int):
    """(reads, options) of fuzz case `seed`."""
    rng = np.random.default_rng(1000 + seed)
    L = int(rng.integers(30, 700))
    t = bytes(rng.choice(list(b"ACGT"), size=L).astype(np.uint8))
    n = int(rng.integers(1, 15))
    rate = float(rng.choice([0.0, 0.02, 0.08, 0.15, 0.25]))
    reads = []
    for _ in range(n):
        r = _mutate(rng, t, rate)
        if rng.random() < 0.3 and len(r) > 10:  # a prefix or suffix only
            a, b = sorted(rng.integers(0, len(r), size=2))
            r = r[a:max(b, a + 5)]
        if rng.random() < 0.1 and len(r) > 20:
            k = int(rng.integers(0, len(r) - 5))
            r = r[:k] + b"NNNN" + r[k + 4:]
        if rng.random() < 0.1:
            r = r.lower()
        reads.append(r)
    opts = OPTION_SETS[int(rng.integers(len(OPTION_SETS)))]
    return reads, list(opts)
