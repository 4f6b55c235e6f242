"""NumPy model of the band proposer's feature kernel (test infrastructure).

The minimizer set follows the reference's mm_sketch (src/minimizer.cpp:60-135,
forward strand, no homopolymer compression): a k-mer is a minimizer when its
hash is the minimum of some window of w consecutive valid k-mers. The
features are the ones poa_b200/csrc/proposer.cu writes per read and bin.
"""
from __future__ import annotations

import numpy as np

BINS, CIN = 32, 8
U64 = np.uint64
MAXH = np.uint64(0xFFFFFFFFFFFFFFFF)
_NT4 = np.full(256, 4, dtype=np.uint8)
for _i, _c in enumerate(b"ACGT"):
    _NT4[_c] = _i
    _NT4[_c | 0x20] = _i


def hash64(key: np.ndarray, mask: int) -> np.ndarray:
    """Thomas Wang's 64-bit hash on uint64 arrays (src/minimizer.cpp:11-21)."""
    m = U64(mask)
    with np.errstate(over="ignore"):
        key = (~key + (key << U64(21))) & m
        key = key ^ (key >> U64(24))
        key = ((key + (key << U64(3))) + (key << U64(8))) & m
        key = key ^ (key >> U64(14))
        key = ((key + (key << U64(2))) + (key << U64(4))) & m
        key = key ^ (key >> U64(28))
        key = (key + (key << U64(31))) & m
    return key


def kmer_hashes(seq: bytes, k: int) -> np.ndarray:
    """Hash of the k-mer ending at every position (MAXH where none is valid)."""
    c = _NT4[np.frombuffer(seq, dtype=np.uint8)] if len(seq) else np.zeros(0, np.uint8)
    n = c.shape[0]
    h = np.full(n, MAXH, dtype=U64)
    if n < k:
        return h
    mask = (1 << (2 * k)) - 1
    ends = np.arange(k - 1, n)
    code = np.zeros(ends.shape[0], dtype=U64)
    bad = np.zeros(ends.shape[0], dtype=bool)
    for j in range(k):
        cj = c[ends - (k - 1) + j]
        bad |= cj >= 4
        code = (code << U64(2)) | (cj & 3).astype(U64)
    hv = hash64(code & U64(mask), mask)
    hv[bad] = MAXH
    h[k - 1:] = hv
    return h


def minimizer_positions(seq: bytes, k: int, w: int) -> np.ndarray:
    """End positions of the minimizers (sorted)."""
    h = kmer_hashes(seq, k)
    n = h.shape[0]
    if n < w:
        return np.zeros(0, dtype=np.int64)
    win = np.lib.stride_tricks.sliding_window_view(h, w)
    full = (win != MAXH).all(axis=1)
    wmin = win.min(axis=1)
    flag = np.zeros(n, dtype=bool)
    for o in range(w):
        flag[o:o + win.shape[0]] |= full & (h[o:o + win.shape[0]] == wmin)
    return np.nonzero(flag)[0]


def mm_key(h: np.ndarray) -> np.ndarray:
    k = ((h ^ (h >> U64(32))) & U64(0xFFFFFFFF)).astype(np.uint32)
    k[k == 0] = 1
    return k


def window_features(reads, k: int = 15, w: int = 10) -> np.ndarray:
    """Features [len(reads), 32, 8] of one window's reads."""
    R = len(reads)
    pos, keys = [], []
    for s in reads:
        p = minimizer_positions(s, k, w)
        pos.append(p)
        keys.append(mm_key(kmer_hashes(s, k)[p]) if p.shape[0] else np.zeros(0, np.uint32))
    allk = np.concatenate(keys) if keys else np.zeros(0, np.uint32)
    uniq, cnt = np.unique(allk, return_counts=True)
    X = np.zeros((R, BINS, CIN), dtype=np.float32)
    f32 = np.float32
    L0 = len(reads[0]) if R else 0
    r1 = max(R - 1, 1)
    for r, s in enumerate(reads):
        L = len(s)
        acc = np.zeros((BINS, 3), dtype=np.float32)
        if pos[r].shape[0]:
            c = cnt[np.searchsorted(uniq, keys[r])]
            others = np.maximum(c.astype(np.int64) - 1, 0)
            b = (pos[r] * BINS) // max(L, 1)
            np.add.at(acc[:, 0], b, 1.0)
            np.add.at(acc[:, 1], b, (others > 0).astype(np.float32))
            np.add.at(acc[:, 2], b, np.minimum(others, r1).astype(np.float32))
        blen = max(f32(L) / f32(BINS), f32(1.0))
        for b in range(BINS):
            nm = acc[b, 0]
            X[r, b, 0] = nm * f32(w + 1) / (f32(2.0) * blen)
            X[r, b, 1] = acc[b, 1] / nm if nm > 0 else 0.0
            X[r, b, 2] = f32(10.0) * acc[b, 2] / (nm * f32(r1)) if nm > 0 else 0.0
            X[r, b, 3] = f32(L) / f32(2048.0)
            X[r, b, 4] = f32(L0) / f32(2048.0)
            X[r, b, 5] = f32(r) / f32(100.0)
            X[r, b, 6] = f32(R) / f32(100.0)
            X[r, b, 7] = (f32(b) + f32(0.5)) / f32(BINS)
    return X
