"""Seeded synthetic POA workloads.

No public dataset is used: every workload is generated from a fixed seed with
the shapes, sizes and error model of the benchmark configurations:

* ``single_graph_consensus`` - 10 x 16,569 bp from one uniform random root,
  1 % substitutions and 0.5 % indels (insert:delete 1:1, geometric length,
  mean 2) per sequence; one POA graph, consensus output.
* ``single_graph_msa`` - 100 sequences from one 16,500 bp root through a
  seeded random binary phylogeny (0.2 % divergence per branch, indel:sub 1:3),
  MSA output with ``-S -r1``.
* ``noisy_long_reads`` - 30 reads sampled from one 10 kb template with 10 %
  error (sub:ins:del 4:3:3), insertions homopolymer-biased with
  probability 0.3 (the inserted base repeats its left neighbour); ``-B``.
* ``polishing_windows`` - independent windows, template 500 +- 100 bp,
  4..64 reads, 8 % error (4:3:3); one POA graph and consensus per window.
* ``learned_band_windows`` - 2,000 bp templates, 20..100 reads, 15 % error
  (4:3:3), 1 % chimeric reads (two halves from two windows).

Everything is numpy-vectorised per window so that 20,000 windows generate in
seconds. Sequences are ASCII ``bytes`` over ``ACGT``.
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import List, Sequence, Tuple

import numpy as np

ACGT = np.frombuffer(b"ACGT", dtype=np.uint8)


def random_root(rng: np.random.Generator, length: int) -> np.ndarray:
    """Uniform iid ACGT codes 0..3."""
    return rng.integers(0, 4, size=length, dtype=np.uint8)


def _geom_len(rng, shape, mean):
    if mean <= 1.0:
        return np.ones(shape, dtype=np.int64)
    return rng.geometric(1.0 / mean, size=shape).astype(np.int64)


def mutate(rng: np.random.Generator, tmpl: np.ndarray, nreads: int,
           p_sub: float, p_ins: float, p_del: float,
           indel_mean: float = 1.0, hp_bias: float = 0.0) -> List[np.ndarray]:
    """Mutate ``tmpl`` (codes 0..3) independently ``nreads`` times.

    Per template position: a substitution (to one of the 3 other bases) with
    probability ``p_sub``; an insertion after the base with ``p_ins``; a
    deletion run starting at the base with ``p_del``. Indel lengths are
    geometric with mean ``indel_mean``. With probability ``hp_bias`` an
    inserted base repeats the base to its left (homopolymer extension).
    Returns a list of code arrays.
    """
    R, L = nreads, int(tmpl.shape[0])
    if R == 0:
        return []
    u = rng.random((R, L))
    is_sub = u < p_sub
    is_ins = (u >= p_sub) & (u < p_sub + p_ins)
    is_del = (u >= p_sub + p_ins) & (u < p_sub + p_ins + p_del)

    base = np.broadcast_to(tmpl, (R, L)).copy()
    shift = rng.integers(1, 4, size=(R, L), dtype=np.uint8)
    base = np.where(is_sub, (base + shift) & 3, base).astype(np.uint8)

    # deletion runs through a difference array, clipped at the read end
    dlen = np.where(is_del, _geom_len(rng, (R, L), indel_mean), 0)
    diff = np.zeros((R, L + 1), dtype=np.int64)
    rr, cc = np.nonzero(is_del)
    if rr.size:
        ends = np.minimum(cc + dlen[rr, cc], L)
        np.add.at(diff, (rr, cc), 1)
        np.add.at(diff, (rr, ends), -1)
    deleted = np.cumsum(diff[:, :L], axis=1) > 0

    ilen = np.where(is_ins, _geom_len(rng, (R, L), indel_mean), 0)
    counts = np.where(deleted, 0, 1 + ilen)
    # an insertion after a deleted base still inserts
    counts = np.where(deleted, ilen, counts)

    flat_counts = counts.reshape(-1)
    total = int(flat_counts.sum())
    out = np.repeat(base.reshape(-1), flat_counts)
    starts = np.cumsum(flat_counts) - flat_counts
    slot = np.arange(total, dtype=np.int64) - np.repeat(starts, flat_counts)
    keep_first = np.repeat(~deleted.reshape(-1), flat_counts)
    # slots after the first copy (or every slot of a deleted base) are inserted
    ins_slot = (slot >= 1) | ~keep_first
    n_ins = int(ins_slot.sum())
    if n_ins:
        rnd = rng.integers(0, 4, size=n_ins, dtype=np.uint8)
        if hp_bias > 0.0:
            left = np.repeat(base.reshape(-1), flat_counts)[ins_slot]
            hp = rng.random(n_ins) < hp_bias
            rnd = np.where(hp, left, rnd).astype(np.uint8)
        out[ins_slot] = rnd
    per_read = counts.sum(axis=1)
    return np.split(out, np.cumsum(per_read)[:-1])


def to_ascii(codes: np.ndarray) -> bytes:
    return ACGT[codes].tobytes()


def single_graph_consensus(seed: int = 1, nseq: int = 10, length: int = 16569) -> List[bytes]:
    rng = np.random.default_rng(seed)
    root = random_root(rng, length)
    reads = mutate(rng, root, nseq, p_sub=0.01, p_ins=0.0025, p_del=0.0025, indel_mean=2.0)
    return [to_ascii(r) for r in reads]


def single_graph_msa(seed: int = 2, nseq: int = 100, length: int = 16500,
                     branch_div: float = 0.002) -> List[bytes]:
    """Yule-process binary phylogeny: split a random leaf until ``nseq``
    leaves; each child gets ``branch_div`` mutations per site (indel:sub 1:3,
    insert:delete 1:1, geometric indel length mean 2)."""
    rng = np.random.default_rng(seed)
    root = random_root(rng, length)
    p_sub = branch_div * 0.75
    p_ind = branch_div * 0.25
    leaves = [root]
    while len(leaves) < nseq:
        k = int(rng.integers(0, len(leaves)))
        parent = leaves.pop(k)
        kids = mutate(rng, parent, 2, p_sub, p_ind / 2, p_ind / 2, indel_mean=2.0)
        leaves.extend(kids)
    order = rng.permutation(len(leaves))
    return [to_ascii(leaves[i]) for i in order]


def noisy_long_reads(seed: int = 3, nreads: int = 30, length: int = 10000,
                     err: float = 0.10) -> List[bytes]:
    rng = np.random.default_rng(seed)
    tmpl = random_root(rng, length)
    reads = mutate(rng, tmpl, nreads, err * 0.4, err * 0.3, err * 0.3, hp_bias=0.3)
    return [to_ascii(r) for r in reads]


@dataclass
class WindowSet:
    """A batch of independent POA windows.

    ``seq`` holds every read's ASCII bases back to back. Read ``r`` is
    ``seq[read_off[r]:read_off[r] + read_len[r]]``; window ``w`` owns reads
    ``win_off[w] .. win_off[w + 1] - 1`` in their input order.
    """
    seq: np.ndarray        # uint8, concatenated ASCII
    read_off: np.ndarray   # int64 [nreads]
    read_len: np.ndarray   # int32 [nreads]
    win_off: np.ndarray    # int32 [nwin + 1]

    @property
    def n_windows(self) -> int:
        return int(self.win_off.shape[0] - 1)

    @property
    def n_reads(self) -> int:
        return int(self.read_len.shape[0])

    def window_reads(self, w: int) -> List[bytes]:
        a, b = int(self.win_off[w]), int(self.win_off[w + 1])
        return [self.seq[self.read_off[r]:self.read_off[r] + self.read_len[r]].tobytes()
                for r in range(a, b)]

    def subset(self, windows: Sequence[int]) -> "WindowSet":
        reads: List[bytes] = []
        offs = [0]
        for w in windows:
            rs = self.window_reads(int(w))
            reads.extend(rs)
            offs.append(offs[-1] + len(rs))
        return pack_windows_from_reads(reads, offs)


def pack_windows_from_reads(reads: Sequence[bytes], win_off: Sequence[int]) -> WindowSet:
    lens = np.array([len(r) for r in reads], dtype=np.int32)
    offs = np.zeros(len(reads), dtype=np.int64)
    if len(reads):
        offs[1:] = np.cumsum(lens[:-1], dtype=np.int64)
    seq = np.frombuffer(b"".join(reads), dtype=np.uint8).copy()
    return WindowSet(seq=seq, read_off=offs, read_len=lens,
                     win_off=np.asarray(win_off, dtype=np.int32))


def windows(seed: int, n_windows: int, tlen: Tuple[int, int], nreads: Tuple[int, int],
            err: float, chimeric: float = 0.0) -> WindowSet:
    """Independent windows: template length uniform in ``tlen`` (inclusive),
    read count uniform in ``nreads`` (inclusive), error ``err`` split 4:3:3
    into substitutions, insertions and deletions. A fraction ``chimeric`` of
    reads is replaced by the first half of a read of this window joined to
    the second half of a read of a random other window."""
    rng = np.random.default_rng(seed)
    pieces: List[np.ndarray] = []
    counts = np.zeros(n_windows + 1, dtype=np.int64)
    tmpls = []
    for w in range(n_windows):
        L = int(rng.integers(tlen[0], tlen[1] + 1))
        R = int(rng.integers(nreads[0], nreads[1] + 1))
        t = random_root(rng, L)
        tmpls.append(t)
        rs = mutate(rng, t, R, err * 0.4, err * 0.3, err * 0.3)
        pieces.extend(rs)
        counts[w + 1] = R
    win_off = np.cumsum(counts).astype(np.int32)
    if chimeric > 0.0 and n_windows > 1:
        nr = len(pieces)
        pick = np.nonzero(rng.random(nr) < chimeric)[0]
        owner = np.searchsorted(win_off, np.arange(nr), side="right") - 1
        for r in pick:
            other = int(rng.integers(0, n_windows - 1))
            if other >= owner[r]:
                other += 1
            donor = mutate(rng, tmpls[other], 1, err * 0.4, err * 0.3, err * 0.3)[0]
            a = pieces[r]
            pieces[r] = np.concatenate([a[: a.shape[0] // 2], donor[donor.shape[0] // 2:]])
    lens = np.array([p.shape[0] for p in pieces], dtype=np.int32)
    offs = np.zeros(len(pieces), dtype=np.int64)
    if len(pieces):
        offs[1:] = np.cumsum(lens[:-1], dtype=np.int64)
    seq = ACGT[np.concatenate(pieces)] if pieces else np.zeros(0, np.uint8)
    return WindowSet(seq=np.ascontiguousarray(seq), read_off=offs, read_len=lens, win_off=win_off)


def polishing_windows(seed: int = 4, n_windows: int = 20000) -> WindowSet:
    return windows(seed, n_windows, (400, 600), (4, 64), 0.08)


def learned_band_windows(seed: int = 5, n_windows: int = 5000) -> WindowSet:
    return windows(seed, n_windows, (2000, 2000), (20, 100), 0.15, chimeric=0.01)


def write_fasta(path: str, seqs: Sequence[bytes], names: Sequence[str] = None) -> None:
    with open(path, "wb") as fh:
        for i, s in enumerate(seqs):
            nm = names[i] if names is not None else f"seq{i + 1}"
            fh.write(b">" + nm.encode() + b"\n" + s + b"\n")


def write_pwin(path: str, ws: WindowSet, windows: Sequence[int] = None) -> None:
    """Write windows to the flat binary window file the host-thread harnesses
    read: b"PWIN", u32 n_windows, u32 n_reads, u32 win_off[n_windows + 1],
    u32 read_len[n_reads], then the reads' ASCII bases back to back."""
    if windows is not None:
        ws = ws.subset(windows)
    lens = ws.read_len.astype(np.uint32)
    with open(path, "wb") as fh:
        fh.write(b"PWIN")
        fh.write(np.array([ws.n_windows, ws.n_reads], dtype=np.uint32).tobytes())
        fh.write(ws.win_off.astype(np.uint32).tobytes())
        fh.write(lens.tobytes())
        if ws.n_reads:
            a = int(ws.read_off[0])
            b = int(ws.read_off[-1]) + int(ws.read_len[-1])
            fh.write(ws.seq[a:b].tobytes())


def read_cons_file(path: str) -> List[bytes]:
    """Consensus strings of a window harness output (u32 length + bases each)."""
    out: List[bytes] = []
    with open(path, "rb") as fh:
        data = fh.read()
    p = 0
    while p + 4 <= len(data):
        n = int(np.frombuffer(data, dtype=np.uint32, count=1, offset=p)[0])
        out.append(data[p + 4:p + 4 + n])
        p += 4 + n
    return out
