"""poa_batch_partition: one window set split over devices by cost (CPU only).

Windows are independent, so several GPUs share one set with no exchange:
the split must give every window to exactly one part, balance the parts'
estimated cost (bases x (reads + 1)), follow the longest-processing-time
rule deterministically, and let the results be put back in input order.
"""
import types

import numpy as np
import pytest

import poa_b200
from poa_b200 import synth


def cost_of(ws):
    rl = ws.read_len.astype(np.int64)
    out = []
    for w in range(ws.n_windows):
        a, b = int(ws.win_off[w]), int(ws.win_off[w + 1])
        out.append(int(rl[a:b].sum()) * (b - a + 1))
    return np.array(out, dtype=np.int64)


@pytest.mark.parametrize("n_parts", [1, 2, 3, 8])
def test_every_window_once_and_balanced(n_parts):
    ws = synth.polishing_windows(seed=41, n_windows=600)
    part, load = poa_b200.partition(ws, n_parts)
    assert part.shape == (600,) and part.min() >= 0 and part.max() < n_parts
    c = cost_of(ws)
    for g in range(n_parts):
        assert load[g] == c[part == g].sum()
    assert load.sum() == c.sum()
    # LPT bound: no part exceeds the mean by more than the largest window
    assert load.max() <= load.mean() + c.max()


def test_lpt_rule_by_hand():
    # costs (bases x (reads + 1)): 1 read each of lengths 10, 7, 6, 5, 4 -> 20, 14, 12, 10, 8
    reads = [b"A" * n for n in (10, 7, 6, 5, 4)]
    ws = synth.pack_windows_from_reads(reads, [0, 1, 2, 3, 4, 5])
    part, load = poa_b200.partition(ws, 2)
    # 20 -> p0; 14 -> p1; 12 -> p1 (14 < 20); 10 -> p0 (20 < 26); 8 -> p0 (30 > 26? no: p0 30 vs p1 26 -> p1)
    assert part.tolist() == [0, 1, 1, 0, 1]
    assert load.tolist() == [30, 34]


def test_gather_restores_input_order():
    ws = synth.polishing_windows(seed=42, n_windows=50)
    part, _ = poa_b200.partition(ws, 3)
    shares = [np.nonzero(part == g)[0] for g in range(3)]
    out = [None] * ws.n_windows
    for idx in shares:
        sub = ws.subset(idx)
        for k, w in enumerate(idx):
            out[w] = sub.window_reads(k)
    assert all(out[w] == ws.window_reads(w) for w in range(ws.n_windows))


def test_empty_and_bad_arguments():
    ws = synth.pack_windows_from_reads([], [0])
    part, load = poa_b200.partition(ws, 4)
    assert part.shape == (0,) and load.tolist() == [0, 0, 0, 0]
    with pytest.raises(poa_b200.PoaError):
        poa_b200.partition(ws, 0)
    # offsets that start before the read list, or run backwards, are rejected
    bad = types.SimpleNamespace(read_len=np.array([5, 5], dtype=np.int32),
                                win_off=np.array([-1, 2], dtype=np.int32))
    with pytest.raises(poa_b200.PoaError):
        poa_b200.partition(bad, 2)
    bad.win_off = np.array([0, 2, 1], dtype=np.int32)
    with pytest.raises(poa_b200.PoaError):
        poa_b200.partition(bad, 2)
