"""Band proposer, CPU side: the minimizer restatement against the reference's
own mm_sketch, and the plan arithmetic of the training script."""
from __future__ import annotations

import os
import subprocess

import numpy as np
import pytest

from tests import proposer_model as pm

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HARNESS = os.path.join(ROOT, "oracle", "_ref", "sketch_harness")


def _rand(rng, n):
    return np.frombuffer(b"ACGT", dtype=np.uint8)[rng.integers(0, 4, n)].tobytes()


def _reads():
    rng = np.random.default_rng(21)
    out = []
    for L in (24, 25, 40, 100, 513, 2000, 2400):
        out.append(_rand(rng, L))
    # repeats: identical k-mers inside one window (ties)
    unit = _rand(rng, 7)
    out.append(unit * 60)
    out.append(b"A" * 80 + _rand(rng, 200))
    out.append(_rand(rng, 300).lower())
    return out


def _reference_sketch(reads, k, w):
    res = subprocess.run([HARNESS, str(k), str(w)], input=b"\n".join(reads) + b"\n", capture_output=True,
                         check=True)
    per = [set() for _ in reads]
    for line in res.stdout.decode().splitlines():
        r, p, h = line.split()
        per[int(r)].add((int(p), int(h)))
    return per


@pytest.mark.skipif(not os.path.exists(HARNESS), reason="oracle/_ref not built (make -C oracle ref)")
@pytest.mark.parametrize("k,w", [(15, 10), (19, 10), (11, 5)])
def test_minimizers_match_reference_sketch(k, w):
    reads = _reads()
    ref = _reference_sketch(reads, k, w)
    for i, s in enumerate(reads):
        if len(s) < w + k - 1:
            continue  # the reference keeps the minimum of a partial window; the features skip such reads
        p = pm.minimizer_positions(s, k, w)
        h = pm.kmer_hashes(s, k)[p]
        mine = {(int(a), int(b)) for a, b in zip(p, h)}
        if mine != ref[i]:
            # Equal k-mers in one window: the reference's streaming loop drops
            # the minimum it held when an equal k-mer completes the first full
            # window of a run (the old minimum is replaced before it may be
            # written). The set definition keeps it; nothing else may differ.
            assert ref[i] <= mine, f"read {i}: reference minimizers missing {sorted(ref[i] - mine)[:5]}"
            hashes = [hh for _, hh in ref[i]]
            for pos, hh in mine - ref[i]:
                assert hashes.count(hh) >= 1, f"read {i}: extra minimizer {pos} is not a tie"


def test_feature_model_shapes_and_ranges():
    rng = np.random.default_rng(3)
    t = _rand(rng, 800)
    reads = [t, t, t[:400] + _rand(rng, 400)]
    X = pm.window_features(reads)
    assert X.shape == (3, 32, 8)
    # identical reads: every minimizer anchors to another read
    assert np.all(X[0, :, 1][X[0, :, 0] > 0] == 1.0)
    # the random second half of read 2 anchors nowhere
    assert X[2, 20:, 1].max() == 0.0
    assert np.allclose(X[:, :, 7], (np.arange(32) + 0.5) / 32)


def test_plan_arithmetic():
    from poa_b200.proposer_train import plan_windows
    read_len = np.array([100, 100, 100, 50], dtype=np.int64)
    win_off = np.array([0, 3, 4], dtype=np.int32)
    pred = np.array([[0, 0, 0, 0], [0.1, 0.5, 2.0, 0.5], [0.2, 0.5, 1.0, 0.5], [0, 0, 0, 0]], dtype=np.float32)
    nodes, tb, cost = plan_windows(pred, read_len, win_off)
    # window 0: 102 nodes, read 1: 102 rows -> cells 0.5*102*101, +10 nodes; read 2: 112 rows
    c1 = 0.5 * 102 * 101
    c2 = 0.5 * 112 * 101
    assert cost[0] == pytest.approx(c1 + c2)
    assert tb[0] == pytest.approx(max(2 * c1, c2) + 4096)
    assert nodes[0] == pytest.approx(102 + 10 + 20 + 64)
    assert nodes[1] == pytest.approx(52 + 64) and cost[1] == 0
