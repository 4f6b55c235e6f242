"""Train the learned band proposer on bands the plain adaptive-band DP emits.

    python -m poa_b200.proposer_train [--reads 50000] [--seed 105] [--epochs 40]
                                      [--out poa_b200/proposer_weights.f32]

Needs a GPU. Steps:

1. Seeded synthetic windows of the learned-band workload (2,000 bp templates,
   20-100 reads, 15 % error 4:3:3, 1 % chimeric reads) from a seed disjoint
   from the benchmark's, until they hold ``--reads`` aligned reads.
2. One plain batched run with ``-B`` (the reference's adaptive band, no plan):
   per aligned read the engine reports its band statistics
   (``poa_batch_read_stats``): band cells, DP rows, graph nodes after the
   read, traceback record bytes, band centre. These are the training targets:
   new nodes per query base, cells / (rows * (qlen + 1)), record bytes per
   cell, centre / (qlen + 1).
3. The minimizer features of the same reads (``poa_batch_features``).
4. Training on 90 % of the windows with the CUDA training kernels; the other
   10 % calibrate the plan margins: the window-level ratios true / predicted
   of graph nodes and of the largest alignment's record bytes, at the
   ``--quantile`` quantile, times ``--slack``.
5. The weights (float32, little endian, ``poa_prop_nweights()`` values) and a
   JSON summary next to them.
"""
from __future__ import annotations

import argparse
import json
import os
import sys
import time

import numpy as np

if __package__ in (None, ""):
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
import poa_b200 as pb  # noqa: E402
from poa_b200 import synth  # noqa: E402

NPARAM_EXTRA = 12  # extras after the network parameters (include/poa_b200.h)


def targets(rs: np.ndarray, read_len: np.ndarray, win_off: np.ndarray):
    """Per-read raw targets and a mask of the reads that ran a DP."""
    n = rs.shape[0]
    prev = np.zeros(n, dtype=np.float64)
    for w in range(win_off.shape[0] - 1):
        a, b = int(win_off[w]), int(win_off[w + 1])
        if b - a < 1:
            continue
        prev[a] = 0
        if b - a > 1:
            prev[a + 1] = read_len[a] + 2           # the first read adds one node per base
            prev[a + 2:b] = rs[a + 1:b - 1, 3]
    rows = rs[:, 2].astype(np.float64)
    cells = rs[:, 1].astype(np.float64)
    m = read_len.astype(np.float64) + 1.0
    dp = rows > 0
    Y = np.zeros((n, 4), dtype=np.float32)
    Y[dp, 0] = (rs[dp, 3] - prev[dp]) / np.maximum(read_len[dp], 1)
    Y[dp, 1] = cells[dp] / (rows[dp] * m[dp])
    Y[dp, 2] = rs[dp, 4] / np.maximum(cells[dp], 1.0)
    Y[dp, 3] = rs[dp, 7] / 1000.0
    return Y, dp, prev


def plan_windows(pred: np.ndarray, read_len: np.ndarray, win_off: np.ndarray, node_margin=1.0, tb_margin=1.0):
    """The device plan kernel's arithmetic (proposer.cu k_plan), without the
    spill term: graph nodes after the window, largest record bytes, cost."""
    nw = win_off.shape[0] - 1
    nodes = np.zeros(nw)
    tb = np.zeros(nw)
    cost = np.zeros(nw)
    for w in range(nw):
        a, b = int(win_off[w]), int(win_off[w + 1])
        nd = 2.0 + read_len[a] if b > a else 2.0
        mt = 0.0
        c = 0.0
        for r in range(a + 1, b):
            rows = nd
            cells = min(max(float(pred[r, 1]), 0.01), 1.0) * rows * (read_len[r] + 1.0)
            bpc = min(max(float(pred[r, 2]), 1.0), 4.0)
            mt = max(mt, cells * bpc)
            c += cells
            nd += max(float(pred[r, 0]), 0.0) * read_len[r]
        nodes[w] = nd * node_margin + 64.0
        tb[w] = mt * tb_margin + 4096.0
        cost[w] = c
    return nodes, tb, cost


def window_truth(rs: np.ndarray, win_off: np.ndarray):
    nw = win_off.shape[0] - 1
    nodes = np.array([rs[win_off[w]:win_off[w + 1], 3].max() if win_off[w + 1] > win_off[w] else 2
                      for w in range(nw)], dtype=np.float64)
    tb = np.array([rs[win_off[w]:win_off[w + 1], 4].max() if win_off[w + 1] > win_off[w] else 0
                   for w in range(nw)], dtype=np.float64)
    spill = np.array([rs[win_off[w]:win_off[w + 1], 5].max() if win_off[w + 1] > win_off[w] else 0
                      for w in range(nw)], dtype=np.float64)
    return nodes, tb, spill


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--reads", type=int, default=50000, help="aligned reads in the training set")
    ap.add_argument("--seed", type=int, default=105)
    ap.add_argument("--epochs", type=int, default=40)
    ap.add_argument("--batch", type=int, default=256)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--quantile", type=float, default=0.995)
    ap.add_argument("--slack", type=float, default=1.02)
    ap.add_argument("--out", default=pb.PROP_WEIGHTS)
    a = ap.parse_args(argv)

    t0 = time.time()
    nwin = max(16, int(a.reads / 59) + 8)
    ws = synth.learned_band_windows(seed=a.seed, n_windows=nwin)
    dp_reads = int((np.diff(ws.win_off) - 1).clip(min=0).sum())
    print(f"{nwin} windows, {ws.n_reads} reads, {dp_reads} aligned reads ({time.time() - t0:.1f} s)", flush=True)

    params = pb.Params.from_cli(["-B"])
    with pb.Context(params) as ctx:
        prop = pb.Proposer()
        ctx.batch_upload(ws)
        ms = ctx.batch_run()
        _, st = ctx.batch_download()
        if any(s != 0 for s in st):
            raise SystemExit(f"plain run failed on {sum(s != 0 for s in st)} windows")
        rs = ctx.batch_read_stats()
        X = ctx.batch_features(prop)
    print(f"plain -B run: {ms / 1e3:.1f} s device time; features {X.shape}", flush=True)

    read_len = ws.read_len.astype(np.int64)
    Y, dp, _ = targets(rs, read_len, ws.win_off)
    win_of = np.searchsorted(ws.win_off, np.arange(ws.n_reads), side="right") - 1
    ntrain_w = int(round(0.9 * nwin))
    tr = dp & (win_of < ntrain_w)
    va_w = np.arange(ntrain_w, nwin)
    print(f"train reads {int(tr.sum())}, validation windows {va_w.shape[0]}", flush=True)

    t1 = time.time()
    losses = prop.train(X[tr], Y[tr], epochs=a.epochs, batch=a.batch, lr=a.lr, seed=a.seed)
    print(f"trained {a.epochs} epochs in {time.time() - t1:.1f} s; loss {losses[0]:.4f} -> {losses[-1]:.4f}",
          flush=True)

    pred = prop.predict(X)
    va_r = dp & (win_of >= ntrain_w)
    r2 = []
    for k in range(4):
        y, p = Y[va_r, k], pred[va_r, k]
        r2.append(float(1.0 - np.mean((y - p) ** 2) / max(np.var(y), 1e-12)))
    print("validation R^2 per output:", [round(x, 3) for x in r2], flush=True)

    # margins from the validation windows
    lo, hi = int(ws.win_off[ntrain_w]), int(ws.win_off[nwin])
    sub_off = ws.win_off[ntrain_w:] - lo
    pn, pt, _ = plan_windows(pred[lo:hi], read_len[lo:hi], sub_off)
    tn, tt, tsp = window_truth(rs[lo:hi], sub_off)
    rn = tn / np.maximum(pn - 64.0, 1.0)
    rt = tt / np.maximum(pt - 4096.0, 1.0)
    node_margin = float(np.quantile(rn, a.quantile) * a.slack)
    tb_margin = float(np.quantile(rt, a.quantile) * a.slack)
    rows_all = rs[dp, 2].astype(np.float64)
    spill_per_row = float(max(1.0, (rs[dp, 5] / np.maximum(rows_all, 1.0)).max() * 1.5))
    w = prop.get_weights()
    base = w.shape[0] - NPARAM_EXTRA
    w[base + 8] = node_margin
    w[base + 9] = tb_margin
    w[base + 10] = spill_per_row
    w[base + 11] = 65536.0
    prop.set_weights(w)
    prop.save(a.out)
    # what the calibrated plan does on the validation windows
    pn2, pt2, _ = plan_windows(pred[lo:hi], read_len[lo:hi], sub_off, node_margin, tb_margin)
    over = (tn > pn2) | (tt > pt2)
    summary = {
        "seed": a.seed, "windows": nwin, "aligned_reads": dp_reads, "train_reads": int(tr.sum()),
        "validation_windows": int(va_w.shape[0]), "epochs": a.epochs, "batch": a.batch, "lr": a.lr,
        "loss_first": float(losses[0]), "loss_last": float(losses[-1]),
        "validation_r2": {"new_nodes_per_base": r2[0], "band_width": r2[1], "record_bytes_per_cell": r2[2],
                          "band_centre": r2[3]},
        "node_margin": node_margin, "tb_margin": tb_margin, "spill_per_row": spill_per_row,
        "validation_fallback_windows": int(over.sum()),
        "validation_plan_over_truth": {"nodes_median": float(np.median(pn2 / tn)),
                                       "record_bytes_median": float(np.median(pt2 / np.maximum(tt, 1.0)))},
        "plain_run_device_s": ms / 1e3,
    }
    with open(os.path.splitext(a.out)[0] + ".json", "w") as fh:
        json.dump(summary, fh, indent=1)
    print(json.dumps(summary), flush=True)


if __name__ == "__main__":
    main()
