"""Launch-shape autotuner for the batched window engine.

    python -m poa_b200.autotune [--workload learned_band|polishing] [--windows N]
                                [--out poa_b200/tuned_launch.json]

Needs a GPU. For one workload it times the persistent batch kernel under each
candidate launch shape (the knobs of ``poa_batch_config``: blocks per SM,
i.e. the 168- or 128-register build, and shared memory per warp, which
trades the static-band row ring and staging against L1 capacity) on a seeded
sample of the workload's windows, and records the fastest shape, with every
measurement, in a JSON file that ``bench.py`` and ``Context.batch_autotuned``
apply. Shapes that the engine rejects for the sample (too little shared
memory for its reads) are skipped. Results never depend on the shape: every
shape computes the same bands and outputs.
"""
from __future__ import annotations

import argparse
import json
import os
import sys
import time

if __package__ in (None, ""):
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
import poa_b200 as pb  # noqa: E402
from poa_b200 import synth  # noqa: E402

TUNED = os.path.join(os.path.dirname(os.path.abspath(__file__)), "tuned_launch.json")

WORKLOADS = {
    # generator, options, sample windows, seed (disjoint from the bench's), proposer
    "learned_band": ("learned_band_windows", ["-B"], 2664, 605, True),
    "polishing": ("polishing_windows", [], 20000, 604, False),
}
CANDIDATES = [(3, 18432), (3, 16384), (3, 12288), (3, 10240), (4, 12288), (4, 10240)]


def tune(workload: str, windows: int = 0, repeats: int = 1, log=print) -> dict:
    gen, opts, n_default, seed, use_prop = WORKLOADS[workload]
    ws = getattr(synth, gen)(seed=seed, n_windows=windows or n_default)
    results = []
    with pb.Context(pb.Params.from_cli(opts)) as ctx:
        prop = pb.Proposer(weights=pb.PROP_WEIGHTS) if use_prop else None
        if prop is not None:
            ctx.batch_use_proposer(prop)
        ctx.batch_upload(ws)
        for bps, smem in CANDIDATES:
            ctx.batch_config(blocks_per_sm=bps, smem_per_warp=smem)
            try:
                ctx.batch_run()  # warm-up (allocations, graph capture)
                t = min(ctx.batch_run() for _ in range(repeats))
            except pb.PoaError as e:
                log(f"  blocks/SM {bps}, smem/warp {smem}: skipped ({e})")
                continue
            st = ctx.batch_stats()
            rate = ws.n_windows / t * 1e3
            results.append({"blocks_per_sm": bps, "smem_per_warp": smem, "ms": round(t, 2),
                            "windows_per_s": round(rate, 2), "fallback_windows": st["fallback"],
                            "retried_windows": st["retried"]})
            log(f"  blocks/SM {bps}, smem/warp {smem}: {t:.1f} ms, {rate:.1f} windows/s, "
                f"fallback {st['fallback']}, retried {st['retried']}")
    if not results:
        raise RuntimeError("no launch shape ran")
    best = max(results, key=lambda r: r["windows_per_s"])
    return {"blocks_per_sm": best["blocks_per_sm"], "smem_per_warp": best["smem_per_warp"],
            "sample": f"{ws.n_windows} windows of {gen} (seed {seed})", "measured": results,
            "when": time.strftime("%Y-%m-%dT%H:%M:%SZ", time.gmtime())}


def load(workload: str, path: str = TUNED):
    """The tuned shape of a workload, or None."""
    if not os.path.exists(path):
        return None
    with open(path) as fh:
        return json.load(fh).get(workload)


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--workload", choices=sorted(WORKLOADS), action="append")
    ap.add_argument("--windows", type=int, default=0)
    ap.add_argument("--repeats", type=int, default=1)
    ap.add_argument("--out", default=TUNED)
    a = ap.parse_args(argv)
    table = {}
    if os.path.exists(a.out):
        with open(a.out) as fh:
            table = json.load(fh)
    for wl in a.workload or sorted(WORKLOADS):
        print(f"tuning {wl}", flush=True)
        table[wl] = tune(wl, a.windows, a.repeats)
        print(f"  best: blocks/SM {table[wl]['blocks_per_sm']}, smem/warp {table[wl]['smem_per_warp']}", flush=True)
        with open(a.out, "w") as fh:
            json.dump(table, fh, indent=1)


if __name__ == "__main__":
    main()
