"""Benchmark: batched POA windows on B200, with the learned band proposer.

Default workload (one step): 5,000 independent learned-band windows (template
2,000 bp, 20-100 reads, 15 % error split 4:3:3 into substitutions, insertions
and deletions, 1 % chimeric reads; seeded synthetic data), each aligned
progressively into its own POA graph with minipoa's adaptive band (-B,
scoring 2/-4/-4/-2, b=100 f=40); output one consensus per window, bit-exact
with minipoa. The learned band proposer plans every window's device slot
inside the timed step (features, network, plan, then the persistent batch
kernel; windows that outgrow their slot are re-run and counted as fallback).
``--workload polishing``: 20,000 polishing windows (500 +- 100 bp, 4-64
reads, 8 % error, static band), no proposer.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload learned_band|polishing]

value  windows/s over all ranks with the inputs resident in HBM (device time
       of the whole step: proposer plan + batch kernel + re-runs, CUDA events
       on the engine's stream).
e2e    windows/s through the public C ABI (poa_batch_consensus) with the
       inputs in pinned host memory: upload, plan, kernel, consensus download.
plain_kernel  windows/s of the plain single-alignment kernel path (poa_run:
       one CTA per poa() call, graph fused on the host) on a sample of the
       same windows, and the batched engine's speed-up over it.
Multi-GPU: one set of N x 5,000 windows, split over the ranks by cost
(poa_batch_partition; weak scaling: the work per GPU stays fixed); no
collective on the data path: torch.distributed gives the barrier, the max
over ranks of the time, and the gather of the consensus strings (in window
order) after the timed region for the parity check.
``--impl reference`` times the reference's own CPU build (oracle/_ref/minipoa,
compiled from the reference sources) on a bounded sample of the same
windows with every host core, one process per window.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time
from concurrent.futures import ThreadPoolExecutor

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "windows/s & GCUPS on 1 B200: learned-band+batched vs plain kernel, bit-exact"
REF_BIN = os.path.join(ROOT, "oracle", "_ref", "minipoa")
PORT_BIN = os.path.join(ROOT, "oracle", "build", "poa_oracle")
POOL_BIN = os.path.join(ROOT, "oracle", "_ref", "ref_pool")
# algorithmic work per DP cell: 1 byte of traceback record written
# (cell = one computed band cell, (Be-Bs-1)*8 per row)
BYTES_PER_CELL = 1.0
# int32 operations per cell and per edge-cell of the recurrence
OPS_PER_CELL, OPS_PER_EDGE_CELL = 5, 7

WORKLOADS = {
    "learned_band": {
        "gen": "learned_band_windows", "seed": 5, "windows": 5000, "opts": ["-B"], "proposer": True,
        "manifest": "windows_learned_band",
        "steps": 1, "ref_windows_per_core": 2, "ref_sample_per_core": 8,
        "desc": "learned_band_windows: 5000 windows, template 2000 bp, 20-100 reads, 15% error (4:3:3), "
                "1% chimeric reads; adaptive band -B; consensus",
        "mode": "consensus, adaptive band (-B) b=100 f=40, learned band proposer sizes the slots"},
    "polishing": {
        "gen": "polishing_windows", "seed": 4, "windows": 20000, "opts": [], "proposer": False,
        "manifest": "windows_polishing",
        "steps": 5, "ref_windows_per_core": 40, "ref_sample_per_core": 400,
        "desc": "polishing_windows: 20000 windows, template 500+-100 bp, 4-64 reads, 8% error (4:3:3), consensus",
        "mode": "consensus, static band b=100 f=40"},
}


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def rank_windows(ws, world: int, rank: int):
    """This rank's share of one window set: the cost-balanced split of
    poa_batch_partition (longest processing time first), in input order."""
    if world == 1:
        return np.arange(ws.n_windows)
    import poa_b200
    part, _ = poa_b200.partition(ws, world)
    return np.nonzero(part == rank)[0]


def gather_in_order(D, idx, items, n_total):
    """Per-window results of every rank, back in the window set's order."""
    pairs = D.gather_objects(list(zip([int(i) for i in idx], items)))
    out = [None] * n_total
    for part in pairs:
        for i, v in part:
            out[i] = v
    return out


def whole_job_rate(total_units: int, steps: int, t_max: float) -> float:
    """Units per second of the whole job (all ranks' units), timed by the slowest rank."""
    return total_units * steps / t_max


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rk = int(os.environ.get("RANK", "0"))
    lr = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rk, lr


class Dist:
    def __init__(self, world):
        self.world = world
        self.pg = None
        if world > 1:
            import datetime

            import torch
            import torch.distributed as dist
            backend = "nccl" if torch.cuda.is_available() else "gloo"
            if torch.cuda.is_available():
                # this rank's GPU before the group exists, so every collective runs on it
                torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=600))
            self.pg = dist

    def barrier(self):
        if self.pg:
            import torch
            if torch.cuda.is_available():
                t = torch.ones(1, device="cuda")
                self.pg.all_reduce(t)
                torch.cuda.synchronize()
            else:
                self.pg.barrier()

    def max(self, x: float) -> float:
        if not self.pg:
            return x
        import torch
        dev = "cuda" if torch.cuda.is_available() else "cpu"
        t = torch.tensor([x], dtype=torch.float64, device=dev)
        self.pg.all_reduce(t, op=self.pg.ReduceOp.MAX)
        return float(t.item())

    def sum(self, x: float) -> float:
        if not self.pg:
            return x
        import torch
        dev = "cuda" if torch.cuda.is_available() else "cpu"
        t = torch.tensor([x], dtype=torch.float64, device=dev)
        self.pg.all_reduce(t)
        return float(t.item())

    def gather_objects(self, obj):
        """Every rank's `obj`, in rank order (all ranks take part)."""
        if not self.pg:
            return [obj]
        out = [None] * self.world
        self.pg.all_gather_object(out, obj)
        return out

    def close(self):
        if self.pg:
            self.pg.destroy_process_group()


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_id: str):
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", gpu_id, "--query-gpu=" + self.Q,
                                       "--format=csv,noheader,nounits", "-lms", "200"],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None

    def stop(self) -> dict:
        if not self.p:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.p.kill()
        self.f.flush()
        self.f.seek(0)
        rows = [r.split(",") for r in self.f.read().strip().splitlines() if r.count(",") >= 8]
        os.unlink(self.f.name)
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        sm, mx, reasons = [], [], set()
        for r in rows:
            try:
                sm.append(float(r[1]))
                mx.append(float(r[2]))
            except ValueError:
                continue
            for k, nm in enumerate(names):
                if "Active" in r[5 + k] and "Not" not in r[5 + k]:
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def gpu_uuid(dev: int) -> str:
    try:
        import torch
        u = torch.cuda.get_device_properties(dev).uuid
        return "GPU-" + str(u)
    except Exception:
        return str(dev)


def load_peaks() -> dict:
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as fh:
            d = json.load(fh)
        return {"hbm_gbs": d.get("hbm_gbs"), "src": "measured", "sm_max_mhz": d.get("sm_max_mhz", 1965.0)}
    return {"hbm_gbs": 6650.0, "src": "fallback", "sm_max_mhz": 1965.0}


def profile_traffic_per_cell(workload: str):
    """DRAM bytes per DP cell of k_batch from the committed ncu summary of the workload."""
    name = {"polishing": "k_batch_dram.json", "learned_band": "k_batch_dram_learned_band.json"}[workload]
    p = os.path.join(ROOT, "profiles", name)
    if not os.path.exists(p):
        return None
    with open(p) as fh:
        d = json.load(fh)
    return d.get("dram_bytes_per_cell")


def int_peak_ops(sm_mhz):
    """Nominal int32 ALU rate (148 SMs x 128 lanes x SM clock), for context only."""
    return 148 * 128 * (sm_mhz or 1965.0) * 1e6


def measure_int_peak(device: int) -> dict:
    """The measured int32 add+max rate of this GPU (poa_int_peak: independent
    v = max(v + inc, floor) chains, 2 ops per step), with the clocks seen
    while it ran. It is the primary roofline's denominator."""
    import poa_b200
    clk = ClockSampler(gpu_uuid(device))
    best, ms = 0.0, 0.0
    for _ in range(3):
        v, t = poa_b200.int_peak(device)
        if v > best:
            best, ms = v, t
    return {"ops_per_s": best, "launch_ms": ms, "clocks": clk.stop(),
            "kernel": "poa_int_peak (16 independent add+max chains per thread, 4 x 256 threads per SM)"}


# --------------------------------------------------------------------- CPU leg
def write_windows(ws, idx, d):
    from poa_b200 import synth
    paths = []
    for w in idx:
        fa = os.path.join(d, f"w{w}.fa")
        synth.write_fasta(fa, ws.window_reads(int(w)))
        paths.append(fa)
    return paths


def run_cpu_windows(binary, paths, cores, opts=()):
    def one(fa):
        return subprocess.run([binary, fa] + list(opts), capture_output=True, check=True).stdout
    with ThreadPoolExecutor(max_workers=cores) as ex:
        return list(ex.map(one, paths))


def run_pool(pwin, opts, cores, first, n, seconds=None):
    """One oracle/_ref/ref_pool run: the reference library (one minipoa run
    per window) on `cores` host threads pulling windows first .. first+n-1
    continuously. Returns (windows done, wall s, summed per-window thread s,
    consensus of the leading done windows)."""
    from poa_b200 import synth
    out = pwin + ".cons"
    cmd = [POOL_BIN] + (["-B"] if "-B" in opts else []) + ["-t", str(cores), "-f", str(first), "-n", str(n)]
    if seconds:
        cmd += ["-s", str(seconds)]
    res = subprocess.run(cmd + [pwin, out], capture_output=True, text=True, check=True)
    f = res.stdout.split()
    kv = dict(zip(f[0::2], f[1::2]))
    cons = synth.read_cons_file(out)
    os.unlink(out)
    return int(kv["windows"]), float(kv["seconds"]), float(kv["busy"]), cons


def cpu_sample(ws, seconds, cores, opts, per_core):
    """The reference on this host's cores over the first windows of ws, for
    about `seconds`: (sustained windows/s = done / (thread time / threads),
    windows done, wall s, their consensus). Without the compiled reference
    the restatement runs instead, one process per window."""
    from poa_b200 import synth
    n = min(ws.n_windows, per_core * cores)
    if os.path.exists(POOL_BIN):
        with tempfile.TemporaryDirectory() as d:
            pw = os.path.join(d, "w.pwin")
            synth.write_pwin(pw, ws, range(n))
            done, wall, busy, cons = run_pool(pw, opts, cores, 0, n, seconds)
        return "reference", done * cores / busy, done, wall, cons
    outs = []
    k = 0
    with tempfile.TemporaryDirectory() as d:
        paths = write_windows(ws, range(n), d)
        t0 = time.perf_counter()
        while k < n and time.perf_counter() - t0 < seconds:
            idx = range(k, min(n, k + cores))
            outs.extend(o.split(b"\n")[1] for o in run_cpu_windows(PORT_BIN, [paths[w] for w in idx], cores, opts))
            k = idx.stop
        dt = time.perf_counter() - t0
    return "port", k / dt, k, dt, outs


def make_windows(wl, n, reads_per_window=0):
    from poa_b200 import synth
    ws = getattr(synth, wl["gen"])(seed=wl["seed"], n_windows=n)
    if reads_per_window > 0:
        # small profiling captures: the first reads of every window
        reads, offs = [], [0]
        for w in range(ws.n_windows):
            rs = ws.window_reads(w)[:reads_per_window]
            reads.extend(rs)
            offs.append(offs[-1] + len(rs))
        ws = synth.pack_windows_from_reads(reads, offs)
    return ws


def manifest_check(wl, cons):
    """Windows whose consensus matches the reference's per-window manifest
    (tests/golden/<manifest>.txt, md5[:16] of each window's consensus, made
    by tests/golden/make_golden.py --windows from the reference binary)."""
    import hashlib
    p = os.path.join(ROOT, "tests", "golden", wl["manifest"] + ".txt")
    if not os.path.exists(p):
        return None
    with open(p) as fh:
        head = json.loads(fh.readline()[2:])
        want = [ln.strip() for ln in fh]
    if head["kwargs"]["seed"] != wl["seed"] or len(cons) != head["windows"]:
        return None  # another set (the chimeric reads depend on the set's size)
    n = min(len(want), len(cons))
    same = sum(1 for w in range(n) if hashlib.md5(cons[w]).hexdigest()[:16] == want[w])
    return {"windows": n, "identical_consensus": same, "manifest": os.path.relpath(p, ROOT)}


# --------------------------------------------------------------------- arms
def ours(args, world, rank, local, D):
    import poa_b200
    from poa_b200 import synth
    wl = WORKLOADS[args.workload]
    nwin = args.windows or wl["windows"]
    t0 = time.perf_counter()
    # one window set of nwin windows per GPU, split over the ranks by cost
    full = make_windows(wl, nwin * world, args.reads_per_window)
    mine = rank_windows(full, world, rank)
    ws = full if world == 1 else full.subset(mine)
    log(f"[rank {rank}] generated {full.n_windows} windows, this rank runs {ws.n_windows} / {ws.n_reads} reads "
        f"in {time.perf_counter() - t0:.1f}s")
    try:
        import torch
        torch.cuda.set_device(local)
    except Exception:
        pass
    ipeak = measure_int_peak(local)
    params = poa_b200.Params.from_cli(wl["opts"])
    ctx = poa_b200.Context(params, device=local)
    prop = None
    if wl["proposer"] and not args.no_proposer:
        prop = poa_b200.Proposer(device=local, weights=poa_b200.PROP_WEIGHTS)
        ctx.batch_use_proposer(prop)
    shape = {"source": "engine defaults"}
    if not (args.blocks_per_sm or args.smem_per_warp or args.no_autotuned):
        t = ctx.batch_autotuned(args.workload)
        if t:
            shape = {"source": "poa_b200/tuned_launch.json (python -m poa_b200.autotune)",
                     "blocks_per_sm": t["blocks_per_sm"], "smem_per_warp": t["smem_per_warp"]}
    if args.max_blocks:
        ctx.batch_config(max_blocks=args.max_blocks)
    if args.blocks_per_sm:
        ctx.batch_config(blocks_per_sm=args.blocks_per_sm)
        shape = {"source": "command line", "blocks_per_sm": args.blocks_per_sm}
    if args.smem_per_warp:
        ctx.batch_config(smem_per_warp=args.smem_per_warp)
        shape = dict(shape, source="command line", smem_per_warp=args.smem_per_warp)

    # ---- device-resident leg: plan + kernel(s) per step, device-timed
    ctx.batch_upload(ws)
    for k in range(args.warmup):
        ms = ctx.batch_run()
        log(f"[rank {rank}] warm-up {k}: {ms / 1e3:.2f}s")
    D.barrier()
    clk = ClockSampler(gpu_uuid(local))
    dev_ms, kern_ms, plan_ms = [], [], []
    launches = fallback = 0
    for _ in range(args.steps):
        dev_ms.append(ctx.batch_run())
        st = ctx.batch_stats()
        kern_ms.append(st["kernel_us"] / 1e3)
        plan_ms.append(st["plan_us"] / 1e3)
        launches += st["launches"]
        fallback += st["fallback"]
    D.barrier()
    clocks = clk.stop()
    st = ctx.batch_stats()
    t_dev = D.max(sum(dev_ms) / 1e3)
    cells = st["cells"]
    failed = int(D.sum(st["failed"]))
    cons, status = ctx.batch_download()
    plan_check = None
    if prop is not None:
        # how often a window's real need exceeded its OWN predicted need (nodes, record
        # bytes of its largest alignment, spilled entries), apart from the launch's slot
        # sizing (every slot sized for the largest predicted window, x PLAN_HEADROOM)
        p_nodes, p_tb, p_sp = ctx.batch_plan_get()
        rs = ctx.batch_read_stats()
        woff = ws.win_off
        miss = 0
        for w in range(ws.n_windows):
            a, b = int(woff[w]), int(woff[w + 1])
            if b <= a:
                continue
            r = rs[a:b]
            if r[-1, 3] > p_nodes[w] or r[:, 4].max() > p_tb[w] or r[:, 5].max() > p_sp[w]:
                miss += 1
        plan_check = {"windows_over_own_prediction": miss, "rate": miss / max(ws.n_windows, 1),
                      "slot_headroom": 1.5,
                      "note": "slots are sized for the largest predicted window x 1.5 (memory allowing); "
                              "this counts windows whose need exceeded their own prediction"}
    # every window of the whole set against the reference's per-window manifest
    all_cons = cons if world == 1 else gather_in_order(D, mine, cons, full.n_windows)
    parity_full = manifest_check(wl, all_cons) if (rank == 0 and not args.reads_per_window) else None
    # proposer kernels per step: features, 3 im2col + 5 GEMM + pool + de-standardise
    # per 4096-read chunk, conversion, plan
    if prop is not None:
        chunks = -(-ws.n_reads // 4096)
        launches += args.steps * (2 + chunks * 11)

    # ---- end-to-end leg through the C ABI with pinned host buffers
    e2e = None
    if not args.no_e2e:
        holders = []
        arrs = []
        for a in (ws.seq, ws.read_off, ws.read_len, ws.win_off):
            h, v = poa_b200.pinned_copy(np.ascontiguousarray(a))
            holders.append(h)
            arrs.append(v)
        pws = synth.WindowSet(seq=arrs[0], read_off=arrs[1], read_len=arrs[2], win_off=arrs[3])
        e2e_warm = args.e2e_warmup if args.e2e_warmup >= 0 else (1 if wl["steps"] > 1 else 0)
        for _ in range(e2e_warm):
            ctx.batch_consensus(pws)
        D.barrier()
        t0 = time.perf_counter()
        for _ in range(args.steps):
            c2, s2 = ctx.batch_consensus(pws)
        D.barrier()
        t_e2e = D.max(time.perf_counter() - t0)
        st2 = ctx.batch_stats()
        e2e = {"value": whole_job_rate(full.n_windows, args.steps, t_e2e), "unit": "windows/s",
               "h2d_bytes_per_step": int(st2["h2d_bytes"]), "d2h_bytes_per_step": int(st2["d2h_bytes"]),
               "ms_per_step": 1e3 * t_e2e / args.steps, "api": "poa_batch_consensus", "warmup": e2e_warm,
               "note": "host wall clock around upload + plan + kernel + download"
                       + ("; the same context ran the device leg's warm-up steps first" if not e2e_warm else "")}
        assert c2 == cons and s2 == status, "end-to-end run disagrees with the device-resident run"
        for h in holders:
            h.close()

    value = whole_job_rate(full.n_windows, args.steps, t_dev)
    cells_all = D.sum(cells)
    kernel_s = D.max(sum(kern_ms) / 1e3) / args.steps
    peaks = load_peaks()
    achieved = cells * BYTES_PER_CELL / kernel_s / 1e9
    int_ops = cells * OPS_PER_CELL + st["edge_cells"] * OPS_PER_EDGE_CELL + (cells if wl["opts"] == ["-B"] else 0)
    tpc = profile_traffic_per_cell(args.workload)
    int_achieved = int_ops / kernel_s
    roofline = {"bound": "int_alu", "achieved": int_achieved / 1e12, "peak": ipeak["ops_per_s"] / 1e12,
                "unit": "Tops/s (int32)", "frac": int_achieved / ipeak["ops_per_s"],
                "peak_src": "measured in this run: " + ipeak["kernel"],
                "peak_clocks": ipeak["clocks"], "kernel": "k_batch", "kernel_s_per_step": kernel_s,
                "int_ops_per_launch": int_ops,
                "int_ops_note": "5 int32 ops per cell + 7 per edge-cell (cell x in-window predecessor)"
                                + (" + 1 per cell for the adaptive argmax" if wl["opts"] == ["-B"] else ""),
                "nominal_frac": int_achieved / int_peak_ops(clocks.get("sm_mhz")),
                "traffic": (tpc * cells if tpc is not None else None),
                "hbm": {"achieved": achieved, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                        "frac": achieved / peaks["hbm_gbs"], "peak_src": peaks["src"],
                        "algorithmic_bytes_per_launch": cells * BYTES_PER_CELL,
                        "traffic": (tpc * cells if tpc is not None else None),
                        "traffic_per_cell": tpc}}
    line = {
        "metric": METRIC, "value": value, "unit": "windows/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * t_dev / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "int32", "data": "synthetic (seeded; no dataset)",
        "config": {"workload": wl["desc"] + (f" (first {args.reads_per_window} reads per window)"
                                              if args.reads_per_window else ""),
                   "windows_per_rank": ws.n_windows, "reads_per_rank": ws.n_reads,
                   "bases_per_rank": int(ws.seq.shape[0]), "mode": wl["mode"] if prop else
                   wl["mode"].replace(", learned band proposer sizes the slots", ""),
                   "parallelism": f"one set of {full.n_windows} windows split over {world} GPU(s) by cost "
                                  "(poa_batch_partition)",
                   "l2": "inputs (%.0f MB) and slots (%.1f GB) larger than L2 (126 MB)"
                         % (ws.seq.shape[0] / 1e6, st["slots"] * st["slot_bytes"] / 1e9)},
        "gcups": cells_all * args.steps / t_dev / 1e9,
        "cells_per_step": cells, "failed_windows": failed,
        "gpu_launches": launches, "retried_windows": st["retried"], "e2e": e2e, "roofline": roofline, "clocks": clocks,
        "parity_full": parity_full,
        "slots": st["slots"], "slot_bytes": st["slot_bytes"], "launch_shape": shape,
        "phase_share": {k: v / max(1, sum(st["phase_cycles"].values())) for k, v in st["phase_cycles"].items()},
        "phase_mcycles_per_window": {k: v / 1e6 / ws.n_windows for k, v in st["phase_cycles"].items()},
    }
    if prop is not None:
        line["proposer"] = {"fallback_windows": int(D.sum(fallback)),
                            "fallback_rate": D.sum(fallback) / (world * ws.n_windows * args.steps),
                            "plan_ms_per_step": sum(plan_ms) / args.steps,
                            "weights": os.path.relpath(poa_b200.PROP_WEIGHTS, ROOT),
                            "exact": "the plan sizes slots only; every DP runs the reference band",
                            "per_window": plan_check}
    if rank == 0 and world == 1 and args.plain_windows > 0:
        # the plain single-alignment kernel on the first windows of the same set
        n = min(args.plain_windows, ws.n_windows)
        t0 = time.perf_counter()
        same = 0
        for w in range(n):
            txt, _ = ctx.run(ws.window_reads(w))
            same += txt == b">consensus sequence\n" + cons[w] + b"\n"
        dt = time.perf_counter() - t0
        line["plain_kernel"] = {"value": n / dt, "unit": "windows/s", "windows": n, "identical_consensus": same,
                                "path": "poa_run: one CTA per poa() call (k_plain_static for the static band, k_plain for -B), graph fused on the host",
                                "speedup": value / (n / dt)}
    if rank == 0 and world == 1 and not args.no_cpu:
        cores = len(os.sched_getaffinity(0))
        kind, v, n, dt, outs = cpu_sample(ws, args.cpu_seconds, cores, wl["opts"], wl["ref_sample_per_core"])
        same = sum(1 for w in range(n) if outs[w] == cons[w])
        line["cpu_baseline"] = {"value": v, "unit": "windows/s", "cores": cores, "kind": kind,
                                "sample": f"first {n} of the {ws.n_windows} windows "
                                          f"({' '.join(wl['opts']) or 'default options'}), "
                                          + ("oracle/_ref/ref_pool: the reference library, one minipoa run per "
                                             f"window, {cores} threads pulling windows; windows / (thread time / "
                                             f"threads); {dt:.1f}s wall, {n / dt:.3f} windows/s by wall clock"
                                             if kind == "reference" else
                                             f"the restatement, one process per window, {dt:.1f}s wall")}
        line["parity_sample"] = {"windows": n, "identical_consensus": same}
    ctx.close()
    return line


def reference(args, world, rank, local, D):
    """The reference's own CPU build on this host's cores (rank 0 only): each
    step runs the next windows of the same seeded set through
    oracle/_ref/ref_pool (the reference library, one minipoa run per window,
    every host thread pulling windows). The rate counts every thread busy:
    windows / (summed per-window thread time / threads); the wall-clock rate
    is reported beside it."""
    if rank != 0:
        return None
    from poa_b200 import synth
    wl = WORKLOADS[args.workload]
    cores = len(os.sched_getaffinity(0))
    per_step = min(args.windows or wl["windows"], wl["ref_windows_per_core"] * cores)
    # every step (warm-up ones too) takes the next windows of the seeded set, so the
    # timed steps see windows of every size rather than the same few again
    total = min(args.windows or wl["windows"], per_step * (args.warmup + args.steps))
    ws = make_windows(wl, total)
    first = lambda k: (k * per_step) % total
    done = 0
    busy_s = wall_s = 0.0
    with tempfile.TemporaryDirectory() as d:
        pw = os.path.join(d, "w.pwin")
        synth.write_pwin(pw, ws)
        if os.path.exists(POOL_BIN):
            kind = "reference"
            for k in range(args.warmup):
                run_pool(pw, wl["opts"], cores, first(k), per_step)
            for k in range(args.warmup, args.warmup + args.steps):
                n, wall, busy, _ = run_pool(pw, wl["opts"], cores, first(k), per_step)
                done += n
                busy_s += busy / cores
                wall_s += wall
        else:
            kind = "port"
            paths = write_windows(ws, range(total), d)
            t0 = time.perf_counter()
            for k in range(args.warmup, args.warmup + args.steps):
                idx = range(first(k), min(first(k) + per_step, total))
                run_cpu_windows(PORT_BIN, [paths[w] for w in idx], cores, wl["opts"])
                done += len(idx)
            busy_s = wall_s = time.perf_counter() - t0
    v = done / busy_s
    return {"impl": "reference", "metric": METRIC, "value": v, "unit": "windows/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * busy_s / args.steps,
            "wall_ms_per_step": 1e3 * wall_s / args.steps, "wall_value": done / wall_s,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int32",
            "data": "synthetic (seeded; no dataset)",
            "config": {"workload": wl["desc"], "windows_per_step": done / max(args.steps, 1), "mode": wl["mode"],
                       "sample": f"{done} windows in {args.steps} steps, the next {per_step} of the seeded set each"},
            "cpu_baseline": {"value": v, "unit": "windows/s", "cores": cores, "kind": kind,
                             "sample": f"{per_step} windows per step "
                                       f"({' '.join(wl['opts']) or 'default options'}); "
                                       + ("oracle/_ref/ref_pool: the reference library, one minipoa run per window, "
                                          f"{cores} threads pulling windows; rate = windows / (thread time / threads), "
                                          f"{done / wall_s:.3f} windows/s by wall clock"
                                          if kind == "reference" else "the restatement, one process per window")},
            "e2e": {"value": v, "unit": "windows/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=None, help="timed steps (default: 1 learned_band, 5 polishing)")
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=sorted(WORKLOADS), default="learned_band")
    ap.add_argument("--windows", type=int, default=0, help="windows per rank (default: the workload's)")
    ap.add_argument("--cpu-seconds", type=float, default=20.0)
    ap.add_argument("--plain-windows", type=int, default=8,
                    help="windows timed on the plain single-alignment kernel path (0 = skip)")
    ap.add_argument("--e2e-warmup", type=int, default=-1)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-proposer", action="store_true", help="learned_band without the proposer's plan")
    ap.add_argument("--reads-per-window", type=int, default=0,
                    help="keep only the first N reads of each window (small profiling captures; 0 = all)")
    ap.add_argument("--max-blocks", type=int, default=0,
                    help="cap the persistent grid (small profiling captures); 0 = one full wave")
    ap.add_argument("--blocks-per-sm", type=int, default=0, help="batch kernel variant: 3 (default) or 4")
    ap.add_argument("--smem-per-warp", type=int, default=0, help="shared memory per warp in bytes")
    ap.add_argument("--no-autotuned", action="store_true", help="ignore poa_b200/tuned_launch.json")
    args = ap.parse_args()
    if args.steps is None:
        args.steps = WORKLOADS[args.workload]["steps"]
    world, rank, local = dist_env()
    if args.impl == "reference":
        if rank != 0:
            return
        line = reference(args, world, rank, local, None)
        print(json.dumps(line), flush=True)
        return
    D = Dist(world)
    try:
        line = ours(args, world, rank, local, D)
    finally:
        D.close()
    if rank == 0 and line is not None:
        print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
