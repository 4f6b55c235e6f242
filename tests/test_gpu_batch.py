"""Batched window engine (graph fusion, topsort and consensus on the device)
against the reference: every window's consensus must equal minipoa's output
on that window's reads."""
import json
import os
import subprocess

import pytest

import poa_b200
from poa_b200 import synth
from tests import fasta

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = os.path.join(HERE, "golden")
with open(os.path.join(GOLD, "manifest.json")) as fh:
    MANIFEST = {c["case"]: c for c in json.load(fh)}

pytestmark = pytest.mark.gpu


def _golden_windows(names):
    reads, offs = [], [0]
    for nm in names:
        _, seqs = fasta.read(os.path.join(GOLD, nm + ".fa"))
        reads.extend(seqs)
        offs.append(offs[-1] + len(seqs))
    return synth.pack_windows_from_reads(reads, offs)


def _cons_of(out_text):
    lines = out_text.split(b"\n")
    return lines[1] if len(lines) > 1 else b""


def _check(names, opts, upload_path=True):
    ws = _golden_windows(names)
    with poa_b200.Context(poa_b200.Params.from_cli(opts)) as ctx:
        if upload_path:
            ctx.batch_upload(ws)
            ctx.batch_run()
            cons, st = ctx.batch_download()
        else:
            cons, st = ctx.batch_consensus(ws)
    for w, nm in enumerate(names):
        want = _cons_of(open(os.path.join(GOLD, nm + ".out"), "rb").read())
        assert st[w] == 0, (nm, st[w])
        assert cons[w] == want, nm


def test_batch_golden_windows():
    _check([f"window_{w:02d}" for w in range(10)], [])


def test_batch_golden_windows_e2e_entry():
    _check([f"window_{w:02d}" for w in range(10)], [], upload_path=False)


def test_batch_golden_adaptive():
    _check([f"lbwindow_{w:02d}" for w in range(3)] + ["noisy_adaptive"], ["-B"])


def test_batch_golden_edges():
    _check(["edge_mixed", "edge_single", "edge_empty_read", "edge_all_n", "edge_identical", "cons_small"], [])


def test_batch_golden_fullband():
    # f = 0: every row spans the whole query (the dynamic-band fill without the adaptive update)
    _check(["cons_fullband"], ["-f", "0"])


def test_batch_golden_edges_adaptive():
    _check(["edge_mixed_adaptive", "edge_single_adaptive", "edge_empty_read_adaptive", "edge_all_n_adaptive",
            "edge_identical_adaptive"], ["-B"])


def test_batch_golden_scoring():
    _check(["cons_scoring"], MANIFEST["cons_scoring"]["opts"])


def test_batch_vs_oracle(oracle_bin, tmp_path):
    ws = synth.polishing_windows(seed=31, n_windows=40)
    with poa_b200.Context() as ctx:
        ctx.batch_upload(ws)
        ctx.batch_run()
        cons, st = ctx.batch_download()
        # a second run on the resident inputs must give the same answer
        ctx.batch_run()
        cons2, st2 = ctx.batch_download()
    assert cons == cons2 and st == st2
    for w in range(ws.n_windows):
        fa = tmp_path / f"w{w}.fa"
        synth.write_fasta(str(fa), ws.window_reads(w))
        want = subprocess.run([oracle_bin, str(fa)], capture_output=True, check=True).stdout
        assert st[w] == 0
        assert cons[w] == _cons_of(want), w


def test_batch_learned_band_config_windows(oracle_bin, tmp_path):
    """2,000 bp windows, 15 % error, 20-24 reads, adaptive band (-B), 1 chimeric
    read in 10: the configuration the learned band proposer works on."""
    ws = synth.windows(41, 3, (2000, 2000), (20, 24), 0.15, chimeric=0.1)
    with poa_b200.Context(poa_b200.Params(ab_band=True)) as ctx:
        ctx.batch_upload(ws)
        ctx.batch_run()
        cons, st = ctx.batch_download()
    for w in range(ws.n_windows):
        fa = tmp_path / f"w{w}.fa"
        synth.write_fasta(str(fa), ws.window_reads(w))
        want = subprocess.run([oracle_bin, str(fa), "-B"], capture_output=True, check=True, timeout=600).stdout
        assert st[w] == 0
        assert cons[w] == _cons_of(want), w


def test_batch_capacity_retry():
    """A window far larger than the rest outgrows the slot sized from the batch
    statistics at first; the engine re-runs it with larger capacities and the
    result is still the reference's."""
    small = synth.windows(42, 30, (300, 300), (4, 6), 0.08)
    big = synth.windows(43, 1, (600, 600), (60, 60), 0.40)
    reads, offs = [], [0]
    for w in range(small.n_windows):
        reads += small.window_reads(w)
        offs.append(len(reads))
    reads += big.window_reads(0)
    offs.append(len(reads))
    ws = synth.pack_windows_from_reads(reads, offs)
    with poa_b200.Context() as ctx:
        ctx.batch_upload(ws)
        ctx.batch_run()
        cons, st = ctx.batch_download()
        stats = ctx.batch_stats()
    assert all(x == 0 for x in st)
    solo = poa_b200.run(big.window_reads(0))
    assert b">consensus sequence\n" + cons[-1] + b"\n" == solo
    print("retried", stats["retried"], "launches", stats["launches"])


def test_autotune_small(tmp_path):
    """The launch-shape autotuner runs every candidate on a small sample, picks one,
    and a tuned context gives the same consensus as the default shape."""
    from poa_b200 import autotune
    t = autotune.tune("polishing", windows=300, log=lambda *a: None)
    assert (t["blocks_per_sm"], t["smem_per_warp"]) in autotune.CANDIDATES
    assert len(t["measured"]) >= 1
    ws = synth.polishing_windows(seed=33, n_windows=50)
    with poa_b200.Context() as ctx:
        cons0, st0 = ctx.batch_consensus(ws)
        ctx.batch_config(blocks_per_sm=t["blocks_per_sm"], smem_per_warp=t["smem_per_warp"])
        cons1, st1 = ctx.batch_consensus(ws)
        cons2, st2 = ctx.batch_consensus(ws)  # replayed launch graph
    assert st0 == [0] * 50 and cons1 == cons0 and st1 == st0 and cons2 == cons0


@pytest.mark.parametrize("opts", [[], ["-B"]])
def test_batch_empty_windows(opts):
    """Windows without reads, or with one empty read, give the empty consensus,
    as minipoa does on such input; their neighbours are unaffected."""
    _, w0 = fasta.read(os.path.join(GOLD, "window_00.fa"))
    reads = list(w0) + [b""] + [b"ACGT"]
    offs = [0, len(w0), len(w0), len(w0) + 1, len(w0) + 2]
    ws = synth.pack_windows_from_reads(reads, offs)
    with poa_b200.Context(poa_b200.Params.from_cli(opts)) as ctx:
        cons, st = ctx.batch_consensus(ws)
        text0, _ = ctx.run(list(w0), None)
    assert st == [0, 0, 0, 0]
    assert cons[0] == text0.split(b"\n")[1]
    assert cons[1] == b"" and cons[2] == b""
    assert cons[3] == b"ACGT"


def test_streamed_files_match_reference(tmp_path):
    """poa_batch_consensus_files: one file per window (plain FASTA, gzip FASTA,
    FASTQ), parsed on host threads in chunks of 4 while the previous chunk runs;
    every consensus equals the reference's output for that window."""
    import gzip
    names = [f"window_{w:02d}" for w in range(10)] + ["lbwindow_00", "edge_mixed"]
    paths = []
    for k, nm in enumerate(names):
        src = os.path.join(GOLD, nm + ".fa")
        if nm.startswith("lbwindow"):
            continue  # adaptive band: its own context below
        if k % 3 == 1:
            p = tmp_path / f"{nm}.fa.gz"
            with open(src, "rb") as fh, gzip.open(p, "wb") as out:
                out.write(fh.read())
        elif k % 3 == 2:
            p = tmp_path / f"{nm}.fq"
            with open(p, "w") as fh:
                for n_, c_, s_ in fasta.read_records(src):
                    fh.write(f"@{n_}\n{s_.decode()}\n+\n{'I' * len(s_)}\n")
        else:
            p = src
        paths.append((nm, str(p)))
    with poa_b200.Context(poa_b200.Params()) as ctx:
        cons, status = ctx.batch_consensus_files([p for _, p in paths], chunk=4, threads=3)
    for (nm, _), c, s in zip(paths, cons, status):
        with open(os.path.join(GOLD, nm + ".out"), "rb") as fh:
            assert s == 0 and b">consensus sequence\n" + c + b"\n" == fh.read(), nm


def _many_pred_window(seed):
    """Reads that delete 1..23 bases before one template position, substitute its
    left neighbour or insert a base before it: that node gets 22 in-window
    predecessors (seed 61), beyond the 15 the fill's one-pass record choices
    hold, so its row takes the full second pass."""
    import numpy as np
    rng = np.random.default_rng(seed)
    t = synth.to_ascii(synth.random_root(rng, 320))
    P = 200
    sub = [t[:P - 1] + bytes([b]) + t[P:] for b in b"ACGT" if b != t[P - 1]]
    ins = [t[:P] + bytes([b]) + t[P:] for b in b"ACGT"]
    return [t] + [t[:P - k] + t[P:] for k in range(1, 24)] + sub + ins  # one node with 22 predecessors


@pytest.mark.parametrize("opts", [[], ["-B"]])
def test_batch_rows_with_many_predecessors(opts, oracle_bin, tmp_path):
    wins = [_many_pred_window(s) for s in (61, 62)]
    reads, offs = [], [0]
    for rs in wins:
        reads.extend(rs)
        offs.append(offs[-1] + len(rs))
    ws = synth.pack_windows_from_reads(reads, offs)
    with poa_b200.Context(poa_b200.Params.from_cli(opts)) as ctx:
        cons, st = ctx.batch_consensus(ws)
    for w, rs in enumerate(wins):
        fa = tmp_path / f"w{w}.fa"
        synth.write_fasta(str(fa), rs)
        want = _cons_of(subprocess.run([oracle_bin, str(fa)] + opts, capture_output=True, check=True).stdout)
        assert st[w] == 0 and cons[w] == want


@pytest.mark.parametrize("opts,smem", [([], 0), (["-B"], 0), (["-B"], 10240)],
                         ids=["static", "adaptive", "adaptive_query_in_slot"])
def test_batch_long_reads(opts, smem, oracle_bin, tmp_path):
    """Windows of 9-12 kb reads at 10 % error. With 10 KB of shared memory per
    warp the adaptive fill cannot stage a 12 kb query next to its records and
    reads it from the slot instead; every variant must print the reference's
    consensus."""
    ws = synth.windows(51, 2, (9000, 12000), (5, 6), 0.10)
    with poa_b200.Context(poa_b200.Params.from_cli(opts)) as ctx:
        if smem:
            ctx.batch_config(smem_per_warp=smem)
        cons, st = ctx.batch_consensus(ws)
    for w in range(ws.n_windows):
        fa = tmp_path / f"w{w}.fa"
        synth.write_fasta(str(fa), ws.window_reads(w))
        want = subprocess.run([oracle_bin, str(fa)] + opts, capture_output=True, check=True, timeout=900).stdout
        assert st[w] == 0
        assert cons[w] == _cons_of(want), w
