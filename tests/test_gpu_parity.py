"""CUDA path against the reference: golden fixtures and the CPU oracle.

Every test here runs the sm_100a kernels through the C ABI (poa_run) and
requires the output to be byte-identical to the reference's: the committed
golden outputs of the unmodified reference, and the CPU restatement in
oracle/ on larger seeded inputs.
"""
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
    CASES = json.load(fh)

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("case", CASES, ids=[c["case"] for c in CASES])
def test_golden(case):
    fa = fasta.golden_input(case)
    _, seqs = fasta.read(fa)
    params = poa_b200.Params.from_cli(case["opts"])
    with poa_b200.Context(params) as ctx:
        if "-i" in case["opts"]:
            with open(os.path.join(GOLD, case["opts"][case["opts"].index("-i") + 1]), "rb") as fh:
                text, scores = ctx.run_gfa(fh.read(), seqs, fasta.headers(fa))
        else:
            text, scores = ctx.run(seqs, fasta.headers(fa))
    with open(os.path.join(GOLD, case["case"] + ".out"), "rb") as fh:
        assert text == fh.read()
    if case["dump"]:
        recs = fasta.read_dump(os.path.join(GOLD, case["case"] + ".dump"))
        first = len(seqs) - len(recs)
        assert scores[first:] == [r[1] for r in recs]


def _oracle(oracle_bin, tmp_path, seqs, opts):
    fa = tmp_path / "in.fa"
    synth.write_fasta(str(fa), seqs)
    res = subprocess.run([oracle_bin, str(fa)] + opts, capture_output=True, check=True, timeout=600)
    return res.stdout, fasta.headers(str(fa))


SEEDED = [
    ("consensus_4kb", lambda: synth.single_graph_consensus(seed=21, nseq=6, length=4000), []),
    ("msa_3kb", lambda: synth.single_graph_msa(seed=22, nseq=10, length=3000), ["-r", "1"]),
    ("noisy_adaptive", lambda: synth.noisy_long_reads(seed=23, nreads=8, length=2500), ["-B"]),
    ("noisy_static", lambda: synth.noisy_long_reads(seed=24, nreads=8, length=2500), []),
    ("window_8pct", lambda: synth.polishing_windows(seed=25, n_windows=1).window_reads(0), []),
    ("window_15pct_adaptive", lambda: synth.windows(26, 1, (2000, 2000), (20, 24), 0.15).window_reads(0), ["-B"]),
    ("scoring_fullband", lambda: synth.single_graph_consensus(seed=27, nseq=5, length=1500),
     ["-M", "1", "-X", "3", "-O", "5", "-E", "1", "-f", "0"]),
]


@pytest.mark.parametrize("name,gen,opts", SEEDED, ids=[s[0] for s in SEEDED])
def test_seeded_vs_oracle(name, gen, opts, oracle_bin, tmp_path):
    seqs = gen()
    want, hdr = _oracle(oracle_bin, tmp_path, seqs, opts)
    with poa_b200.Context(poa_b200.Params.from_cli(opts)) as ctx:
        got, _ = ctx.run(seqs, hdr)
    assert got == want


CLI = os.path.join(os.path.dirname(HERE), "poa_b200", "minipoa_b200")
CLI_CASES = ["cons_small", "msa_small", "noisy_adaptive", "cons_scoring", "edge_mixed_msa", "window_00",
             "gfa_small", "edge_empty_read_gfa", "prog_msa", "seeded_msa", "inc_msa", "inc_adaptive"]


@pytest.mark.parametrize("name", CLI_CASES)
def test_cli_drop_in(name):
    """minipoa_b200 prints exactly what minipoa prints, given the same options."""
    case = [c for c in CASES if c["case"] == name][0]
    fa = os.path.join(GOLD, name + ".fa")
    opts = [os.path.join(GOLD, o) if k > 0 and case["opts"][k - 1] == "-i" else o for k, o in enumerate(case["opts"])]
    res = subprocess.run([CLI, fa] + opts, capture_output=True, timeout=120)
    assert res.returncode == 0, res.stderr
    with open(os.path.join(GOLD, name + ".out"), "rb") as fh:
        assert res.stdout == fh.read()
