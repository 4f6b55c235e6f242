"""Seeded random inputs through the CUDA path (poa_run, both single-alignment
kernels): byte-identical to the CPU restatement in oracle/, which
tests/test_oracle_fuzz.py checks against the unmodified reference on the same
cases, and to the reference binary itself where oracle/_ref is present.
"""
import os
import subprocess

import pytest

import poa_b200
from poa_b200 import synth
from tests import fasta, fuzzcases

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.path.join(ROOT, "oracle", "_ref", "minipoa")
SEEDS = list(range(int(os.environ.get("POA_FUZZ_CASES", "150"))))

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("seed", SEEDS)
def test_fuzz_vs_oracle(seed, oracle_bin, tmp_path):
    reads, opts = fuzzcases.case(seed)
    fa = tmp_path / "in.fa"
    with open(fa, "wb") as fh:
        for k, r in enumerate(reads):
            fh.write(b">r%d\n%s\n" % (k + 1, r))
    want = subprocess.run([oracle_bin, str(fa)] + opts, capture_output=True, check=True, timeout=120).stdout
    if os.path.exists(REF):
        ref = subprocess.run([REF, str(fa)] + opts, capture_output=True, timeout=120)
        if ref.returncode == 0:
            assert ref.stdout == want
    _, seqs = fasta.read(str(fa))
    with poa_b200.Context(poa_b200.Params.from_cli(opts)) as ctx:
        got, _ = ctx.run(seqs, fasta.headers(str(fa)))
    assert got == want


BATCH_OPTS = [[], ["-B"], ["-f", "0"], ["-M", "3", "-X", "5", "-O", "6", "-E", "1", "-b", "20", "-f", "10"],
              ["-M", "1", "-X", "2", "-O", "3", "-E", "1", "-B"]]


@pytest.mark.parametrize("opts", BATCH_OPTS, ids=["static", "adaptive", "fullband", "scoring", "scoring_adaptive"])
def test_batch_fuzz_vs_oracle(opts, oracle_bin, tmp_path):
    """The same random reads as windows of one batched launch (graph, topsort
    and consensus on the device): every window's consensus equals the
    restatement's on that window's reads."""
    cases = [fuzzcases.case(s)[0] for s in range(120)]
    reads, offs = [], [0]
    for c in cases:
        reads.extend(c)
        offs.append(offs[-1] + len(c))
    ws = synth.pack_windows_from_reads(reads, offs)
    with poa_b200.Context(poa_b200.Params.from_cli(opts)) as ctx:
        cons, st = ctx.batch_consensus(ws)
    for w, c in enumerate(cases):
        fa = tmp_path / f"w{w}.fa"
        with open(fa, "wb") as fh:
            for k, r in enumerate(c):
                fh.write(b">r%d\n%s\n" % (k + 1, r))
        out = subprocess.run([oracle_bin, str(fa)] + opts, capture_output=True, check=True, timeout=120).stdout
        lines = out.split(b"\n")
        assert st[w] == 0, (w, st[w])
        assert cons[w] == (lines[1] if len(lines) > 1 else b""), w
