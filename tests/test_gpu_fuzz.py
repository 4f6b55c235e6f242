"""Seeded random inputs through the CUDA path (poa_run, both single-alignment
kernels): byte-identical to the CPU restatement in oracle/, which
tests/test_oracle_fuzz.py checks against the unmodified reference on the same
cases, and to the reference binary itself where oracle/_ref is present.
"""
import os
import subprocess

import pytest

import poa_b200
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
