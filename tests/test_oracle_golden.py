"""The CPU restatement (oracle/) against the reference's own outputs.

Every fixture in tests/golden/ was produced by the unmodified reference
(oracle/_ref/minipoa and oracle/ref_harness, see tests/golden/make_golden.py).
The restatement must reproduce the CLI output byte for byte and, where a
per-call dump exists, every alignment() score and path.
"""
import json
import os
import subprocess

import pytest

from tests import fasta

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
with open(os.path.join(GOLD, "manifest.json")) as fh:
    MANIFEST = json.load(fh)
# seeding (-S), the progressive order (-p) and GFA input (-i) are host-side steps the
# restatement leaves out; the product's host driver is checked on them through
# the CPU model of the kernels (test_model_golden.py) and on the GPU
CASES = [c for c in MANIFEST if not {"-S", "-p", "-i"} & set(c["opts"])]


@pytest.mark.parametrize("case", CASES, ids=[c["case"] for c in CASES])
def test_restatement_matches_reference(case, oracle_bin, tmp_path):
    fa = fasta.golden_input(case)
    args = [oracle_bin, fa] + case["opts"]
    dump = tmp_path / "o.dump"
    if case["dump"]:
        args += ["-d", str(dump)]
    res = subprocess.run(args, capture_output=True, check=True, timeout=120)
    with open(os.path.join(GOLD, case["case"] + ".out"), "rb") as fh:
        assert res.stdout == fh.read()
    if case["dump"]:
        with open(os.path.join(GOLD, case["case"] + ".dump"), "rb") as fh:
            assert dump.read_bytes() == fh.read()
