"""minipoa itself, with its poa() replaced by the GPU drop-in.

oracle/_ref/minipoa_gpu is the reference's own main(), alignment(), graph
code and output, compiled from its sources by oracle/Makefile (`make shim`),
with poa() (include/align.h:15) taken from poa_b200/shim/minipoa_shim.cpp:
the same signature, the DP on the B200 through poa_align. Every golden case
must print exactly what the unmodified reference printed, and the shim must
report that the alignments really ran on the GPU.
"""
import json
import os
import re
import subprocess

import pytest

from tests import fasta

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
GOLD = os.path.join(HERE, "golden")
BIN = os.path.join(ROOT, "oracle", "_ref", "minipoa_gpu")
with open(os.path.join(GOLD, "manifest.json")) as fh:
    CASES = json.load(fh)

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("case", CASES, ids=[c["case"] for c in CASES])
def test_reference_main_with_gpu_poa(case):
    if not os.path.exists(BIN):
        pytest.fail("oracle/_ref/minipoa_gpu is missing: build it with `make -C oracle shim REF=<reference tree>`")
    fa = fasta.golden_input(case)
    opts = [os.path.join(GOLD, o) if k > 0 and case["opts"][k - 1] == "-i" else o
            for k, o in enumerate(case["opts"])]
    env = dict(os.environ, POA_SHIM_STATS="1")
    res = subprocess.run([BIN, fa] + opts, capture_output=True, timeout=300, env=env)
    assert res.returncode == 0, res.stderr[-2000:]
    with open(os.path.join(GOLD, case["case"] + ".out"), "rb") as fh:
        assert res.stdout == fh.read()
    m = re.search(rb"poa_shim: (\d+) poa\(\) calls on the GPU", res.stderr)
    if case["nseq"] >= 2 or (case["nseq"] >= 1 and "-i" in case["opts"]):
        # every read after the first is aligned by poa(): the shim ran them
        assert m and int(m.group(1)) >= 1, res.stderr[-500:]
