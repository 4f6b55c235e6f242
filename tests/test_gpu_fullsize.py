"""Full-size single-graph configurations on the GPU, bit-exact with the
reference: the inputs are regenerated from their seeds and the md5 of
poa_run's output must equal the md5 of the unmodified reference's stdout
(tests/golden/fullsize.json, made by tests/golden/make_golden.py --fullsize).

config 1: 10 x 16,569 bp consensus; config 2: 100 x 16.5 kb MSA with
minimizer seeding (-S -r1, 2,400 sub-window DPs); config 3: 30 x 10 kb noisy
reads with the adaptive band (-B) and the static band.
"""
import hashlib
import json
import os
import time

import pytest

import poa_b200
from poa_b200 import synth

HERE = os.path.dirname(os.path.abspath(__file__))
with open(os.path.join(HERE, "golden", "fullsize.json")) as fh:
    CASES = json.load(fh)

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("case", CASES, ids=[c["case"] for c in CASES])
def test_fullsize_md5(case):
    reads = getattr(synth, case["generator"])(**case["kwargs"])
    headers = [f"seq{i + 1} " for i in range(len(reads))]
    with poa_b200.Context(poa_b200.Params.from_cli(case["opts"])) as ctx:
        t0 = time.perf_counter()
        text, _ = ctx.run(reads, headers)
        dt = time.perf_counter() - t0
        st = ctx.stats()
    print(f"{case['case']}: {dt:.2f}s wall, {st['alignments']} DP calls, {st['cells'] / 1e6:.0f} M cells "
          f"(reference CPU {case['reference_seconds']}s)")
    assert len(text) == case["bytes"]
    assert hashlib.md5(text).hexdigest() == case["md5"]
