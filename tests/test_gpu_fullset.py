"""The batched engine on the benchmark's full window sets, every window checked.

tests/golden/windows_polishing.txt and windows_learned_band.txt hold, per
window, the first 16 hex digits of the md5 of the consensus the unmodified
reference prints for that window (oracle/_ref/ref_pool, one minipoa run per
window; made by tests/golden/make_golden.py --windows). The sets are
regenerated here from their seeds: 20,000 polishing windows (500 +- 100 bp,
4-64 reads, 8 % error, static band) and 5,000 learned-band windows (2 kb,
20-100 reads, 15 % error, 1 % chimeric reads, -B, planned by the proposer).
"""
import hashlib
import json
import os

import pytest

import poa_b200
from poa_b200 import synth

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = os.path.join(HERE, "golden")

pytestmark = pytest.mark.gpu


def _manifest(name):
    path = os.path.join(GOLD, name + ".txt")
    if not os.path.exists(path):
        pytest.fail(f"{path} is missing: make it with tests/golden/make_golden.py --windows")
    with open(path) as fh:
        head = json.loads(fh.readline()[2:])
        return head, [ln.strip() for ln in fh if ln.strip()]


@pytest.mark.parametrize("name,proposer", [("windows_polishing", False), ("windows_learned_band", True)])
def test_every_window_matches_reference(name, proposer):
    head, want = _manifest(name)
    ws = getattr(synth, head["generator"])(**head["kwargs"])
    assert ws.n_windows == len(want) == head["windows"]
    with poa_b200.Context(poa_b200.Params.from_cli(head["opts"])) as ctx:
        if proposer:
            ctx.batch_use_proposer(poa_b200.Proposer(weights=poa_b200.PROP_WEIGHTS))
        cons, status = ctx.batch_consensus(ws)
        st = ctx.batch_stats()
    assert all(s == 0 for s in status)
    got = [hashlib.md5(c).hexdigest()[:16] for c in cons]
    bad = [w for w in range(ws.n_windows) if got[w] != want[w]]
    assert not bad, f"{len(bad)} of {ws.n_windows} windows differ from the reference, first {bad[:10]}"
    if proposer:
        # the plan held: windows that outgrew their planned slot stay under 2 %
        assert st["fallback"] <= 0.02 * ws.n_windows
