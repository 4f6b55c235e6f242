"""The committed launch-shape table (poa_b200/tuned_launch.json, written by
python -m poa_b200.autotune) is what bench.py and Context.batch_autotuned
apply: every workload the autotuner knows has an entry, each entry picks one
of the shapes it measured, and the shape is one the engine accepts (CPU only).
"""
import json
import os

from poa_b200 import autotune

HERE = os.path.dirname(os.path.abspath(__file__))
TUNED = os.path.join(os.path.dirname(HERE), "poa_b200", "tuned_launch.json")


def test_every_workload_has_a_measured_shape():
    with open(TUNED) as fh:
        table = json.load(fh)
    assert set(autotune.WORKLOADS) <= set(table)
    for wl, t in table.items():
        shape = (t["blocks_per_sm"], t["smem_per_warp"])
        assert shape in autotune.CANDIDATES, wl
        measured = {(m["blocks_per_sm"], m["smem_per_warp"]): m["ms"] for m in t["measured"]}
        assert shape in measured, wl
        # the recorded choice is the fastest of its own measurements
        assert measured[shape] == min(measured.values()), wl
        assert t["smem_per_warp"] % 16 == 0 and t["blocks_per_sm"] in (3, 4)


def test_load_returns_the_entry():
    for wl in autotune.WORKLOADS:
        t = autotune.load(wl)
        assert t is not None and t["blocks_per_sm"] in (3, 4)
