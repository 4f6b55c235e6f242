"""Seeded random inputs: the CPU restatement and the CPU kernel model against
the unmodified reference (oracle/_ref/minipoa, compiled from the reference's
sources by oracle/Makefile). Skipped where the reference binary is absent.

A case where the reference itself exits non-zero is skipped: minipoa has no
error path for the inputs it rejects (it exits inside poa(), src/align.cpp:
1584-1588, 1730-1731), so there is no output to match.
"""
import ctypes
import os
import subprocess

import pytest

from tests import fasta, fuzzcases
from tests.test_model_golden import model, opts_to_params  # noqa: F401  (fixture)

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.path.join(ROOT, "oracle", "_ref", "minipoa")
SEEDS = list(range(int(os.environ.get("POA_FUZZ_CASES", "150"))))

pytestmark = pytest.mark.skipif(not os.path.exists(REF), reason="reference not built (make -C oracle ref)")


def _write(tmp_path, reads):
    fa = tmp_path / "in.fa"
    with open(fa, "wb") as fh:
        for k, r in enumerate(reads):
            fh.write(b">r%d\n%s\n" % (k + 1, r))
    return str(fa)


def _reference(fa, opts):
    res = subprocess.run([REF, fa] + opts, capture_output=True, timeout=120)
    if res.returncode != 0:
        pytest.skip(f"the reference exits {res.returncode} on this input")
    return res.stdout


@pytest.mark.parametrize("seed", SEEDS)
def test_restatement_vs_reference(seed, oracle_bin, tmp_path):
    reads, opts = fuzzcases.case(seed)
    fa = _write(tmp_path, reads)
    want = _reference(fa, opts)
    got = subprocess.run([oracle_bin, fa] + opts, capture_output=True, check=True, timeout=120).stdout
    assert got == want


@pytest.mark.parametrize("seed", SEEDS)
def test_model_vs_reference(seed, model, tmp_path):  # noqa: F811
    reads, opts = fuzzcases.case(seed)
    fa = _write(tmp_path, reads)
    want = _reference(fa, opts)
    names, seqs = fasta.read(fa)
    n = len(seqs)
    arr = (ctypes.c_char_p * max(n, 1))(*seqs)
    lens = (ctypes.c_int * max(n, 1))(*[len(s) for s in seqs])
    par = (ctypes.c_int * 10)(*opts_to_params(opts))
    hdrs = fasta.headers(fa)
    harr = (ctypes.c_char_p * max(n, 1))(*[h.encode() if isinstance(h, str) else h for h in hdrs])
    out = ctypes.c_void_p()
    st = model.model_run_gfa(n, arr, lens, par, None, -1, harr, ctypes.byref(out), None, 0)
    assert st == 0
    got = ctypes.string_at(out.value)
    model.model_free(out)
    assert got == want
