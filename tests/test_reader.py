"""The product's FASTA / FASTQ reader (poa_b200/csrc/reader.cpp), on the CPU.

minipoa reads its input with kseq over gzread (src/handle_input.cpp:13-43):
plain or gzip files, FASTA or FASTQ, multi-line sequences, the name up to the
first blank and the rest of the header as the comment. The streamed batch
input (poa_batch_consensus_files) and the CLI use this reader; here it must
agree with tests/fasta.py (the same semantics) on every golden input and on
FASTQ, gzip and CRLF variants.
"""
import glob
import gzip
import os
import subprocess

import pytest

from tests import fasta

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
BIN = os.path.join(HERE, "model", "build", "reader_check")


@pytest.fixture(scope="module")
def reader():
    srcs = [os.path.join(HERE, "model", "reader_check.cpp"), os.path.join(ROOT, "poa_b200", "csrc", "reader.cpp")]
    os.makedirs(os.path.dirname(BIN), exist_ok=True)
    if not os.path.exists(BIN) or max(os.path.getmtime(s) for s in srcs) > os.path.getmtime(BIN):
        subprocess.run(["g++", "-O2", "-std=c++17", "-I" + os.path.join(ROOT, "poa_b200", "csrc")] + srcs +
                       ["-lz", "-o", BIN], check=True)
    return BIN


def _records(binary, path):
    out = subprocess.run([binary, path], capture_output=True, check=True).stdout.decode()
    return [tuple(ln.split("\t")) for ln in out.split("\n") if ln]


def _want(path):
    return [(n, c, s.decode()) for n, c, s in fasta.read_records(path)]


@pytest.mark.parametrize("path", sorted(glob.glob(os.path.join(HERE, "golden", "*.fa"))),
                         ids=lambda p: os.path.basename(p))
def test_golden_inputs(reader, path):
    assert _records(reader, path) == _want(path)


def test_gzip_fastq_and_crlf(reader, tmp_path):
    src = os.path.join(HERE, "golden", "edge_mixed.fa")
    recs = _want(src)
    # gzip of the same FASTA
    gz = tmp_path / "a.fa.gz"
    with open(src, "rb") as fh, gzip.open(gz, "wb") as out:
        out.write(fh.read())
    assert _records(reader, str(gz)) == recs
    # FASTQ with multi-line sequence and quality, including a quality line starting with '@'
    fq = tmp_path / "b.fq"
    with open(fq, "w") as fh:
        for k, (n, c, s) in enumerate(recs):
            fh.write(f"@{n}{' ' + c if c else ''}\n{s[:7]}\n{s[7:]}\n+\n{('@' + 'I' * len(s))[:len(s)]}\n")
    assert _records(reader, str(fq)) == [(n, c, s) for n, c, s in recs]
    # CRLF line ends, sequence wrapped at 10
    crlf = tmp_path / "c.fa"
    with open(crlf, "wb") as fh:
        for n, c, s in recs:
            fh.write(f">{n}{' ' + c if c else ''}\r\n".encode())
            for i in range(0, len(s), 10):
                fh.write(s[i:i + 10].encode() + b"\r\n")
    assert _records(reader, str(crlf)) == recs


def test_unreadable_file(reader, tmp_path):
    res = subprocess.run([reader, str(tmp_path / "missing.fa")], capture_output=True)
    assert res.returncode == 1
