"""Generate the golden fixtures in this directory from the UNMODIFIED reference.

Run from the repository root after ``make -C oracle ref`` (which compiles the
reference's own sources into ``oracle/_ref/``):

    python tests/golden/make_golden.py              # small cases
    python tests/golden/make_golden.py --fullsize   # md5 of full-size runs
    python tests/golden/make_golden.py --windows    # per-window manifests of the
                                                    # full batched window sets
    python tests/golden/make_golden.py --fixtures   # the reference's own data
                                                    # file (POA_REF_DIR/data)

For every case it writes ``<case>.fa`` (seeded synthetic input),
``<case>.out`` (the reference CLI's stdout, byte for byte: consensus, MSA or GFA) and, where the case
has per-call records, ``<case>.dump`` (one score + path per alignment() call,
from ``oracle/ref_harness``). ``manifest.json`` lists the cases and options; an ``-i`` case names its graph
file ``<case>.gfa`` (relative to this directory), the reference's own GFA
output on seeded base reads.
The fixtures are kept small so the CPU test-suite stays fast; the full-size
configurations are checked on the GPU through size-independent properties and
against the CPU restatement.
"""
from __future__ import annotations

import json
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
from poa_b200 import synth  # noqa: E402

REF_BIN = os.path.join(ROOT, "oracle", "_ref", "minipoa")
POOL = os.path.join(ROOT, "oracle", "_ref", "ref_pool")
HARNESS = os.path.join(ROOT, "oracle", "_ref", "ref_harness")


def edge_reads():
    rng = np.random.default_rng(7)
    t = synth.to_ascii(synth.random_root(rng, 300))
    extra = synth.to_ascii(synth.random_root(rng, 120))
    return {
        # ragged lengths, an N run, lower case, a prefix, a 5 bp read, an
        # extended read, a read with N, an unrelated (reversed) read
        "edge_mixed": [t, t[:150] + b"NNNN" + t[154:], t.lower(), t[20:280], t[:5],
                       t + extra, b"ACGTN", t[::-1][:200]],
        "edge_single": [t],
        "edge_empty_read": [t, b"", t[:100]],
        "edge_all_n": [b"NNNNNNNN", b"NNNNN", t[:50]],
        "edge_identical": [t[:200]] * 5,
    }


def long_indel_reads():
    """Reads with 45-80 bp insertions and deletions against one template: the
    graph gets rows whose successor lies 45+ rows ahead in rank order, so the
    kernels' row rings must hand those rows to the global row store."""
    rng = np.random.default_rng(31)
    t = synth.to_ascii(synth.random_root(rng, 1500))
    ins = [synth.to_ascii(synth.random_root(rng, k)) for k in (60, 45, 80)]
    sub = bytearray(t)
    for x in rng.choice(len(sub), 15, replace=False):
        sub[x] = b"ACGT"[(b"ACGT".index(sub[x]) + 1) % 4]
    return [t,
            t[:400] + ins[0] + t[400:900] + t[960:],
            t[:400] + ins[0] + t[400:],
            t[:900] + t[960:],
            bytes(sub[:1200]) + ins[1] + bytes(sub[1200:]),
            t[:250] + ins[2] + t[250:700] + t[780:],
            t]


def cases():
    out = []
    out.append(("cons_small", synth.single_graph_consensus(seed=11, nseq=6, length=800), [], True))
    out.append(("cons_scoring", synth.single_graph_consensus(seed=11, nseq=6, length=800),
                ["-M", "3", "-X", "5", "-O", "6", "-E", "1", "-b", "20", "-f", "10"], True))
    out.append(("cons_fullband", synth.single_graph_consensus(seed=16, nseq=5, length=400), ["-f", "0"], True))
    out.append(("msa_small", synth.single_graph_msa(seed=12, nseq=8, length=700), ["-r", "1"], True))
    noisy = synth.noisy_long_reads(seed=13, nreads=6, length=1200)
    out.append(("noisy_adaptive", noisy, ["-B"], True))
    out.append(("noisy_static", noisy, [], True))
    out.append(("noisy_adaptive_msa", noisy, ["-B", "-r", "1"], False))
    ws = synth.polishing_windows(seed=14, n_windows=10)
    for w in range(ws.n_windows):
        out.append((f"window_{w:02d}", ws.window_reads(w), [], w < 3))
    lb = synth.windows(15, 3, (600, 600), (8, 12), 0.15, chimeric=0.1)
    for w in range(lb.n_windows):
        out.append((f"lbwindow_{w:02d}", lb.window_reads(w), ["-B"], w < 2))
    for name, reads in edge_reads().items():
        out.append((name, reads, [], True))
        out.append((name + "_adaptive", reads, ["-B"], False))
        out.append((name + "_msa", reads, ["-r", "1"], False))
        out.append((name + "_gfa", reads, ["-r", "2"], False))
    li = long_indel_reads()
    out.append(("long_indel", li, [], True))
    out.append(("long_indel_fullband", li, ["-f", "0"], True))
    out.append(("long_indel_adaptive", li, ["-B"], True))
    out.append(("long_indel_msa", li, ["-r", "1"], False))
    seed_in = synth.single_graph_msa(seed=17, nseq=10, length=3000)
    out.append(("seeded_msa", seed_in, ["-S", "-r", "1"], False))
    out.append(("seeded_cons", seed_in, ["-S"], False))
    out.append(("seeded_gfa", seed_in, ["-S", "-r", "2"], False))
    out.append(("gfa_small", synth.single_graph_msa(seed=19, nseq=8, length=600), ["-r", "2"], False))
    out.append(("gfa_adaptive", noisy, ["-B", "-r", "2"], False))
    prog = synth.single_graph_msa(seed=23, nseq=12, length=1500)
    out.append(("prog_msa", prog, ["-p", "-r", "1"], False))
    out.append(("prog_cons", prog, ["-p"], False))
    # no "-p -r 2" case: the reference aborts there (output_gfa sizes each path by
    # rid_to_ord but fills it by read ord, src/graph.cpp:369, 397-401)
    out.append(("prog_adaptive", noisy, ["-p", "-B"], False))
    out.append(("prog_seeded_msa", seed_in, ["-p", "-S", "-r", "1"], False))
    out.append(("prog_edge", edge_reads()["edge_mixed"], ["-p", "-r", "1"], False))
    return out


def inc_cases():
    """-i cases: (name, reads to add, options, reads the graph is made of). The
    graph file <name>.gfa is the reference's own -r 2 output on the base reads.
    Not covered: -i with -S or -p (the reference aborts) and with -r 2 (it
    writes the GFA paths out of bounds)."""
    fam = synth.single_graph_msa(seed=19, nseq=12, length=600)
    noisy = synth.noisy_long_reads(seed=29, nreads=6, length=900)
    names = [f"g{i}" for i in range(12)]
    return [
        ("inc_cons", fam[8:], [], (fam[:8], names[:8])),
        ("inc_msa", fam[8:], ["-r", "1"], (fam[:8], names[:8])),
        ("inc_adaptive", noisy[3:], ["-B"], (noisy[:3], names[:3])),
        ("inc_graph_only", [], [], (fam[:5], names[:5])),
        ("inc_graph_only_msa", [], ["-r", "1"], (fam[:5], names[:5])),
    ]


# Full-size configurations: inputs are regenerated from their seeds by the
# tests; only the md5 of the reference's stdout is stored.
FULLSIZE = [
    ("config1_consensus_10x16569", "single_graph_consensus", dict(seed=1), []),
    ("config2_msa_100x16500", "single_graph_msa", dict(seed=2), ["-S", "-r", "1"]),
    ("config3_noisy_30x10k_adaptive", "noisy_long_reads", dict(seed=3), ["-B"]),
    ("config3_noisy_30x10k_static", "noisy_long_reads", dict(seed=3), []),
]


def fullsize():
    import hashlib
    import time
    out = []
    for name, gen, kw, opts in FULLSIZE:
        reads = getattr(synth, gen)(**kw)
        fa = os.path.join("/tmp", name + ".fa")
        synth.write_fasta(fa, reads)
        t0 = time.time()
        res = subprocess.run([REF_BIN, fa] + opts, capture_output=True, check=True)
        dt = time.time() - t0
        out.append({"case": name, "generator": gen, "kwargs": kw, "opts": opts,
                    "md5": hashlib.md5(res.stdout).hexdigest(), "bytes": len(res.stdout),
                    "reference_seconds": round(dt, 2)})
        os.unlink(fa)
    with open(os.path.join(HERE, "fullsize.json"), "w") as fh:
        json.dump(out, fh, indent=1)


# Full batched window sets (the benchmark's two workloads at full size): the
# reference runs every window (oracle/_ref/ref_pool, one minipoa run per
# window on all host threads) and the manifest keeps the first 16 hex digits
# of each window's consensus md5, in window order.
WINDOW_SETS = [
    ("windows_polishing", "polishing_windows", dict(seed=4, n_windows=20000), []),
    ("windows_learned_band", "learned_band_windows", dict(seed=5, n_windows=5000), ["-B"]),
]


def window_manifests(only=None):
    import hashlib
    import time
    for name, gen, kw, opts in WINDOW_SETS:
        if only and name not in only:
            continue
        ws = getattr(synth, gen)(**kw)
        pw, co = os.path.join("/tmp", name + ".pwin"), os.path.join("/tmp", name + ".cons")
        synth.write_pwin(pw, ws)
        t0 = time.time()
        res = subprocess.run([POOL] + opts + [pw, co], capture_output=True, text=True, check=True)
        cons = synth.read_cons_file(co)
        assert len(cons) == ws.n_windows, res.stdout
        head = {"generator": gen, "kwargs": kw, "opts": opts, "windows": ws.n_windows,
                "hash": "md5(consensus bases)[:16]", "reference_seconds": round(time.time() - t0, 1),
                "pool": res.stdout.strip()}
        with open(os.path.join(HERE, name + ".txt"), "w") as fh:
            fh.write("# " + json.dumps(head) + "\n")
            for c in cons:
                fh.write(hashlib.md5(c).hexdigest()[:16] + "\n")
        os.unlink(pw)
        os.unlink(co)
        print(name, head["reference_seconds"], "s")


# The reference's only fixture, data/mtDNA.fasta (393 HVS-II control-region
# reads), with the modes its README runs plus -r 2 and -B; copied into
# mtdna.fa and shared by the four cases ("input" in the manifest). Not
# covered: `-S -t 12 -r1` (the README's second command) faults in the
# reference on this file (segmentation fault), so it has no output to match.
REF_FIXTURES = [("mtdna_cons", []), ("mtdna_msa", ["-r", "1"]), ("mtdna_gfa", ["-r", "2"]),
                ("mtdna_adaptive", ["-B"])]


def reference_fixtures():
    import shutil
    ref_dir = os.environ.get("POA_REF_DIR", "/root/reference")
    src = os.path.join(ref_dir, "data", "mtDNA.fasta")
    dst = os.path.join(HERE, "mtdna.fa")
    shutil.copyfile(src, dst)
    with open(os.path.join(HERE, "manifest.json")) as fh:
        manifest = [c for c in json.load(fh) if not c["case"].startswith("mtdna_")]
    _, seqs = fasta_read(dst)
    for name, opts in REF_FIXTURES:
        res = subprocess.run([REF_BIN, dst] + opts, capture_output=True, check=True)
        with open(os.path.join(HERE, name + ".out"), "wb") as fh:
            fh.write(res.stdout)
        manifest.append({"case": name, "opts": opts, "nseq": len(seqs), "dump": False, "input": "mtdna.fa"})
    with open(os.path.join(HERE, "manifest.json"), "w") as fh:
        json.dump(manifest, fh, indent=1)
    print(f"{len(REF_FIXTURES)} reference fixture cases written")


def fasta_read(path):
    sys.path.insert(0, ROOT)
    from tests import fasta
    return fasta.read(path)


def main():
    if not (os.path.exists(REF_BIN) and os.path.exists(HARNESS)):
        sys.exit("build the reference first: make -C oracle ref")
    if "--fullsize" in sys.argv:
        fullsize()
        return
    if "--fixtures" in sys.argv:
        reference_fixtures()
        return
    if "--windows" in sys.argv:
        window_manifests([a for a in sys.argv[1:] if not a.startswith("--")])
        return
    manifest = []
    for name, reads, opts, (base, base_names) in inc_cases():
        bfa = os.path.join("/tmp", name + "_base.fa")
        synth.write_fasta(bfa, base, base_names)
        gfa = subprocess.run([REF_BIN, bfa, "-r", "2"], capture_output=True, check=True).stdout
        os.unlink(bfa)
        with open(os.path.join(HERE, name + ".gfa"), "wb") as fh:
            fh.write(gfa)
        fa = os.path.join(HERE, name + ".fa")
        synth.write_fasta(fa, reads)
        full = ["-i", name + ".gfa"] + opts
        res = subprocess.run([REF_BIN, fa, "-i", os.path.join(HERE, name + ".gfa")] + opts, capture_output=True,
                             check=True)
        with open(os.path.join(HERE, name + ".out"), "wb") as fh:
            fh.write(res.stdout)
        manifest.append({"case": name, "opts": full, "nseq": len(reads), "dump": False})
    for name, reads, opts, dump in cases():
        fa = os.path.join(HERE, name + ".fa")
        synth.write_fasta(fa, reads)
        res = subprocess.run([REF_BIN, fa] + opts, capture_output=True, check=True)
        with open(os.path.join(HERE, name + ".out"), "wb") as fh:
            fh.write(res.stdout)
        if dump:
            subprocess.run([HARNESS, fa] + opts + ["-d", os.path.join(HERE, name + ".dump")],
                           capture_output=True, check=True)
        manifest.append({"case": name, "opts": opts, "nseq": len(reads), "dump": dump})
    with open(os.path.join(HERE, "manifest.json"), "w") as fh:
        json.dump(manifest, fh, indent=1)
    print(f"{len(manifest)} cases written")


if __name__ == "__main__":
    main()
