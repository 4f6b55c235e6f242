"""Small readers for the test fixtures (FASTA and per-call dumps)."""
import os

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def golden_input(case):
    """Input FASTA of a manifest case: its own <case>.fa, or the shared file it
    names in "input" (the reference's data/mtDNA.fasta serves four cases)."""
    return os.path.join(GOLD, case.get("input", case["case"] + ".fa"))


def read_records(path):
    """[(name, comment, seq)] like kseq: name up to the first blank."""
    recs = []
    with open(path, "rb") as fh:
        for line in fh:
            line = line.rstrip(b"\r\n")
            if line.startswith(b">"):
                hdr = line[1:].decode()
                parts = hdr.split(None, 1)
                name = parts[0] if parts else ""
                comment = parts[1] if len(parts) > 1 else ""
                recs.append([name, comment, b""])
            elif recs:
                recs[-1][2] += line
    return [tuple(r) for r in recs]


def read(path):
    recs = read_records(path)
    return [r[0] for r in recs], [r[2] for r in recs]


def headers(path):
    """The header text minipoa prints for each read: 'name comment'."""
    return [f"{n} {c}" for n, c, _ in read_records(path)]


def read_dump(path):
    """Records of oracle/ref_harness: (read index, score, [(from, base, aligned)])."""
    out = []
    with open(path) as fh:
        lines = fh.read().split("\n")
    i = 0
    while i < len(lines):
        if lines[i].startswith("A "):
            _, ri, sc, ln = lines[i].split()
            path = []
            if int(ln):
                for tok in lines[i + 1].split():
                    a, b, c = tok.split(",")
                    path.append((int(a), int(b), int(c)))
            out.append((int(ri), int(sc), path))
            i += 2
        else:
            i += 1
    return out
