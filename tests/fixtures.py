"""Readers for the committed golden fixtures in tests/golden/bbt/."""
import gzip
import os

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "bbt")


def golden(name):
    return os.path.join(GOLDEN, name)


def read_fastx(path):
    """Minimal FASTA/FASTQ reader for the fixtures: [(name, seq bytes)]."""
    op = gzip.open if path.endswith(".gz") else open
    with op(path, "rb") as f:
        lines = f.read().split(b"\n")
    recs = []
    i = 0
    while i < len(lines):
        line = lines[i]
        if line.startswith(b">"):
            name = line[1:].split()[0].decode() if line[1:].split() else ""
            seq = []
            i += 1
            while i < len(lines) and not lines[i].startswith(b">"):
                seq.append(lines[i].strip())
                i += 1
            recs.append((name, b"".join(seq)))
        elif line.startswith(b"@"):
            name = line[1:].split()[0].decode()
            recs.append((name, lines[i + 1].strip()))
            i += 4
        else:
            i += 1
    return recs


def expected_hits(name):
    """Per-read hit sets and the summary text written by the reference harness."""
    rows = []
    summary = []
    in_summary = False
    with open(golden(f"expected_hits_{name}.tsv")) as f:
        for line in f:
            if line.startswith("#SUMMARY"):
                in_summary = True
                continue
            if in_summary:
                summary.append(line)
                continue
            rname, hits = line.rstrip("\n").split("\t")
            if "|" in hits:
                a, b = hits.split("|")
                rows.append((rname, _ids(a), _ids(b)))
            else:
                rows.append((rname, _ids(hits)))
    return rows, "".join(summary)


def _ids(s):
    return set(int(x) for x in s.split(",") if x != "")


def filter_ids():
    return ["f0", "f1", "f2"]


def filter_paths():
    return [golden(f"f{i}.bf") for i in range(3)]
