#!/usr/bin/env python3
"""Generate the golden fixtures in tests/golden/bbt/ from the reference's own
code, compiled from the reference sources into oracle/_ref (run
``make -C oracle ref`` first; it needs the reference source tree).

What is produced (all small, committed):
  f0/f1/f2.{bf,txt}   filters built by the reference's biobloommaker
                      (BioBloomMaker.cpp, BloomFilterGenerator.cpp) from three
                      seeded 20 kbp genomes, k=25, FPR 0.075 (hash count auto).
  len.{bf,txt}        k=4, h=2, 8000-bit filter loaded from "NNNNNAAAAA" as
                      Tests/SeqEvalTests.cpp:9-23 does (built with the oracle).
  reads_se.fa.gz      single-end reads: from each genome with 1% substitutions,
                      random reads, N runs, lowercase, IUPAC codes, reads shorter
                      than k, an empty record.
  reads_1.fq.gz, reads_2.fq.gz   read pairs of the same kinds.
  expected_*.tsv      per-read hit lists and summary text from
                      oracle/_ref/ref_harness (the reference's SeqEval::evalRead
                      and ResultsManager) and summary.tsv files written by the
                      reference's biobloomcategorizer CLI.

Usage: python tests/golden/make_golden.py
"""
import gzip
import os
import shutil
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
REF_BIN = os.path.join(ROOT, "oracle", "_ref")
OUT = os.path.join(HERE, "bbt")
BASES = np.frombuffer(b"ACGT", dtype=np.uint8)


def genome(rng, n, gc):
    u = rng.random(n)
    out = np.where(u < gc / 2, ord("C"), np.where(u < gc, ord("G"),
                   np.where(u < gc + (1 - gc) / 2, ord("A"), ord("T"))))
    return out.astype(np.uint8)


def revcomp(s):
    t = bytes.maketrans(b"ACGTacgtN", b"TGCAtgcaN")
    return s.translate(t)[::-1]


def mutate(rng, s, sub=0.0, nrate=0.0, lower=0.0, iupac=0.0):
    a = np.frombuffer(s, dtype=np.uint8).copy()
    n = len(a)
    m = rng.random(n) < sub
    a[m] = BASES[rng.integers(0, 4, m.sum())]
    m = rng.random(n) < nrate
    a[m] = ord("N")
    m = rng.random(n) < iupac
    a[m] = np.frombuffer(b"RYKMSW", dtype=np.uint8)[rng.integers(0, 6, m.sum())]
    m = (rng.random(n) < lower) & (a != ord("N"))
    a[m] |= 0x20  # ASCII lower case
    return a.tobytes()


def sample_read(rng, genomes, kind, L):
    """kind: genome index, or -1 for random."""
    if kind < 0:
        return BASES[rng.integers(0, 4, L)].tobytes(), None
    g = genomes[kind]
    start = int(rng.integers(0, len(g) - L))
    s = g[start:start + L].tobytes()
    if rng.random() < 0.5:
        s = revcomp(s)
    return s, start


def make_reads(rng, genomes, n, paired):
    recs = []
    for i in range(n):
        kind = int(rng.integers(-1, len(genomes)))
        style = i % 10
        L = 150
        if style == 7:
            L = int(rng.integers(1, 25))        # shorter than k (some < k-1)
        elif style == 8:
            L = int(rng.integers(25, 60))
        if paired:
            frag = int(rng.integers(300, 500))
            if kind >= 0:
                g = genomes[kind]
                st = int(rng.integers(0, len(g) - frag))
                f = g[st:st + frag].tobytes()
                if rng.random() < 0.5:
                    f = revcomp(f)
                m1, m2 = f[:L], revcomp(f)[:L]
            else:
                m1 = BASES[rng.integers(0, 4, L)].tobytes()
                m2 = BASES[rng.integers(0, 4, L)].tobytes()
            mates = [m1, m2]
        else:
            mates = [sample_read(rng, genomes, kind, L)[0]]
        out = []
        for m in mates:
            if style == 1:
                m = mutate(rng, m, sub=0.01)
            elif style == 2:
                m = mutate(rng, m, sub=0.01, nrate=0.02)
            elif style == 3:
                m = mutate(rng, m, lower=0.3)
            elif style == 4:
                m = mutate(rng, m, iupac=0.01, sub=0.005)
            elif style == 5:
                b = bytearray(m)
                q = int(rng.integers(0, max(1, len(b))))
                run = int(rng.integers(1, 40))
                b[q:q + run] = b"N" * len(b[q:q + run])
                m = bytes(b)
            elif style == 6:
                m = mutate(rng, m, sub=0.05)
            out.append(m)
        recs.append(out)
    # an empty record and an all-N record
    recs.append([b"" for _ in range(2 if paired else 1)])
    recs.append([b"N" * 150 for _ in range(2 if paired else 1)])
    return recs


def write_fasta_gz(path, names, seqs):
    with gzip.open(path, "wb", compresslevel=9) as f:
        for n, s in zip(names, seqs):
            f.write(b">" + n.encode() + b"\n" + s + b"\n")


def write_fastq_gz(path, names, seqs):
    with gzip.open(path, "wb", compresslevel=9) as f:
        for n, s in zip(names, seqs):
            f.write(b"@" + n.encode() + b"\n" + s + b"\n+\n" + b"I" * len(s) + b"\n")


def run(cmd, cwd):
    p = subprocess.run(cmd, cwd=cwd, capture_output=True, text=True)
    if p.returncode:
        sys.stderr.write(p.stderr)
        raise SystemExit(f"failed: {' '.join(cmd)}")
    return p.stdout


def main():
    for b in ("biobloommaker", "biobloomcategorizer", "ref_harness"):
        if not os.path.exists(os.path.join(REF_BIN, b)):
            raise SystemExit("build oracle/_ref first: make -C oracle ref")
    sys.path.insert(0, ROOT)
    from tests import oracle_lib

    os.makedirs(OUT, exist_ok=True)
    rng = np.random.default_rng(20240611)
    genomes = [genome(rng, 20000, gc) for gc in (0.5, 0.41, 0.6)]
    # make genome 2 share a 2 kb block with genome 0 so multiMatch occurs
    genomes[2][5000:7000] = genomes[0][1000:3000]

    with tempfile.TemporaryDirectory() as tmp:
        for i, g in enumerate(genomes):
            fa = os.path.join(tmp, f"g{i}.fa")
            with open(fa, "wb") as f:
                f.write(f">g{i}\n".encode() + g.tobytes() + b"\n")
            run([os.path.join(REF_BIN, "biobloommaker"), "-p", f"f{i}", "-k", "25",
                 "-f", "0.075", fa], cwd=tmp)
            for ext in ("bf", "txt"):
                shutil.copy(os.path.join(tmp, f"f{i}.{ext}"), os.path.join(OUT, f"f{i}.{ext}"))

        se = make_reads(rng, genomes, 600, paired=False)
        se_names = [f"se{i}" for i in range(len(se))]
        write_fasta_gz(os.path.join(OUT, "reads_se.fa.gz"), se_names, [r[0] for r in se])
        pe = make_reads(rng, genomes, 400, paired=True)
        pe_names = [f"pe{i}" for i in range(len(pe))]
        write_fastq_gz(os.path.join(OUT, "reads_1.fq.gz"), pe_names, [r[0] for r in pe])
        write_fastq_gz(os.path.join(OUT, "reads_2.fq.gz"), pe_names, [r[1] for r in pe])

        filters = ",".join(os.path.join(OUT, f"f{i}.bf") for i in range(3))
        harness = os.path.join(REF_BIN, "ref_harness")
        cases = {
            "se_s0.15_r3": ["hits", "0.15", "3", filters, os.path.join(OUT, "reads_se.fa.gz")],
            "se_s0.5_r1": ["hits", "0.5", "1", filters, os.path.join(OUT, "reads_se.fa.gz")],
            "se_s0.05_r0": ["hits", "0.05", "0", filters, os.path.join(OUT, "reads_se.fa.gz")],
            "se_s40": ["hits", "40", "3", filters, os.path.join(OUT, "reads_se.fa.gz")],
            "pe_s0.15_r3": ["hits", "0.15", "3", filters, os.path.join(OUT, "reads_1.fq.gz"),
                            os.path.join(OUT, "reads_2.fq.gz")],
        }
        for name, args in cases.items():
            out = run([harness] + args, cwd=tmp)
            with open(os.path.join(OUT, f"expected_hits_{name}.tsv"), "w") as f:
                f.write(out)

        # summary.tsv written by the reference CLI itself
        cat = os.path.join(REF_BIN, "biobloomcategorizer")
        fl = " ".join(os.path.join(OUT, f"f{i}.bf") for i in range(3))
        clis = {
            "se": ["-p", "se", "-f", fl, os.path.join(OUT, "reads_se.fa.gz")],
            "pe": ["-p", "pe", "-e", "-f", fl, os.path.join(OUT, "reads_1.fq.gz"),
                   os.path.join(OUT, "reads_2.fq.gz")],
            "pe_incl": ["-p", "pe_incl", "-e", "-i", "-f", fl, os.path.join(OUT, "reads_1.fq.gz"),
                        os.path.join(OUT, "reads_2.fq.gz")],
            "se_s40": ["-p", "se_s40", "-s", "40", "-f", fl, os.path.join(OUT, "reads_se.fa.gz")],
        }
        for name, args in clis.items():
            run([cat] + args, cwd=tmp)
            shutil.copy(os.path.join(tmp, f"{name}_summary.tsv"),
                        os.path.join(OUT, f"expected_summary_{name}.tsv"))

    # Tests/SeqEvalTests.cpp:9-23 filter: k=4, h=2, 8000 bits, from NNNNNAAAAA
    bf = oracle_lib.Filter.create(8000, 2, 4)
    bf.insert_sequence(b"NNNNNAAAAA")
    bf.store(os.path.join(OUT, "len.bf"))
    oracle_lib.write_info(os.path.join(OUT, "len.txt"), "len", 4, 0.0078125, 2, 7,
                          "NNNNNAAAAA", 8000, 1, 0.0001, 0, 0.0001)
    print("golden fixtures written to", OUT)


if __name__ == "__main__":
    main()
