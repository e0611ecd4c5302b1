#!/usr/bin/env python3
"""Golden files for DUST masking (-D, -T, -W), written by the reference's own
code: oracle/_ref/ref_harness (compiled from the reference sources by
``make -C oracle ref``; BBT_DUST="T,W" turns on opt::dust) and the reference
biobloomcategorizer CLI (through make_golden_print.py's MODE_CASES).

Inputs (written here, seeded): tests/golden/bbt/reads_dust.fa.gz and
reads_dust_2.fa.gz, reads of the committed fixtures (which the fixture
filters match) with low-complexity stretches spliced in: homopolymers,
di-/tri-/tetranucleotide repeats, two-letter random runs, near-homopolymers,
in either case, with N runs; long reads up to a few kb; and edge cases (empty,
all-N, a 2 kb poly-A, a 2 kb (AC)n).

Outputs:
  expected_dust_<T>_<W>.tsv         the masked intervals of every read
                                    (Common/sdust.c via ref_harness dust)
  expected_hits_<case>.tsv          per-read hits and summary with masking
  expected_scores_<case>.tsv        evalScore with masking

Usage: python tests/golden/make_golden_dust.py
"""
import gzip
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
BBT = os.path.join(HERE, "bbt")
HARNESS = os.path.join(ROOT, "oracle", "_ref", "ref_harness")
READS = os.path.join(BBT, "reads_dust.fa.gz")
READS2 = os.path.join(BBT, "reads_dust_2.fa.gz")

DUST_PARAMS = {"T20_W64": (20, 64), "T30_W32": (30, 32), "T10_W16": (10, 16)}
# name: (method, -s, streak, paired)
HIT_CASES = {
    "dust_se_s0.15_r3": ("simple", "0.15", "3", False),
    "dust_se_s40": ("simple", "40", "3", False),
    "dust_harmonic_s0.15_r3": ("harmonic", "0.15", "3", False),
    "dust_binomial_s100_r3": ("binomial", "100", "3", False),
    "dust_pe_s0.15_r3": ("simple", "0.15", "3", True),
}
# name: (method, streak)
SCORE_CASES = {
    "dust_simple_r3": ("simple", 3),
    "dust_length_r3": ("length", 3),
    "dust_binomial_r3": ("binomial", 3),
}


def _fastx_seqs(path):
    with gzip.open(path, "rt") as f:
        lines = f.read().split("\n")
    if lines[0].startswith("@"):
        return [lines[i + 1] for i in range(0, len(lines) - 3, 4)]
    out = []
    for line in lines:
        if line.startswith(">"):
            out.append("")
        elif out:
            out[-1] += line.strip()
    return out


def _low_complexity(rng):
    n = int(rng.integers(4, 90))
    kind = int(rng.integers(0, 7))
    if kind == 0:
        s = "ACGT"[int(rng.integers(4))] * n
    elif kind == 1:
        s = ["AC", "AT", "GT", "CG", "AG"][int(rng.integers(5))] * n
    elif kind == 2:
        s = ["ACG", "AAT", "CTG", "GGA"][int(rng.integers(4))] * n
    elif kind == 3:
        s = ["AACG", "GATA", "TTTC"][int(rng.integers(3))] * n
    elif kind == 4:
        s = "".join(rng.choice(list("AT"), n))
    elif kind == 5:
        s = "".join("A" if rng.random() < 0.9 else "G" for _ in range(n))
    else:
        s = "".join(rng.choice(list("CCCCT"), n))
    s = s[:n]
    return s.lower() if rng.random() < 0.2 else s


def make_reads(seed, n):
    rng = np.random.default_rng(seed)
    pool = _fastx_seqs(os.path.join(BBT, "reads_se.fa.gz"))
    pool += _fastx_seqs(os.path.join(BBT, "reads_1.fq.gz"))
    pool = [p for p in pool if len(p) >= 60]
    reads = []
    for i in range(n):
        if i % 40 == 39:  # long read
            parts = []
            for _ in range(int(rng.integers(8, 25))):
                parts.append(pool[int(rng.integers(len(pool)))])
                if rng.random() < 0.5:
                    parts.append(_low_complexity(rng))
                if rng.random() < 0.1:
                    parts.append("N" * int(rng.integers(1, 30)))
            reads.append("".join(parts))
            continue
        s = pool[int(rng.integers(len(pool)))]
        for _ in range(int(rng.integers(0, 4))):
            at = int(rng.integers(0, len(s) + 1))
            lc = _low_complexity(rng)
            s = s[:at] + lc + s[at + (len(lc) if rng.random() < 0.5 else 0):]
        if rng.random() < 0.1:
            at = int(rng.integers(0, len(s) + 1))
            s = s[:at] + "N" * int(rng.integers(1, 8)) + s[at:]
        reads.append(s)
    reads += ["", "N" * 40, "A" * 2000, "AC" * 1000, "ACGT" * 6, "A" * 30 + "N" + "A" * 30]
    return reads


def write_fasta(path, prefix, reads):
    with gzip.GzipFile(path, "wb", compresslevel=9, mtime=0) as f:
        for i, s in enumerate(reads):
            f.write(f">{prefix}{i}\n{s}\n".encode())


def run(args, env=None):
    p = subprocess.run(args, capture_output=True, env=env)
    if p.returncode:
        sys.stderr.write(p.stderr.decode(errors="replace"))
        raise SystemExit(f"failed: {args}")
    return p.stdout


def main():
    if not os.path.exists(HARNESS):
        raise SystemExit("build oracle/_ref first: make -C oracle ref")
    write_fasta(READS, "d", make_reads(7, 400))
    write_fasta(READS2, "d", make_reads(8, 400))
    for name, (t, w) in DUST_PARAMS.items():
        out = run([HARNESS, "dust", str(t), str(w), READS])
        with open(os.path.join(BBT, f"expected_dust_{name}.tsv"), "wb") as f:
            f.write(out)
    filters = ",".join(os.path.join(BBT, f"f{i}.bf") for i in range(3))
    env = dict(os.environ, BBT_DUST="20,64")
    for name, (method, score, streak, paired) in HIT_CASES.items():
        e = dict(env, BBT_SCORING=method) if method != "simple" else env
        out = run([HARNESS, "hits", score, streak, filters, READS] + ([READS2] if paired else []),
                  env=e)
        with open(os.path.join(BBT, f"expected_hits_{name}.tsv"), "wb") as f:
            f.write(out)
    for name, (method, streak) in SCORE_CASES.items():
        out = run([HARNESS, "scores", method, str(streak), filters, READS], env=env)
        with open(os.path.join(BBT, f"expected_scores_{name}.tsv"), "wb") as f:
            f.write(out)
    print("written", len(DUST_PARAMS) + len(HIT_CASES) + len(SCORE_CASES), "files")


if __name__ == "__main__":
    main()
