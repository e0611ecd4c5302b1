#!/usr/bin/env python3
"""Golden summary of the reference biobloomcategorizer
(oracle/_ref/biobloomcategorizer, compiled from the reference sources by
``make -C oracle ref``) on input that ends in a truncated FASTQ record.

truncated.fq holds the first 200 records of reads_1.fq.gz and then a record
whose quality line is shorter than its sequence at the end of the file:
kseq_read returns -2 there, which the reference treats as the end of that
file (BioBloomClassifier.cpp:64,87-88) before it goes on to the next input.
after.fq holds the next 50 records.  The reference's summary of
`-f "f0.bf f1.bf f2.bf" truncated.fq after.fq` is stored as
expected_summary_truncated.tsv.

Usage: python tests/golden/make_golden_failures.py
"""
import gzip
import os
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
BBT = os.path.join(HERE, "bbt")
CLI = os.path.join(ROOT, "oracle", "_ref", "biobloomcategorizer")


def records(path):
    with gzip.open(path, "rt") as f:
        lines = f.read().split("\n")
    return ["\n".join(lines[i:i + 4]) + "\n" for i in range(0, len(lines) - 3, 4)]


def main():
    if not os.path.exists(CLI):
        sys.exit("build the reference first: make -C oracle ref")
    recs = records(os.path.join(BBT, "reads_1.fq.gz"))
    seq = recs[200].split("\n")[1]
    trunc = "".join(recs[:200]) + f"@truncated\n{seq}\n+\n{'I' * (len(seq) // 3)}\n"
    with open(os.path.join(BBT, "truncated.fq"), "w") as f:
        f.write(trunc)
    with open(os.path.join(BBT, "after.fq"), "w") as f:
        f.write("".join(recs[201:251]))
    filters = " ".join(os.path.join(BBT, f"f{i}.bf") for i in range(3))
    with tempfile.TemporaryDirectory() as d:
        prefix = os.path.join(d, "t")
        subprocess.run([CLI, "-t", "1", "-p", prefix, "-f", filters,
                        os.path.join(BBT, "truncated.fq"), os.path.join(BBT, "after.fq")],
                       check=True, capture_output=True)
        with open(prefix + "_summary.tsv") as f:
            summary = f.read()
    with open(os.path.join(BBT, "expected_summary_truncated.tsv"), "w") as f:
        f.write(summary)
    print(summary)


if __name__ == "__main__":
    main()
