#!/usr/bin/env python3
"""Golden miBF files written by the reference's own miBF maker
(oracle/_ref/biobloommimaker: BioBloomMaker/BioBloomMIMaker.cpp and
MIBFGen.hpp compiled from the reference sources by ``make -C oracle ref``,
over the shim's restated MIBFConstructSupport / MIBloomFilter, the
btl_bloomfilter classes absent from the reference tree).

The reference's driver decides what the restatement cannot: IDs by file (-F)
or by FASTA name in file order (a repeated name takes the later ID for all its
sequences), the expected frame count (sum of len - k + 1 over records, a short
record included, in size_t arithmetic), k-mer mode (-k -g) or spaced seeds
(-S), and the _ids.txt layout.  Inputs: three small FASTA files written here
(several contigs, a repeated name, an N run, a record shorter than k).  Each
case's <case>.bf, .sdsl and _ids.txt go to tests/golden/mimaker/ (gzipped).

Usage: python tests/golden/make_golden_mimaker.py
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
OUT = os.path.join(HERE, "mimaker")
MAKER = os.path.join(ROOT, "oracle", "_ref", "biobloommimaker")
SEEDS = ["1111110111101101111111111", "1111111111011011110111111",
         "1111111111101111011111100"]
CASES = {
    # name: (arguments)
    "file_kmer": ["-F", "-k", "25", "-g", "3"],
    "file_seeds": ["-F", "-S", " ".join(SEEDS)],
    "name_kmer": ["-k", "25", "-g", "3"],
    "name_seeds": ["-S", " ".join(SEEDS)],
}


def inputs():
    """{file name: [(record name, sequence)]} (seeded)."""
    rng = np.random.default_rng(5)
    bases = np.frombuffer(b"ACGT", dtype=np.uint8)

    def rs(n):
        return rng.choice(bases, n).tobytes()
    return {
        "a.fa": [("c1", rs(6000)), ("c2", rs(3000))],
        "b.fa": [("d1", rs(5000) + b"N" * 40 + rs(2000)), ("c1", rs(1500)), ("tiny", b"ACGTACGT")],
        "c.fa": [("e1", rs(7000))],
    }


def write_inputs(d):
    for fn, recs in inputs().items():
        with open(os.path.join(d, fn), "wb") as f:
            for n, s in recs:
                f.write(b">" + n.encode() + b"\n" + s + b"\n")


def main():
    if not os.path.exists(MAKER):
        sys.exit("build the reference first: make -C oracle ref")
    os.makedirs(OUT, exist_ok=True)
    with tempfile.TemporaryDirectory() as d:
        write_inputs(d)
        for case, args in CASES.items():
            subprocess.run([MAKER, "-t", "1", "-p", case] + args + sorted(inputs()), cwd=d,
                           check=True, capture_output=True)
            for ext in (".bf", ".sdsl", "_ids.txt"):
                with open(os.path.join(d, case + ext), "rb") as src, \
                        gzip.open(os.path.join(OUT, case + ext + ".gz"), "wb") as dst:
                    shutil.copyfileobj(src, dst)
    print("wrote", sorted(os.listdir(OUT)))


if __name__ == "__main__":
    main()
