#!/usr/bin/env python3
"""Golden SeqEval::evalScore values (Common/SeqEval.h:534-560) of the
reference's own code, driven by oracle/_ref/ref_harness (compiled from the
reference sources by ``make -C oracle ref``) on the committed fixtures:
every read of tests/golden/bbt/reads_se.fa.gz against filters f0, f1, f2,
for each scoring method.  One line per read, "<name>\\t<bits>,<bits>,<bits>"
with each score as the 16 hex digits of its IEEE double.

BINOMIAL goes through the binomial tail of oracle/shim/boost (Boost is not
installed here; the shim restates boost's cdf(complement(...)) as the sum of
the probability masses above the count).

Usage: python tests/golden/make_golden_scores.py
"""
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
BBT = os.path.join(HERE, "bbt")
HARNESS = os.path.join(ROOT, "oracle", "_ref", "ref_harness")

# name: (method, streak)
CASES = {
    "simple_r3": ("simple", 3),
    "simple_r1": ("simple", 1),
    "length_r3": ("length", 3),
    "harmonic_r3": ("harmonic", 3),
    "binomial_r3": ("binomial", 3),
    "binomial_r2": ("binomial", 2),
}


def main():
    if not os.path.exists(HARNESS):
        raise SystemExit("build oracle/_ref first: make -C oracle ref")
    filters = ",".join(os.path.join(BBT, f"f{i}.bf") for i in range(3))
    for case, (method, streak) in CASES.items():
        out = subprocess.run([HARNESS, "scores", method, str(streak), filters,
                              os.path.join(BBT, "reads_se.fa.gz")],
                             check=True, capture_output=True).stdout
        with open(os.path.join(BBT, f"expected_scores_{case}.tsv"), "wb") as f:
            f.write(out)
    print("written", ", ".join(f"expected_scores_{c}.tsv" for c in CASES))


if __name__ == "__main__":
    main()
