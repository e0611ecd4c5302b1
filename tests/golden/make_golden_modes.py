#!/usr/bin/env python3
"""Golden per-read hits and summary.tsv for the HARMONIC and BINOMIAL scoring
methods (-S harmonic / -S binomial), written by the reference's own
SeqEval::evalRead + ResultsManager (oracle/_ref/ref_harness, BBT_SCORING
selects the method) and by the reference biobloomcategorizer CLI, on the
committed fixtures in tests/golden/bbt/.

Usage: python tests/golden/make_golden_modes.py
"""
import os
import shutil
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
BBT = os.path.join(HERE, "bbt")
REF = os.path.join(ROOT, "oracle", "_ref")

# name: (method, -s value, streak, paired)
CASES = {
    "harmonic_s0.15_r3": ("harmonic", "0.15", "3", False),
    "harmonic_s0.4_r1": ("harmonic", "0.4", "1", False),
    "harmonic_pe_s0.15_r3": ("harmonic", "0.15", "3", True),
    "binomial_s100_r3": ("binomial", "100", "3", False),
    "binomial_s30_r2": ("binomial", "30", "2", False),
    "binomial_pe_s100_r3": ("binomial", "100", "3", True),
}


def reads(paired):
    if paired:
        return [os.path.join(BBT, "reads_1.fq.gz"), os.path.join(BBT, "reads_2.fq.gz")]
    return [os.path.join(BBT, "reads_se.fa.gz")]


def main():
    filters = ",".join(os.path.join(BBT, f"f{i}.bf") for i in range(3))
    for name, (method, score, streak, paired) in CASES.items():
        env = dict(os.environ, BBT_SCORING=method)
        p = subprocess.run([os.path.join(REF, "ref_harness"), "hits", score, streak, filters] +
                           reads(paired), capture_output=True, text=True, env=env)
        if p.returncode:
            sys.stderr.write(p.stderr)
            raise SystemExit(f"failed: {name}")
        with open(os.path.join(BBT, f"expected_hits_{name}.tsv"), "w") as f:
            f.write(p.stdout)
        with tempfile.TemporaryDirectory() as tmp:
            args = ["-p", os.path.join(tmp, "o"), "-S", method, "-s", score, "-r", streak,
                    "-f", filters.replace(",", " ")]
            if paired:
                args.append("-e")
            c = subprocess.run([os.path.join(REF, "biobloomcategorizer")] + args + reads(paired),
                               capture_output=True, text=True)
            if c.returncode:
                sys.stderr.write(c.stderr)
                raise SystemExit(f"CLI failed: {name}")
            shutil.copy(os.path.join(tmp, "o_summary.tsv"),
                        os.path.join(BBT, f"expected_summary_{name}.tsv"))
    print("written", len(CASES), "cases")


if __name__ == "__main__":
    main()
