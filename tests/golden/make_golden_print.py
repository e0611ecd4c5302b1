#!/usr/bin/env python3
"""Golden categorized-read outputs of the reference biobloomcategorizer
(oracle/_ref/biobloomcategorizer, compiled from the reference sources by
``make -C oracle ref``) on the committed fixtures in tests/golden/bbt/:
--fq (single end), --fa (pairs), -d and -d -n (stdout), each with one thread
so that records come in input order.  Every output file of a run is stored in
tests/golden/bbt/print_<case>.txt.gz as "### <file name>" followed by its
contents (stdout as "### stdout").

Usage: python tests/golden/make_golden_print.py
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

CASES = {
    # name: (args, paired)
    "se_fq": (["--fq"], False),
    "se_fa_gz": (["--fa", "-g"], False),
    "pe_fa": (["--fa", "-e"], True),
    "pe_fq_incl": (["--fq", "-e", "-i"], True),
    "se_stdout": (["-d"], False),
    "se_stdout_inv": (["-d", "-n"], False),
}


def inputs(paired):
    if paired:
        return [os.path.join(BBT, "reads_1.fq.gz"), os.path.join(BBT, "reads_2.fq.gz")]
    return [os.path.join(BBT, "reads_se.fa.gz")]


def collect(tmp, stdout):
    parts = []
    for name in sorted(os.listdir(tmp)):
        if name.startswith("out_") and not name.endswith("_summary.tsv"):
            path = os.path.join(tmp, name)
            op = gzip.open if name.endswith(".gz") else open
            with op(path, "rb") as f:
                parts.append(b"### " + name.encode() + b"\n" + f.read())
    parts.append(b"### stdout\n" + stdout)
    return b"".join(parts)


def main():
    if not os.path.exists(CLI):
        raise SystemExit("build oracle/_ref first: make -C oracle ref")
    filters = " ".join(os.path.join(BBT, f"f{i}.bf") for i in range(3))
    for case, (args, paired) in CASES.items():
        with tempfile.TemporaryDirectory() as tmp:
            p = subprocess.run([CLI, "-t", "1", "-p", os.path.join(tmp, "out"), "-f", filters] +
                               args + inputs(paired), capture_output=True)
            if p.returncode:
                sys.stderr.write(p.stderr.decode(errors="replace"))
                raise SystemExit(f"failed: {case}")
            with gzip.open(os.path.join(BBT, f"print_{case}.txt.gz"), "wb", compresslevel=9) as f:
                f.write(collect(tmp, p.stdout))
    print("written", ", ".join(f"print_{c}.txt.gz" for c in CASES))


if __name__ == "__main__":
    main()
