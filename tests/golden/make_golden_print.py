#!/usr/bin/env python3
"""Golden categorized-read outputs of the reference biobloomcategorizer
(oracle/_ref/biobloomcategorizer, compiled from the reference sources by
``make -C oracle ref``) on the committed fixtures in tests/golden/bbt/:
--fq (single end), --fa (pairs), -d and -d -n (stdout), each with one thread
so that records come in input order.  Every output file of a run is stored in
tests/golden/bbt/print_<case>.txt.gz as "### <file name>" followed by its
contents (stdout as "### stdout").

MODE_CASES cover the filtering modes (-c ordered, -b best hit, -w with
scores), single-file paired input (reads_smart.fq.gz, written here from the
paired fixtures with "/1" and "/2" names, mates out of order and orphans) and
file lists (-l, written into the run's directory) and DUST masking (-D, -T,
-W, on the reads of make_golden_dust.py, which runs first); their golden files
also hold "<prefix>_summary.tsv".

Usage: python tests/golden/make_golden_print.py [--all]
(--all also rewrites the CASES files, which the MODE_CASES run leaves as they are)
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


# name: (args, input kind)
MODE_CASES = {
    "ord_se": (["-c"], "se"),
    "ord_se_fa": (["-c", "--fa"], "se"),
    "ord_pe": (["-c", "-e"], "pe"),
    "ord_pe_incl_fq": (["-c", "-e", "-i", "--fq"], "pe"),
    "best_se_fa": (["-b", "--fa"], "se"),
    "best_se_fq": (["-b", "--fq"], "se"),
    "best_pe_fa": (["-b", "-e", "--fa"], "pe"),
    "best_pe_incl_fq": (["-b", "-e", "-i", "--fq"], "pe"),
    "best_se_stdout": (["-b", "-d"], "se"),
    "best_harmonic_se_fa": (["-b", "-S", "harmonic", "--fa"], "se"),
    "best_binomial_se_fq": (["-b", "-S", "binomial", "--fq"], "se"),
    "scores_se_fa": (["-w", "--fa"], "se"),
    "scores_pe_fq": (["-w", "-e", "--fq"], "pe"),
    "scores_length_se_fq": (["-w", "-s", "40", "--fq"], "se"),
    "scores_harmonic_se_fa": (["-w", "-S", "harmonic", "--fa"], "se"),
    "scores_binomial_se_fa": (["-w", "-S", "binomial", "--fa"], "se"),
    "smart_summary": (["-e"], "smart"),
    "smart_fq": (["-e", "--fq"], "smart"),
    "smart_incl_best_fa": (["-e", "-i", "-b", "--fa"], "smart"),
    "list_se": ([], "list_se"),
    "list_se_fa": (["--fa"], "list_se"),
    "list_pe": (["-e"], "list_pe"),
    "dust_se_fa": (["-D", "--fa"], "dust_se"),
    "dust_t30_w32_se": (["-D", "-T", "30", "-W", "32"], "dust_se"),
    "dust_pe_fq": (["-D", "-e", "--fq"], "dust_pe"),
    "dust_best_se_fa": (["-D", "-b", "--fa"], "dust_se"),
    "dust_ord_pe_incl": (["-D", "-c", "-e", "-i"], "dust_pe"),
    "dust_scores_length_se_fq": (["-D", "-w", "-s", "30", "--fq"], "dust_se"),
}
# Not a case: -e -d with -l.  That path prints kseq records
# (BioBloomClassifier.h:249-287) and inserts comment.s into std::cout, a null
# pointer for records without a comment, which puts std::cout in a failed
# state and silently drops the rest of stdout.

SMART = os.path.join(BBT, "reads_smart.fq.gz")


def inputs(paired):
    if paired:
        return [os.path.join(BBT, "reads_1.fq.gz"), os.path.join(BBT, "reads_2.fq.gz")]
    return [os.path.join(BBT, "reads_se.fa.gz")]


def mode_inputs(kind, tmp):
    """Input arguments of a MODE_CASES kind; list files are written into tmp."""
    if kind == "se":
        return inputs(False)
    if kind == "pe":
        return inputs(True)
    if kind == "smart":
        return [SMART]
    if kind == "dust_se":
        return [os.path.join(BBT, "reads_dust.fa.gz")]
    if kind == "dust_pe":
        return [os.path.join(BBT, "reads_dust.fa.gz"), os.path.join(BBT, "reads_dust_2.fa.gz")]
    lst = os.path.join(tmp, "list.txt")
    se = os.path.join(BBT, "reads_se.fa.gz")
    r1, r2 = inputs(True)
    with open(lst, "w") as f:
        if kind == "list_se":
            f.write(f"{se}\n{r1} {r2}\n")
        else:
            f.write(f"{r1} {r2}\n{r2}\t{r1}\n")
    return ["-l", lst]


def read_fastq(path):
    with gzip.open(path, "rt") as f:
        lines = f.read().split("\n")
    return [(lines[i][1:], lines[i + 1], lines[i + 3]) for i in range(0, len(lines) - 3, 4)]


def write_smart_fixture():
    """reads_smart.fq.gz: the pairs of reads_1/reads_2 as one file with names
    "<name>/1" and "<name>/2".  Most pairs are adjacent; every 7th pair comes
    mate 2 first, every 5th pair has its mate 2 one pair later, every 11th
    pair loses mate 2 (an orphan, never counted), and two records named
    "odd" (no 1/2 suffix) pair with each other."""
    m1 = read_fastq(os.path.join(BBT, "reads_1.fq.gz"))
    m2 = read_fastq(os.path.join(BBT, "reads_2.fq.gz"))
    recs, held = [], []
    for i, (a, b) in enumerate(zip(m1, m2)):
        ra = (a[0] + "/1", a[1], a[2])
        rb = (b[0] + "/2", b[1], b[2])
        if i % 11 == 3:
            recs.append(ra)
        elif i % 7 == 2:
            recs += [rb, ra]
        elif i % 5 == 1:
            recs.append(ra)
            held.append(rb)
            continue
        else:
            recs += [ra, rb]
        recs += held
        held = []
        if i == 10:
            recs.append(("odd", m1[0][1], m1[0][2]))
        if i == 40:
            recs.append(("odd", m2[0][1], m2[0][2]))
    recs += held
    with gzip.GzipFile(SMART, "wb", compresslevel=9, mtime=0) as f:
        for name, seq, qual in recs:
            f.write(f"@{name}\n{seq}\n+\n{qual}\n".encode())


def collect(tmp, stdout, summary=False):
    parts = []
    for name in sorted(os.listdir(tmp)):
        if name.startswith("out_") and (summary or not name.endswith("_summary.tsv")):
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
    for case, (args, paired) in (CASES.items() if "--all" in sys.argv else ()):
        with tempfile.TemporaryDirectory() as tmp:
            p = subprocess.run([CLI, "-t", "1", "-p", os.path.join(tmp, "out"), "-f", filters] +
                               args + inputs(paired), capture_output=True)
            if p.returncode:
                sys.stderr.write(p.stderr.decode(errors="replace"))
                raise SystemExit(f"failed: {case}")
            with gzip.open(os.path.join(BBT, f"print_{case}.txt.gz"), "wb", compresslevel=9) as f:
                f.write(collect(tmp, p.stdout))
    write_smart_fixture()
    for case, (args, kind) in MODE_CASES.items():
        with tempfile.TemporaryDirectory() as tmp:
            p = subprocess.run([CLI, "-t", "1", "-p", os.path.join(tmp, "out"), "-f", filters] +
                               args + mode_inputs(kind, tmp), capture_output=True)
            if p.returncode:
                sys.stderr.write(p.stderr.decode(errors="replace"))
                raise SystemExit(f"failed: {case}")
            with gzip.GzipFile(os.path.join(BBT, f"print_{case}.txt.gz"), "wb", compresslevel=9,
                               mtime=0) as f:
                f.write(collect(tmp, p.stdout, summary=True))
    print("written", ", ".join(f"print_{c}.txt.gz" for c in list(CASES) + list(MODE_CASES)))


if __name__ == "__main__":
    main()
