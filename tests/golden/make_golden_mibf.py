#!/usr/bin/env python3
"""Generate the multi-index Bloom filter (miBF) golden fixtures in
tests/golden/mibf/ from the reference's own MI categorizer
(BioBloomCategorizer/BioBloomMICategorizer.cpp + MIBFClassifier.hpp +
ResultsManager.hpp), compiled from the reference sources into
oracle/_ref/biobloommicategorizer (``make -C oracle ref``).  The miBF data
structure classes it includes come from the btl_bloomfilter submodule, which
the reference tree does not hold; they are compiled from the restatement in
oracle/mibf_oracle.c (via oracle/shim/btl_bloomfilter/).  So the categorizer
layer (minCount quantiles, frame-count rules, record and summary formatting,
paired-end handling, the command-line options) is the reference's own code and
the filter layer is the oracle's.

What is produced (all small, committed):
  ss.{bf,sdsl}, ss_ids.txt   miBF with 3 spaced seeds (span 25, weight 19) over
                             8 seeded targets (one target has two contigs, one
                             shares a block with another, one is repeat-rich).
  km.{bf,sdsl}, km_ids.txt   the same targets indexed by 3 ntHash hashes of
                             25-mers (k-mer mode).
  reads_se.fa.gz, reads_1.fq.gz, reads_2.fq.gz   reads of the kinds the
                             Bloom-filter fixtures hold, some with comments.
  mi_<case>.tsv              the categorizer's stdout (per-read records).
  mi_<case>_summary.tsv      the categorizer's <prefix>_summary.tsv.

Single-end summaries come from a 3-thread run: with one thread the reference's
single-end loop never counts reads (MIBFClassifier.hpp:217-226 leaves
m_numRead at 0), so its summary rates divide by zero; the per-read records of
those cases come from a 1-thread run, which keeps input order.  The threaded
loop copies records with cpy_kseq (Common/kseq_util.h:17-36), which skips
empty fields and so reuses a recycled record's old sequence or comment (or a
null one); reads_se.fa.gz therefore holds no empty record, and the empty /
short / all-N records sit in reads_edge.fa.gz, used with one thread only.

Usage: python tests/golden/make_golden_mibf.py
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
OUT = os.path.join(HERE, "mibf")
sys.path.insert(0, HERE)
sys.path.insert(0, ROOT)

from make_golden import genome, make_reads  # noqa: E402

SEEDS = [
    # zeros at {4,8,11,13,16,20}, {2,7,10,14,17,22}, {5,6,9,15,18,19}: symmetric
    "".join("0" if i in z else "1" for i in range(25))
    for z in ({4, 8, 11, 13, 16, 20}, {2, 7, 10, 14, 17, 22}, {5, 6, 9, 15, 18, 19})
]

CASES = {
    # name: (filter prefix, extra args, paired)
    "ss_se": ("ss", [], False),
    "ss_se_s50_m2": ("ss", ["-s", "50", "-m", "2"], False),
    "ss_se_a2_c2": ("ss", ["-a", "2", "-c", "2"], False),
    "ss_se_a3_b": ("ss", ["-a", "3", "-b"], False),
    "ss_se_hit": ("ss", ["-i"], False),
    "ss_se_fa": ("ss", ["--fa"], False),
    "ss_pe": ("ss", [], True),
    "ss_pe_hit_b": ("ss", ["-i", "-b", "-m", "3"], True),
    "ss_pe_fq": ("ss", ["--fq"], True),
    "ss_edge": ("ss", [], None),
    "km_se": ("km", [], False),
    "km_pe": ("km", [], True),
}


def targets(rng):
    gcs = [0.50, 0.41, 0.60, 0.45, 0.55, 0.38, 0.62, 0.48]
    seqs = [genome(rng, 5000, gc) for gc in gcs]
    seqs[7][1000:2500] = seqs[0][2000:3500]             # shared block
    unit = genome(rng, 60, 0.5)
    seqs[5][500:3500] = np.tile(unit, 50)                 # repeat-rich target
    recs = [(i + 1, f"t{i + 1}", s) for i, s in enumerate(seqs)]
    recs.append((3, "t3", genome(rng, 1500, 0.52)))       # second contig of ID 3
    return recs


def with_comments(names):
    return [n + (" cmt=%d" % i if i % 7 == 3 else "") for i, n in enumerate(names)]


def write_fa(path, names, seqs):
    with gzip.open(path, "wb", compresslevel=9) as f:
        for n, s in zip(names, seqs):
            f.write(b">" + n.encode() + b"\n" + s + b"\n")


def write_fq(path, names, seqs):
    with gzip.open(path, "wb", compresslevel=9) as f:
        for n, s in zip(names, seqs):
            f.write(b"@" + n.encode() + b"\n" + s + b"\n+\n" + b"I" * len(s) + b"\n")


def run(cmd, cwd):
    p = subprocess.run(cmd, cwd=cwd, capture_output=True)
    if p.returncode:
        sys.stderr.write(p.stderr.decode(errors="replace"))
        raise SystemExit(f"failed: {' '.join(cmd)}")
    return p.stdout


def main():
    cat = os.path.join(REF_BIN, "biobloommicategorizer")
    if not os.path.exists(cat):
        raise SystemExit("build oracle/_ref first: make -C oracle ref")
    from tests import oracle_lib

    os.makedirs(OUT, exist_ok=True)
    rng = np.random.default_rng(20240612)
    recs = targets(rng)
    seqs = [s.tobytes() for _, _, s in recs]
    ids = [i for i, _, _ in recs]
    names = {}
    for i, n, _ in recs:
        names[i] = n
    for prefix, seeds in (("ss", SEEDS), ("km", None)):
        f = oracle_lib.MIBF.build(seeds=seeds, seqs=seqs, ids=ids, k=25, h=3, occupancy=0.5)
        f.store(os.path.join(OUT, prefix))
        with open(os.path.join(OUT, f"{prefix}_ids.txt"), "w") as fh:
            for i in sorted(names):
                fh.write(f"{i}\t{names[i]}\n")

    gen = [np.frombuffer(s, dtype=np.uint8).copy() for s in seqs[:8]]
    se = [r for r in make_reads(rng, gen, 500, paired=False) if r[0]]
    se_names = with_comments([f"se{i}" for i in range(len(se))])
    write_fa(os.path.join(OUT, "reads_se.fa.gz"), se_names, [r[0] for r in se])
    edge = [b"", b"ACGT", seqs[1][100:124], seqs[1][100:125], b"N" * 150, b"",
            seqs[2][300:450], b"acgtn" * 30, seqs[7][1200:1350]]
    write_fa(os.path.join(OUT, "reads_edge.fa.gz"),
             with_comments([f"edge{i}" for i in range(len(edge))]), edge)
    pe = make_reads(rng, gen, 300, paired=True)
    pe_names = with_comments([f"pe{i}" for i in range(len(pe))])
    write_fq(os.path.join(OUT, "reads_1.fq.gz"), pe_names, [r[0] for r in pe])
    write_fq(os.path.join(OUT, "reads_2.fq.gz"), pe_names, [r[1] for r in pe])

    with tempfile.TemporaryDirectory() as tmp:
        for name, (prefix, extra, paired) in CASES.items():
            filt = os.path.join(OUT, f"{prefix}.bf")
            if paired is None:
                inputs = [os.path.join(OUT, "reads_edge.fa.gz")]
            elif paired:
                inputs = ["-e", os.path.join(OUT, "reads_1.fq.gz"),
                          os.path.join(OUT, "reads_2.fq.gz")]
            else:
                inputs = [os.path.join(OUT, "reads_se.fa.gz")]
            out = run([cat, "-t", "1", "-p", "one", "-f", filt] + extra + inputs, cwd=tmp)
            with open(os.path.join(OUT, f"mi_{name}.tsv"), "wb") as fh:
                fh.write(out)
            if paired is None:
                continue
            if paired:
                shutil.copy(os.path.join(tmp, "one_summary.tsv"),
                            os.path.join(OUT, f"mi_{name}_summary.tsv"))
            else:
                run([cat, "-t", "3", "-p", "three", "-f", filt] + extra + inputs, cwd=tmp)
                shutil.copy(os.path.join(tmp, "three_summary.tsv"),
                            os.path.join(OUT, f"mi_{name}_summary.tsv"))
    print("miBF golden fixtures written to", OUT)


if __name__ == "__main__":
    main()
