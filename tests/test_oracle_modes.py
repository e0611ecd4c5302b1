"""The CPU oracle's exhaustive scores (SeqEval::evalScore) and filtering modes
(ordered -c, best hit -b, with scores -w) against the reference's own code:
scores from oracle/_ref/ref_harness (tests/golden/make_golden_scores.py) and
summaries from the reference CLI (tests/golden/make_golden_print.py)."""
import gzip
import os
import re
import sys

import numpy as np
import pytest

from tests import oracle_lib as ol
from tests.fixtures import filter_ids, filter_paths, golden, read_fastx

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))

import make_golden_print as mgp  # noqa: E402
import make_golden_scores as mgs  # noqa: E402

METHODS = {"simple": ol.SIMPLE, "length": ol.LENGTH, "harmonic": ol.HARMONIC,
           "binomial": ol.BINOMIAL}


def expected_scores(case):
    names, rows = [], []
    with open(golden(f"expected_scores_{case}.tsv")) as f:
        for line in f:
            name, vals = line.rstrip("\n").split("\t")
            names.append(name)
            rows.append([int(v, 16) for v in vals.split(",")])
    return names, np.array(rows, dtype=np.uint64)


@pytest.mark.parametrize("case", sorted(mgs.CASES))
def test_oracle_scores_match_reference_bit_for_bit(case):
    method, streak = mgs.CASES[case]
    filters = [ol.Filter.load(p) for p in filter_paths()]
    recs = read_fastx(golden("reads_se.fa.gz"))
    seq, off = ol.pack_reads([s for _, s in recs])
    got = ol.classify_scores(seq, off, filters, METHODS[method], streak)
    names, want = expected_scores(case)
    assert names == [n for n, _ in recs]
    assert np.array_equal(got.view(np.uint64), want)


def golden_sections(case):
    """{file name: contents} of a golden print file ("### <name>\n" headers)."""
    with gzip.open(golden(f"print_{case}.txt.gz"), "rb") as f:
        text = f.read().decode()
    parts = re.split(r"^### (.*)\n", text, flags=re.M)
    return dict(zip(parts[1::2], parts[2::2]))


def case_options(args):
    """The CLI's reading of the mode, scoring and threshold options
    (BioBloomCategorizer.cpp:276-318, 414-441)."""
    mode = "std"
    method, score, inclusive = "simple", None, False
    i = 0
    while i < len(args):
        a = args[i]
        if a == "-c":
            mode = "ordered"
        elif a == "-b":
            mode = "besthit"
        elif a == "-w":
            mode = "scores"
        elif a == "-i":
            inclusive = True
        elif a == "-S":
            method = args[i + 1]
            i += 1
        elif a == "-s":
            score = float(args[i + 1])
            i += 1
        i += 1
    if method == "binomial":
        thr = 10.0 ** (-((100.0 if score is None else score) / 10.0))
        scoring = ol.BINOMIAL
    else:
        thr = 0.15 if score is None else score
        scoring = METHODS[method]
        if mode != "besthit" and int(thr) > 1:
            thr, scoring = float(int(thr)), ol.LENGTH
    return mode, scoring, thr, inclusive


def mode_hits(mode, scoring, thr, filters, seq, off):
    if mode == "besthit":
        hits, _ = ol.best_hit(ol.classify_scores(seq, off, filters, scoring, 3))
        return hits
    hits, _ = ol.classify(seq, off, filters, thr, 3, scoring)
    return hits


SUMMARY_CASES = sorted(c for c, (_, kind) in mgp.MODE_CASES.items() if kind in ("se", "pe"))


@pytest.mark.parametrize("case", SUMMARY_CASES)
def test_oracle_mode_summaries_match_reference_cli(case):
    args, kind = mgp.MODE_CASES[case]
    mode, scoring, thr, inclusive = case_options(args)
    filters = [ol.Filter.load(p) for p in filter_paths()]
    if kind == "pe":
        r1 = read_fastx(golden("reads_1.fq.gz"))
        r2 = read_fastx(golden("reads_2.fq.gz"))
        s1, o1 = ol.pack_reads([s for _, s in r1])
        s2, o2 = ol.pack_reads([s for _, s in r2])
        h1 = mode_hits(mode, scoring, thr, filters, s1, o1)
        h2 = mode_hits(mode, scoring, thr, filters, s2, o2)
        if mode == "ordered":
            h1, h2 = ol.ordered(h1, 3, h2, inclusive)
        counts, _ = ol.summary_counts(h1, 3, h2, inclusive=inclusive)
        n = len(r1)
    else:
        recs = read_fastx(golden("reads_se.fa.gz"))
        seq, off = ol.pack_reads([s for _, s in recs])
        hits = mode_hits(mode, scoring, thr, filters, seq, off)
        if mode == "ordered":
            hits, _ = ol.ordered(hits, 3)
        counts, _ = ol.summary_counts(hits, 3)
        n = len(recs)
    want = golden_sections(case)["out_summary.tsv"]
    assert ol.summary_tsv(counts, filter_ids(), n) == want


def test_ordered_keeps_the_first_filter_of_the_combined_hits():
    h1 = np.array([[0b110], [0b000], [0b101]], dtype=np.uint64)
    h2 = np.array([[0b100], [0b010], [0b001]], dtype=np.uint64)
    a, b = ol.ordered(h1, 3, h2, inclusive=False)
    assert a.ravel().tolist() == [0b100, 0, 0b001] and np.array_equal(a, b)
    a, b = ol.ordered(h1, 3, h2, inclusive=True)
    assert a.ravel().tolist() == [0b010, 0b010, 0b001] and np.array_equal(a, b)
    a, _ = ol.ordered(h1, 3)
    assert a.ravel().tolist() == [0b010, 0, 0b001]


def test_best_hit_ties_and_threshold():
    nan = float("nan")
    sc = np.array([[0.5, 0.7, 0.7], [0.0, 0.0, 0.0], [nan, 0.2, 0.1], [-0.0, 0.0, 0.0]])
    hits, best = ol.best_hit(sc)
    assert hits.ravel().tolist() == [0b110, 0, 0b010, 0]
    assert best.tolist() == [0.7, 0.0, 0.2, 0.0]
