"""The CPU oracle's SDUST masking (-D) against the reference's own code on the
DUST fixtures (tests/golden/make_golden_dust.py): masked intervals of
Common/sdust.c for three (T, W) settings, and per-read hits, summaries and
evalScore values of SeqEval with masking on."""
import os
import sys

import numpy as np
import pytest

from tests import oracle_lib as ol
from tests.fixtures import expected_hits, filter_ids, filter_paths, golden, read_fastx

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))

import make_golden_dust as mgd  # noqa: E402


def _hitsets(hits, nf):
    return [set(f for f in range(nf) if (int(h[f // 64]) >> (f % 64)) & 1) for h in hits]


def expected_intervals(name):
    out = []
    with open(golden(f"expected_dust_{name}.tsv")) as f:
        for line in f:
            rname, iv = line.rstrip("\n").split("\t")
            out.append((rname, [tuple(int(x) for x in p.split("-")) for p in iv.split(",")]
                        if iv else []))
    return out


@pytest.mark.parametrize("name", sorted(mgd.DUST_PARAMS))
def test_oracle_sdust_matches_reference(name):
    T, W = mgd.DUST_PARAMS[name]
    recs = read_fastx(golden("reads_dust.fa.gz"))
    want = expected_intervals(name)
    assert [n for n, _ in recs] == [n for n, _ in want]
    for (_, seq), (_, iv) in zip(recs, want):
        got, _ = ol.sdust(seq, T, W)
        assert got == iv


def test_sdust_properties():
    # a homopolymer is masked whole; ordinary sequence is not masked
    assert ol.sdust(b"A" * 100)[0] == [(0, 100)]
    rng = np.random.default_rng(3)
    rand = rng.choice(np.frombuffer(b"ACGT", dtype=np.uint8), 400).tobytes()
    assert ol.sdust(rand)[0] == []
    # an N ends a run: masked pieces stay on their side of it
    iv, _ = ol.sdust(b"A" * 30 + b"N" + b"A" * 30)
    assert all(not (s <= 30 < f) for s, f in iv)
    # the pending list grows with the square of the window on repeats
    _, mp = ol.sdust(b"AC" * 1000, 20, 64)
    assert mp > 64


def _method(method, score):
    if method == "binomial":
        return 10.0 ** (-(float(score) / 10.0)), ol.BINOMIAL
    if method == "harmonic":
        return float(score), ol.HARMONIC
    if float(score) > 1:
        return float(int(float(score))), ol.LENGTH
    return float(score), ol.SIMPLE


@pytest.mark.parametrize("name", sorted(mgd.HIT_CASES))
def test_oracle_hits_with_dust_match_reference(name):
    method, score, streak, paired = mgd.HIT_CASES[name]
    thr, scoring = _method(method, score)
    filters = [ol.Filter.load(p) for p in filter_paths()]
    rows, summary = expected_hits(name)
    r1 = read_fastx(golden("reads_dust.fa.gz"))
    s1, o1 = ol.pack_reads([s for _, s in r1])
    with ol.dust(20, 64):
        h1, _ = ol.classify(s1, o1, filters, thr, int(streak), scoring)
        h2 = None
        if paired:
            r2 = read_fastx(golden("reads_dust_2.fa.gz"))
            s2, o2 = ol.pack_reads([s for _, s in r2])
            h2, _ = ol.classify(s2, o2, filters, thr, int(streak), scoring)
    assert _hitsets(h1, 3) == [r[1] for r in rows]
    if paired:
        assert _hitsets(h2, 3) == [r[2] for r in rows]
    counts, _ = ol.summary_counts(h1, 3, h2)
    assert ol.summary_tsv(counts, filter_ids(), len(r1)) == summary


@pytest.mark.parametrize("name", sorted(mgd.SCORE_CASES))
def test_oracle_scores_with_dust_match_reference(name):
    method, streak = mgd.SCORE_CASES[name]
    scoring = {"simple": ol.SIMPLE, "length": ol.LENGTH, "binomial": ol.BINOMIAL}[method]
    filters = [ol.Filter.load(p) for p in filter_paths()]
    recs = read_fastx(golden("reads_dust.fa.gz"))
    seq, off = ol.pack_reads([s for _, s in recs])
    with ol.dust(20, 64):
        got = ol.classify_scores(seq, off, filters, scoring, streak)
    rows = []
    with open(golden(f"expected_scores_{name}.tsv")) as f:
        for line in f:
            rows.append([int(v, 16) for v in line.rstrip("\n").split("\t")[1].split(",")])
    assert np.array_equal(got.view(np.uint64), np.array(rows, dtype=np.uint64))
