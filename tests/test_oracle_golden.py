"""The CPU oracle against the golden fixtures written by the reference's own
code (tests/golden/make_golden.py) and against the properties the reference's
unit tests assert."""
import numpy as np
import pytest

from tests import oracle_lib as ol
from tests.fixtures import expected_hits, filter_ids, filter_paths, golden, read_fastx

SE_CASES = [("se_s0.15_r3", 0.15, 3), ("se_s0.5_r1", 0.5, 1), ("se_s0.05_r0", 0.05, 0),
            ("se_s40", 40, 3)]


def _hitsets(hits, nf):
    return [set(f for f in range(nf) if (int(h[f // 64]) >> (f % 64)) & 1) for h in hits]


@pytest.mark.parametrize("name,score,streak", SE_CASES)
def test_oracle_single_end_matches_reference(name, score, streak):
    filters = [ol.Filter.load(p) for p in filter_paths()]
    recs = read_fastx(golden("reads_se.fa.gz"))
    seq, off = ol.pack_reads([s for _, s in recs])
    scoring = ol.LENGTH if score > 1 else ol.SIMPLE
    hits, _ = ol.classify(seq, off, filters, score, streak, scoring)
    rows, summary = expected_hits(name)
    assert [r[0] for r in rows] == [n for n, _ in recs]
    assert _hitsets(hits, 3) == [r[1] for r in rows]
    counts, _ = ol.summary_counts(hits, 3)
    assert ol.summary_tsv(counts, filter_ids(), len(recs)) == summary


def test_oracle_pairs_match_reference():
    filters = [ol.Filter.load(p) for p in filter_paths()]
    r1 = read_fastx(golden("reads_1.fq.gz"))
    r2 = read_fastx(golden("reads_2.fq.gz"))
    s1, o1 = ol.pack_reads([s for _, s in r1])
    s2, o2 = ol.pack_reads([s for _, s in r2])
    h1, _ = ol.classify(s1, o1, filters)
    h2, _ = ol.classify(s2, o2, filters)
    rows, summary = expected_hits("pe_s0.15_r3")
    assert _hitsets(h1, 3) == [r[1] for r in rows]
    assert _hitsets(h2, 3) == [r[2] for r in rows]
    counts, _ = ol.summary_counts(h1, 3, h2, inclusive=False)
    assert ol.summary_tsv(counts, filter_ids(), len(r1)) == summary
    with open(golden("expected_summary_pe.tsv")) as f:
        assert ol.summary_tsv(counts, filter_ids(), len(r1)) == f.read()
    counts, _ = ol.summary_counts(h1, 3, h2, inclusive=True)
    with open(golden("expected_summary_pe_incl.tsv")) as f:
        assert ol.summary_tsv(counts, filter_ids(), len(r1)) == f.read()


def test_oracle_summary_matches_reference_cli():
    filters = [ol.Filter.load(p) for p in filter_paths()]
    recs = read_fastx(golden("reads_se.fa.gz"))
    seq, off = ol.pack_reads([s for _, s in recs])
    for name, score in (("se", 0.15), ("se_s40", 40)):
        hits, _ = ol.classify(seq, off, filters, score, 3, ol.LENGTH if score > 1 else ol.SIMPLE)
        counts, _ = ol.summary_counts(hits, 3)
        with open(golden(f"expected_summary_{name}.tsv")) as f:
            assert ol.summary_tsv(counts, filter_ids(), len(recs)) == f.read()


def test_oracle_maker_matches_reference_maker():
    """The oracle's maker reproduces the reference maker's bit array."""
    rng = np.random.default_rng(20240611)
    from tests.golden.make_golden import genome
    g0 = genome(rng, 20000, 0.5).tobytes()
    ref = ol.Filter.load(golden("f0.bf"))
    mine = ol.Filter.make([g0], k=25, fpr=0.075)
    assert (mine.m, mine.h, mine.k) == (ref.m, ref.h, ref.k)
    assert np.array_equal(mine.bits(), ref.bits())


def test_bloomfilter_tests_properties():
    """Tests/BloomFilterTests.cpp:44-59: 4 inserted 20-mers are contained and
    2 others are not, k=20, h=5 (filter 1e6 bits instead of 1e9)."""
    f = ol.Filter.create(1000000, 5, 20)
    for s in (b"ATCGGGTCATCAACCAATAT", b"ATCGGGTCATCAACCAATAC",
              b"ATCGGGTCATCAACCAATAG", b"ATCGGGTCATCAACCAATAA"):
        f.insert_sequence(s)
    for s in (b"ATCGGGTCATCAACCAATAT", b"ATCGGGTCATCAACCAATAC",
              b"ATCGGGTCATCAACCAATAG", b"ATCGGGTCATCAACCAATAA"):
        assert f.contains_kmer(s)
    assert not f.contains_kmer(b"ATCGGGTCATCAACCAATTA")
    assert not f.contains_kmer(b"ATCGGGTCATCAACCAATTC")


def test_seqeval_tests_length_mode():
    """Tests/SeqEvalTests.cpp:26-40: with a k=4, h=2 filter loaded from
    NNNNNAAAAA, LENGTH scoring accepts AAAAANNNNN at 5 bases and rejects at 6."""
    f = ol.Filter.load(golden("len.bf"))
    seq, off = ol.pack_reads([b"AAAAANNNNN"])
    h5, _ = ol.classify(seq, off, [f], 5, 3, ol.LENGTH)
    h6, _ = ol.classify(seq, off, [f], 6, 3, ol.LENGTH)
    assert int(h5[0, 0]) == 1 and int(h6[0, 0]) == 0


def test_nthash_canonical_and_rolling():
    """Canonical hash is strand independent; the rolling iterator equals the
    direct hash at every position, and skips k-mers with non-ACGT bases."""
    rng = np.random.default_rng(7)
    s = rng.choice(np.frombuffer(b"ACGT", dtype=np.uint8), 200).tobytes()
    rc = s.translate(bytes.maketrans(b"ACGT", b"TGCA"))[::-1]
    k = 25
    L = ol.lib()
    fw = ol.kmers(s, 3, k)
    rv = ol.kmers(rc, 3, k)
    assert len(fw) == len(rv) == 200 - k + 1
    for (p, hv), (q, hr) in zip(fw, reversed(rv)):
        assert hv == hr
        f = L.oracle_nt_forward(s[p:p + k], k)
        r = L.oracle_nt_reverse(s[p:p + k], k)
        assert hv[0] == min(f, r)
    t = bytearray(s)
    t[50] = ord("N")
    pos = [p for p, _ in ol.kmers(bytes(t), 1, k)]
    assert pos == [p for p in range(200 - k + 1) if not (p <= 50 < p + k)]
    assert [h for _, h in ol.kmers(s.lower(), 3, k)] == [h for _, h in fw]


def test_sizing_matches_reference_formulas():
    # Common/BloomFilterInfo.h:57-76 for the 5 Mbp, k=25, FPR 0.075 filter
    assert ol.lib().oracle_calc_optimal_hash_num(0.075) == 3
    assert ol.lib().oracle_calc_optimal_size(5000000 - 24, 0.075, 3) == 27387648


# HARMONIC / BINOMIAL scoring (-S), golden files from tests/golden/make_golden_modes.py
MODE_CASES = [("harmonic_s0.15_r3", "harmonic", 0.15, 3, False),
              ("harmonic_s0.4_r1", "harmonic", 0.4, 1, False),
              ("harmonic_pe_s0.15_r3", "harmonic", 0.15, 3, True),
              ("binomial_s100_r3", "binomial", 100, 3, False),
              ("binomial_s30_r2", "binomial", 30, 2, False),
              ("binomial_pe_s100_r3", "binomial", 100, 3, True)]


def mode_args(method, score):
    """(threshold, scoring) as BioBloomCategorizer.cpp:414-441 derives them."""
    if method == "binomial":
        return 10.0 ** (-(score / 10.0)), ol.BINOMIAL
    return score, ol.HARMONIC


@pytest.mark.parametrize("name,method,score,streak,paired", MODE_CASES)
def test_oracle_scoring_modes_match_reference(name, method, score, streak, paired):
    filters = [ol.Filter.load(p) for p in filter_paths()]
    thr, scoring = mode_args(method, score)
    rows, summary = expected_hits(name)
    if paired:
        r1 = read_fastx(golden("reads_1.fq.gz"))
        r2 = read_fastx(golden("reads_2.fq.gz"))
        s1, o1 = ol.pack_reads([s for _, s in r1])
        s2, o2 = ol.pack_reads([s for _, s in r2])
        h1, _ = ol.classify(s1, o1, filters, thr, streak, scoring)
        h2, _ = ol.classify(s2, o2, filters, thr, streak, scoring)
        assert _hitsets(h1, 3) == [r[1] for r in rows]
        assert _hitsets(h2, 3) == [r[2] for r in rows]
        counts, _ = ol.summary_counts(h1, 3, h2)
        n = len(r1)
    else:
        recs = read_fastx(golden("reads_se.fa.gz"))
        seq, off = ol.pack_reads([s for _, s in recs])
        hits, _ = ol.classify(seq, off, filters, thr, streak, scoring)
        assert _hitsets(hits, 3) == [r[1] for r in rows]
        counts, _ = ol.summary_counts(hits, 3)
        n = len(recs)
    assert ol.summary_tsv(counts, filter_ids(), n) == summary
    with open(golden(f"expected_summary_{name}.tsv")) as f:
        assert ol.summary_tsv(counts, filter_ids(), n) == f.read()
