"""The CPU oracle against the reference's own code, live, on seeded random
cases (oracle/_ref/ref_harness, compiled from the reference sources):
SeqEval::evalRead on filters with k from 12 to 64 and 1 to 7 hash functions,
reads of 10 bp to 2 kb with N runs, lower-case bases and substitutions, scores
from 0 to 0.8 and streak thresholds 0 to 5, single reads and pairs (per-read
hit sets equal); SeqEval::evalScore under the four scoring methods (bit for
bit); sdust's masked intervals on reads with tandem repeats (equal); and the
reference biobloommaker's bit arrays for several k, FPR and hash counts; and
the reference CLI's summary.tsv (reads, pairs, -i, a match length).  Host
only; skipped where the reference has not been built (make -C oracle ref)."""
import os

import numpy as np
import pytest

from tests import oracle_lib as ol

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HARNESS = os.path.join(ROOT, "oracle", "_ref", "ref_harness")


def _reads(rng, genomes, n):
    acgt = np.frombuffer(b"ACGT", dtype=np.uint8)
    out = []
    for _ in range(n):
        length = int(rng.integers(10, 2000))
        src = int(rng.integers(-1, len(genomes)))
        if src >= 0:
            st = int(rng.integers(0, len(genomes[src]) - length))
            r = genomes[src][st:st + length].copy()
        else:
            r = rng.choice(acgt, length)
        m = rng.random(length) < 0.01
        r[m] = rng.choice(acgt, int(m.sum()))
        if rng.random() < 0.3:
            a = int(rng.integers(0, length))
            r[a:a + int(rng.integers(1, 30))] = ord("N")
        if rng.random() < 0.2:
            r = np.where(rng.random(length) < 0.5, r | 0x20, r).astype(np.uint8)
        out.append(r.tobytes())
    return out


@pytest.mark.parametrize("seed,k,h,score,streak", [
    (1, 25, 0, 0.15, 3), (2, 12, 2, 0.5, 1), (3, 31, 5, 0.05, 0), (4, 64, 1, 0.8, 5),
    (5, 21, 7, 0.0, 2), (6, 17, 3, 0.3, 4)])
def test_oracle_equals_reference_seqeval(seed, k, h, score, streak, tmp_path):
    import bench
    if not os.path.exists(HARNESS):
        pytest.skip("oracle/_ref/ref_harness is not built (make -C oracle ref)")
    rng = np.random.default_rng(seed)
    acgt = np.frombuffer(b"ACGT", dtype=np.uint8)
    genomes = [rng.choice(acgt, 40000) for _ in range(2)]
    filters = [ol.Filter.make([g.tobytes()], k=k, fpr=0.2, h=h) for g in genomes]
    paths = []
    for i, f in enumerate(filters):
        stem = str(tmp_path / f"o{i}")
        f.store(stem + ".bf")
        ol.write_info(stem + ".txt", f"o{i}", f.k, 0.2, f.h, 1, "x", f.m, 1, 0.1, 0, 0.1)
        paths.append(stem + ".bf")
    reads = _reads(rng, genomes, 1500)
    seq, off = ol.pack_reads(reads)
    want, _ = ol.classify(seq, off, filters, score, streak)
    fq = str(tmp_path / "r.fq")
    bench.write_single_fastq(fq, np.frombuffer(seq, dtype=np.uint8), off, len(reads))
    rows = bench.harness_hits(HARNESS, paths, fq, score=score, streak=streak)
    got = np.array([r[0] for r in rows], dtype=np.uint64)
    assert len(got) == len(reads)
    assert want[:, 0].any()          # the case exercises hits
    assert np.array_equal(got, want[:, 0])


@pytest.mark.parametrize("seed,score,streak", [(11, 0.15, 3), (12, 0.4, 1)])
def test_oracle_pairs_equal_reference_seqeval(seed, score, streak, tmp_path):
    """Pairs: each mate is evaluated on its own (evaluateReadStd per mate)."""
    import bench
    if not os.path.exists(HARNESS):
        pytest.skip("oracle/_ref/ref_harness is not built (make -C oracle ref)")
    rng = np.random.default_rng(seed)
    acgt = np.frombuffer(b"ACGT", dtype=np.uint8)
    genomes = [rng.choice(acgt, 40000) for _ in range(3)]
    filters = [ol.Filter.make([g.tobytes()], k=25, fpr=0.1) for g in genomes]
    paths = []
    for i, f in enumerate(filters):
        stem = str(tmp_path / f"p{i}")
        f.store(stem + ".bf")
        ol.write_info(stem + ".txt", f"p{i}", f.k, 0.1, f.h, 1, "x", f.m, 1, 0.1, 0, 0.1)
        paths.append(stem + ".bf")
    m1, m2 = _reads(rng, genomes, 1000), _reads(rng, genomes, 1000)
    s1, off1 = ol.pack_reads(m1)
    s2, off2 = ol.pack_reads(m2)
    w1, _ = ol.classify(s1, off1, filters, score, streak)
    w2, _ = ol.classify(s2, off2, filters, score, streak)
    fq1, fq2 = str(tmp_path / "r_1.fq"), str(tmp_path / "r_2.fq")
    bench.write_single_fastq(fq1, np.frombuffer(s1, dtype=np.uint8), off1, len(m1))
    bench.write_single_fastq(fq2, np.frombuffer(s2, dtype=np.uint8), off2, len(m2))
    rows = bench.harness_hits(HARNESS, paths, fq1, fq2, score=score, streak=streak)
    assert len(rows) == len(m1)
    assert w1[:, 0].any() and w2[:, 0].any()
    assert np.array_equal(np.array([r[0] for r in rows], dtype=np.uint64), w1[:, 0])
    assert np.array_equal(np.array([r[1] for r in rows], dtype=np.uint64), w2[:, 0])


def _filters(rng, tmp_path, tag, n=2, k=25, fpr=0.1):
    acgt = np.frombuffer(b"ACGT", dtype=np.uint8)
    genomes = [rng.choice(acgt, 40000) for _ in range(n)]
    filters = [ol.Filter.make([g.tobytes()], k=k, fpr=fpr) for g in genomes]
    paths = []
    for i, f in enumerate(filters):
        stem = str(tmp_path / f"{tag}{i}")
        f.store(stem + ".bf")
        ol.write_info(stem + ".txt", f"{tag}{i}", f.k, fpr, f.h, 1, "x", f.m, 1, 0.1, 0, 0.1)
        paths.append(stem + ".bf")
    return genomes, filters, paths


@pytest.mark.parametrize("method,scoring", [("simple", ol.SIMPLE), ("length", ol.LENGTH),
                                            ("harmonic", ol.HARMONIC),
                                            ("binomial", ol.BINOMIAL)])
def test_oracle_scores_equal_reference_evalscore(method, scoring, tmp_path):
    """SeqEval::evalScore of every read against every filter, bit for bit."""
    import subprocess

    import bench
    if not os.path.exists(HARNESS):
        pytest.skip("oracle/_ref/ref_harness is not built (make -C oracle ref)")
    rng = np.random.default_rng(21)
    genomes, filters, paths = _filters(rng, tmp_path, "s")
    reads = _reads(rng, genomes, 800)
    seq, off = ol.pack_reads(reads)
    want = ol.classify_scores(seq, off, filters, scoring=scoring, streak=3)
    fq = str(tmp_path / "r.fq")
    bench.write_single_fastq(fq, np.frombuffer(seq, dtype=np.uint8), off, len(reads))
    p = subprocess.run([HARNESS, "scores", method, "3", ",".join(paths), fq],
                       capture_output=True, text=True, check=True)
    got = np.array([[int(x, 16) for x in line.split("\t")[1].split(",")]
                    for line in p.stdout.splitlines()], dtype=np.uint64)
    assert got.shape == want.shape
    assert (want > 0).any()
    assert np.array_equal(got, want.view(np.uint64))


@pytest.mark.parametrize("T,W", [(20, 64), (10, 32), (30, 64)])
def test_oracle_sdust_equals_reference(T, W, tmp_path):
    """The intervals the reference's sdust masks, on reads with tandem repeats
    and homopolymers spliced into random sequence."""
    import subprocess

    import bench
    if not os.path.exists(HARNESS):
        pytest.skip("oracle/_ref/ref_harness is not built (make -C oracle ref)")
    rng = np.random.default_rng(T * 100 + W)
    acgt = np.frombuffer(b"ACGT", dtype=np.uint8)
    reads = []
    for _ in range(500):
        r = rng.choice(acgt, int(rng.integers(30, 600)))
        for _ in range(int(rng.integers(0, 4))):
            unit = rng.choice(acgt, int(rng.integers(1, 7)))
            rep = np.tile(unit, int(rng.integers(3, 40)))
            a = int(rng.integers(0, len(r)))
            r = np.concatenate([r[:a], rep, r[a:]])
        if rng.random() < 0.2:
            r[int(rng.integers(0, len(r)))] = ord("N")
        reads.append(r.tobytes())
    seq, off = ol.pack_reads(reads)
    fq = str(tmp_path / "d.fq")
    bench.write_single_fastq(fq, np.frombuffer(seq, dtype=np.uint8), off, len(reads))
    p = subprocess.run([HARNESS, "dust", str(T), str(W), fq], capture_output=True, text=True,
                       check=True)
    lines = p.stdout.splitlines()
    assert len(lines) == len(reads)
    masked = 0
    for r, line in zip(reads, lines):
        field = line.split("\t")[1] if "\t" in line else ""
        got = [tuple(int(v) for v in iv.split("-")) for iv in field.split(",") if iv]
        want, _ = ol.sdust(r, T, W)
        masked += bool(want)
        assert got == want
    assert masked > 0


@pytest.mark.parametrize("k,fpr,g", [(25, 0.075, 0), (16, 0.01, 0), (31, 0.2, 5), (64, 0.05, 2)])
def test_oracle_maker_equals_reference_maker(k, fpr, g, tmp_path):
    """The reference biobloommaker (BloomFilterGenerator) on multi-record FASTA
    with N runs and lower case: the oracle's maker gives the same m, h, k and
    bit array."""
    import subprocess
    maker = os.path.join(ROOT, "oracle", "_ref", "biobloommaker")
    if not os.path.exists(maker):
        pytest.skip("oracle/_ref/biobloommaker is not built (make -C oracle ref)")
    rng = np.random.default_rng(k * 1000 + g)
    acgt = np.frombuffer(b"ACGT", dtype=np.uint8)
    recs = []
    for _ in range(4):
        r = rng.choice(acgt, int(rng.integers(50, 30000)))
        if rng.random() < 0.5:
            a = int(rng.integers(0, len(r)))
            r[a:a + int(rng.integers(1, 50))] = ord("N")
        if rng.random() < 0.5:
            r = np.where(rng.random(len(r)) < 0.3, r | 0x20, r).astype(np.uint8)
        recs.append(r.tobytes())
    with open(tmp_path / "in.fa", "wb") as f:
        for i, r in enumerate(recs):
            f.write(b">c%d\n%s\n" % (i, r))
    cmd = [maker, "-p", "m", "-k", str(k), "-f", str(fpr)] + (["-g", str(g)] if g else [])
    subprocess.run(cmd + ["in.fa"], cwd=tmp_path, check=True, capture_output=True)
    ref = ol.Filter.load(str(tmp_path / "m.bf"))
    mine = ol.Filter.make(recs, k=k, fpr=fpr, h=g)
    assert (mine.m, mine.h, mine.k) == (ref.m, ref.h, ref.k)
    assert np.array_equal(mine.bits(), ref.bits())


@pytest.mark.parametrize("paired,inclusive,score", [(False, False, 0.15), (True, False, 0.15),
                                                    (True, True, 0.3), (False, False, 40)])
def test_oracle_summary_equals_reference_cli(paired, inclusive, score, tmp_path):
    """summary.tsv of the reference CLI (oracle/_ref/biobloomcategorizer, the
    reference's ResultsManager) on random reads and pairs, with and without -i
    and with a minimum match length: the oracle's counters and summary text
    give the same file."""
    import subprocess

    import bench
    cli = os.path.join(ROOT, "oracle", "_ref", "biobloomcategorizer")
    if not os.path.exists(cli):
        pytest.skip("oracle/_ref/biobloomcategorizer is not built (make -C oracle ref)")
    rng = np.random.default_rng(31 + paired + 2 * inclusive)
    genomes, filters, paths = _filters(rng, tmp_path, "c", n=3)
    mates = [_reads(rng, genomes, 700) for _ in range(2 if paired else 1)]
    scoring = ol.LENGTH if score > 1 else ol.SIMPLE
    hits, files = [], []
    for m, reads in enumerate(mates):
        seq, off = ol.pack_reads(reads)
        hits.append(ol.classify(seq, off, filters, score, 3, scoring)[0])
        files.append(str(tmp_path / f"r_{m + 1}.fq"))
        bench.write_single_fastq(files[-1], np.frombuffer(seq, dtype=np.uint8), off, len(reads))
    counts, _ = ol.summary_counts(hits[0], 3, hits[1] if paired else None, inclusive=inclusive)
    args = [cli, "-t", "1", "-p", "out", "-s", str(score), "-f", " ".join(paths)]
    args += (["-e"] if paired else []) + (["-i"] if inclusive else []) + files
    subprocess.run(args, cwd=tmp_path, check=True, capture_output=True)
    with open(tmp_path / "out_summary.tsv") as f:
        want = f.read()
    ids = [f"c{i}" for i in range(3)]
    assert ol.summary_tsv(counts, ids, len(mates[0])) == want
