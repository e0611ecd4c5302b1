"""Parity of the CUDA path with the CPU oracle and with the golden fixtures
written by the reference's own code.  Every check is bit-exact: per-read
filter hits, categories and summary.tsv text."""
import os
import subprocess
import tempfile

import numpy as np
import pytest

from tests import oracle_lib as ol
from tests.fixtures import expected_hits, filter_ids, filter_paths, golden, read_fastx

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module", autouse=True)
def _need_gpu():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("GPU tests need a CUDA device")
    from biobloom_b200 import _lib
    _lib.lib()  # raises if the library is missing: no fallback


def _sets(hits, nf):
    return [set(f for f in range(nf) if (int(h[f // 64]) >> (f % 64)) & 1) for h in hits]


def _classifier(paths, score=0.15, streak=3, **kw):
    from biobloom_b200 import BioBloomClassifier
    return BioBloomClassifier(paths, score, streak_threshold=streak, **kw)


PATHS = [dict(path=1), dict(path=2), dict(path=2, frames_per_lane=8),
         dict(path=1, warps_per_block=4, frames_per_lane=8), dict(path=3),
         dict(path=3, frames_per_lane=8), dict(path=2, steps=1), dict(path=2, steps=2),
         dict(path=2, steps=3, frames_per_lane=8)]
PATH_IDS = ["plain", "persistent", "persistent-seg8", "plain-w4-seg8", "filter-major",
            "filter-major-seg8", "persistent-full-steps", "persistent-wide-steps",
            "persistent-wide-full-steps-seg8"]


@pytest.mark.parametrize("launch", PATHS, ids=PATH_IDS)
@pytest.mark.parametrize("name,score,streak", [("se_s0.15_r3", 0.15, 3), ("se_s0.5_r1", 0.5, 1),
                                               ("se_s0.05_r0", 0.05, 0), ("se_s40", 40, 3)])
def test_golden_single_end(name, score, streak, launch):
    recs = read_fastx(golden("reads_se.fa.gz"))
    with _classifier(filter_paths(), score, streak, **launch) as bbc:
        hits, _, cat = bbc.classify([s for _, s in recs])
        rows, summary = expected_hits(name)
        assert _sets(hits, 3) == [r[1] for r in rows]
        assert bbc.summary_tsv() == summary


@pytest.mark.parametrize("launch", [PATHS[0], PATHS[1], PATHS[4]],
                         ids=["plain", "persistent", "filter-major"])
def test_golden_pairs(launch):
    r1 = read_fastx(golden("reads_1.fq.gz"))
    r2 = read_fastx(golden("reads_2.fq.gz"))
    rows, summary = expected_hits("pe_s0.15_r3")
    with _classifier(filter_paths(), **launch) as bbc:
        h1, h2, cat = bbc.classify([s for _, s in r1], [s for _, s in r2])
        assert _sets(h1, 3) == [r[1] for r in rows]
        assert _sets(h2, 3) == [r[2] for r in rows]
        assert bbc.summary_tsv() == summary
        with open(golden("expected_summary_pe.tsv")) as f:
            assert bbc.summary_tsv() == f.read()
    with _classifier(filter_paths(), **launch) as bbc:
        bbc.setInclusive()
        bbc.classify([s for _, s in r1], [s for _, s in r2])
        with open(golden("expected_summary_pe_incl.tsv")) as f:
            assert bbc.summary_tsv() == f.read()


def test_file_pipeline_and_read_status():
    with tempfile.TemporaryDirectory() as tmp:
        prefix = os.path.join(tmp, "se")
        status = os.path.join(tmp, "se_readStatus.tsv")
        with _classifier(filter_paths(), 0.15, 3) as bbc:
            bbc.prefix = prefix
            bbc.filter([golden("reads_se.fa.gz")], read_status=status)
        with open(prefix + "_summary.tsv") as f, open(golden("expected_summary_se.tsv")) as g:
            assert f.read() == g.read()
        rows, _ = expected_hits("se_s0.15_r3")
        ids = filter_ids()
        want = []
        for name, hs in rows:
            cat = "noMatch" if not hs else (ids[min(hs)] if len(hs) == 1 else "multiMatch")
            want.append(f"{name}\t{cat}")
        with open(status) as f:
            assert f.read().splitlines() == want
        prefix = os.path.join(tmp, "pe")
        with _classifier(filter_paths()) as bbc:
            bbc.prefix = prefix
            bbc.filterPair(golden("reads_1.fq.gz"), golden("reads_2.fq.gz"))
        with open(prefix + "_summary.tsv") as f, open(golden("expected_summary_pe.tsv")) as g:
            assert f.read() == g.read()


def test_cli_matches_reference_summary():
    cli = os.path.join(ROOT, "biobloom_b200", "bin", "biobloomcategorizer")
    fl = " ".join(filter_paths())
    with tempfile.TemporaryDirectory() as tmp:
        for name, extra, files in (
                ("se", [], [golden("reads_se.fa.gz")]),
                ("pe", ["-e"], [golden("reads_1.fq.gz"), golden("reads_2.fq.gz")]),
                ("pe_incl", ["-e", "-i"], [golden("reads_1.fq.gz"), golden("reads_2.fq.gz")]),
                ("se_s40", ["-s", "40"], [golden("reads_se.fa.gz")])):
            p = subprocess.run([cli, "-p", os.path.join(tmp, name), "-f", fl] + extra + files,
                               capture_output=True, text=True)
            assert p.returncode == 0, p.stderr
            with open(os.path.join(tmp, name + "_summary.tsv")) as f, \
                    open(golden(f"expected_summary_{name}.tsv")) as g:
                assert f.read() == g.read()


def test_seqeval_tests_length_mode_on_gpu():
    """Tests/SeqEvalTests.cpp:26-40 on the device path."""
    for score, want in ((5, 1), (6, 0)):
        with _classifier([golden("len.bf")], score) as bbc:
            hits, _, _ = bbc.classify([b"AAAAANNNNN"])
            assert int(hits[0, 0]) == want


def _random_case(seed, n_filters=3, k=25, h=None, fpr=0.075, glen=30000):
    rng = np.random.default_rng(seed)
    genomes = [rng.choice(np.frombuffer(b"ACGT", dtype=np.uint8), glen) for _ in range(n_filters)]
    filters = [ol.Filter.make([g.tobytes()], k=k, fpr=fpr, h=h or 0) for g in genomes]
    return rng, genomes, filters


def _random_reads(rng, genomes, n, lmin=20, lmax=400, nrate=0.02, sub=0.01):
    reads = []
    for _ in range(n):
        L = int(rng.integers(lmin, lmax))
        src = int(rng.integers(-1, len(genomes)))
        if src >= 0 and L < len(genomes[src]):
            st = int(rng.integers(0, len(genomes[src]) - L))
            r = genomes[src][st:st + L].copy()
        else:
            r = rng.choice(np.frombuffer(b"ACGT", dtype=np.uint8), L)
        m = rng.random(L) < sub
        r[m] = rng.choice(np.frombuffer(b"ACGT", dtype=np.uint8), m.sum())
        if rng.random() < 0.3:
            m = rng.random(L) < nrate
            r[m] = ord("N")
        if rng.random() < 0.1:
            r = np.where(rng.random(L) < 0.5, r | 0x20, r).astype(np.uint8)
        reads.append(r.tobytes())
    return reads


@pytest.mark.parametrize("seed,k,h,score,streak", [
    (1, 25, 0, 0.15, 3), (2, 21, 2, 0.3, 2), (3, 31, 4, 0.05, 1), (4, 17, 1, 0.9, 5),
    (5, 25, 3, 0.0, 3), (6, 25, 3, 1.0, 3), (7, 12, 3, 0.4, 0), (8, 64, 3, 0.15, 3),
    (9, 21, 6, 0.15, 3)])
@pytest.mark.parametrize("launch", PATHS, ids=PATH_IDS)
def test_random_parity_with_oracle(seed, k, h, score, streak, launch, tmp_path):
    rng, genomes, filters = _random_case(seed, k=k, h=h, fpr=0.2)
    paths = []
    for i, f in enumerate(filters):
        stem = str(tmp_path / f"r{i}")
        f.store(stem + ".bf")
        ol.write_info(stem + ".txt", f"r{i}", f.k, 0.2, f.h, 1, "x", f.m, 1, 0.1, 0, 0.1)
        paths.append(stem + ".bf")
    reads = _random_reads(rng, genomes, 3000)
    seq, off = ol.pack_reads(reads)
    want, _ = ol.classify(seq, off, filters, score, streak)
    with _classifier(paths, score, streak, **launch) as bbc:
        hits, _, cat = bbc.classify(reads)
    assert np.array_equal(hits, want)
    counts, cats = ol.summary_counts(want, len(filters))
    assert np.array_equal(cat, cats)


@pytest.mark.parametrize("score,streak,h", [(0.15, 3, 0), (0.5, 1, 0), (0.15, 3, 2), (0.15, 3, 4),
                                            (0.3, 2, 7)])
def test_algorithmic_probe_counts_on_every_step_form(score, streak, h, tmp_path):
    """The counting pass (bbt_set_counting) reports the filter words the
    sequential SeqEval::evalSimple reads, whatever the steps of the kernel:
    plain, persistent with decision-sized, full and two-frames-per-lane steps
    all count the oracle's number; the words issued are never fewer."""
    import torch
    rng, genomes, filters = _random_case(21, n_filters=2, glen=60000, h=h)
    paths = _store(filters, tmp_path, "c")
    reads = _random_reads(rng, genomes, 2500, lmin=20, lmax=600)
    seq, off = ol.pack_reads(reads)
    want, alg = ol.classify(seq, off, filters, score, streak, count_probes=True)
    dseq = torch.tensor(np.frombuffer(seq, dtype=np.uint8), device="cuda")
    doff = torch.tensor(off.astype(np.int64), device="cuda")
    for launch in (dict(path=1), dict(path=2), dict(path=2, steps=1), dict(path=2, steps=2),
                   dict(path=2, steps=3), dict(path=2, steps=2, frames_per_lane=8)):
        with _classifier(paths, score, streak, **launch) as bbc:
            bbc.set_counting(True)
            hits, _, _ = bbc.classify_device(dseq, doff)
            torch.cuda.synchronize()
            st = bbc.last_stats()
            assert np.array_equal(hits.cpu().numpy().view(np.uint64), want), launch
            assert st["probes_algorithmic"] == alg, launch
            assert st["probes_issued"] >= alg, launch


def test_device_batches_and_long_reads(tmp_path):
    """Reads resident on the device, lengths up to 10 kb (several hash windows
    per read), against the oracle; plain and persistent paths agree."""
    import torch
    rng, genomes, filters = _random_case(11, n_filters=2, glen=60000)
    paths = []
    for i, f in enumerate(filters):
        stem = str(tmp_path / f"l{i}")
        f.store(stem + ".bf")
        ol.write_info(stem + ".txt", f"l{i}", f.k, 0.075, f.h, 1, "x", f.m, 1, 0.1, 0, 0.1)
        paths.append(stem + ".bf")
    reads = _random_reads(rng, genomes, 400, lmin=20, lmax=10000, nrate=0.001, sub=0.005)
    seq, off = ol.pack_reads(reads)
    want, _ = ol.classify(seq, off, filters, 0.15, 3)
    dseq = torch.tensor(np.frombuffer(seq, dtype=np.uint8), device="cuda")
    doff = torch.tensor(off.astype(np.int64), device="cuda")
    for launch in PATHS:
        with _classifier(paths, **launch) as bbc:
            hits, _, cat = bbc.classify_device(dseq, doff)
            torch.cuda.synchronize()
            assert np.array_equal(hits.cpu().numpy().view(np.uint64), want)


def _store(filters, tmp_path, tag):
    paths = []
    for i, f in enumerate(filters):
        stem = str(tmp_path / f"{tag}{i}")
        f.store(stem + ".bf")
        ol.write_info(stem + ".txt", f"{tag}{i}", f.k, 0.075, f.h, 1, "x", f.m, 1, 0.1, 0, 0.1)
        paths.append(stem + ".bf")
    return paths


def test_long_first_schedule_autotune_and_graph(tmp_path):
    """Mixed-length reads (20 bp - 10 kb) on the device: the long-first read
    order, the autotuned configuration and a CUDA graph of odd-sized launches
    all give the oracle's hits; autotuning leaves the summary untouched and
    each graph launch adds one batch to it."""
    import torch
    rng, genomes, filters = _random_case(13, n_filters=2, glen=60000)
    paths = _store(filters, tmp_path, "v")
    reads = _random_reads(rng, genomes, 1500, lmin=20, lmax=300)
    reads += _random_reads(rng, genomes, 100, lmin=300, lmax=10000, nrate=0.001)
    order = rng.permutation(len(reads))
    reads = [reads[i] for i in order]
    seq, off = ol.pack_reads(reads)
    want, _ = ol.classify(seq, off, filters, 0.15, 3)
    wc, wcat = ol.summary_counts(want, 2)
    dseq = torch.tensor(np.frombuffer(seq, dtype=np.uint8), device="cuda")
    doff = torch.tensor(off.astype(np.int64), device="cuda")
    with _classifier(paths, path=2) as bbc:
        for lb in (0, 500, 1):
            bbc.set_schedule(lb)
            hits, _, cat = bbc.classify_device(dseq, doff)
            torch.cuda.synchronize()
            assert np.array_equal(hits.cpu().numpy().view(np.uint64), want), lb
        before = bbc.summary()
        tune = bbc.autotune(dseq, doff)
        after = bbc.summary()
        assert np.array_equal(before[0], after[0]) and before[1] == after[1]
        assert tune["path"] in (1, 2, 3) and tune["reads_per_s"] > 0
        hits, _, cat = bbc.classify_device(dseq, doff)
        torch.cuda.synchronize()
        assert np.array_equal(hits.cpu().numpy().view(np.uint64), want)
    for launch in (dict(path=1), dict(path=2)):
        with _classifier(paths, **launch) as bbc:
            bbc.set_schedule(1000)
            n = len(reads)
            hits = torch.zeros((n, 1), dtype=torch.int64, device="cuda")
            cat = torch.zeros(n, dtype=torch.int32, device="cuda")
            bbc.classify_device(dseq, doff, hits=hits, category=cat)  # warm-up, same sizes
            torch.cuda.synchronize()
            bbc.reset_summary()
            hits.zero_()
            g = bbc.graph(dseq, doff, hits, category=cat, reads_per_launch=97)
            assert g.launches == (n + 96) // 97
            s = torch.cuda.Stream()
            g.launch(s)
            g.launch(s)
            s.synchronize()
            assert np.array_equal(hits.cpu().numpy().view(np.uint64), want)
            assert np.array_equal(cat.cpu().numpy(), wcat)
            counts, seen = bbc.summary()
            assert np.array_equal(counts, 2 * wc) and seen == 2 * n
            g.close()


def test_staging_splits_large_host_batches(tmp_path):
    """Host batches larger than the staging slots are split and pipelined."""
    rng, genomes, filters = _random_case(12)
    paths = []
    for i, f in enumerate(filters):
        stem = str(tmp_path / f"s{i}")
        f.store(stem + ".bf")
        ol.write_info(stem + ".txt", f"s{i}", f.k, 0.075, f.h, 1, "x", f.m, 1, 0.1, 0, 0.1)
        paths.append(stem + ".bf")
    reads = _random_reads(rng, genomes, 5000, lmin=100, lmax=200)
    seq, off = ol.pack_reads(reads)
    want, _ = ol.classify(seq, off, filters)
    with _classifier(paths, max_batch_reads=700, max_batch_bases=50000) as bbc:
        hits, _, cat = bbc.classify(reads)
        counts, reads_seen = bbc.summary()
    assert np.array_equal(hits, want)
    wc, _ = ol.summary_counts(want, 3)
    assert np.array_equal(counts, wc) and reads_seen == 5000


def test_gpu_maker_matches_oracle_maker(tmp_path):
    from biobloom_b200 import synth
    g = synth.genome(77, 300000, gc=0.41, repeat_frac=0.05, rep_min=300, rep_max=300)
    g2 = synth.genome(78, 1000, gc=0.5)
    g2[100:110] = ord("N")
    stem = str(tmp_path / "m")
    synth.make_filter([g, g2], stem, "m", k=25, fpr=0.075)
    mine = ol.Filter.load(stem + ".bf")
    ref = ol.Filter.make([g.tobytes(), g2.tobytes()], k=25, fpr=0.075)
    assert (mine.m, mine.h, mine.k) == (ref.m, ref.h, ref.k)
    assert np.array_equal(mine.bits(), ref.bits())
    info = open(stem + ".txt").read()
    assert "filter_id=m\n" in info and "kmer_size=25\n" in info
    # num_entries / redundant_sequences as a sequential insertion counts them
    valid = sum(len(ol.kmers(s.tobytes(), 1, 25)) for s in (g, g2))
    assert f"\nnum_entries={valid - ref.redundant}\n" in info
    assert f"\nredundant_sequences={ref.redundant}\n" in info


def test_gpu_maker_equals_reference_maker_files(tmp_path):
    """The reference's biobloommaker output (tests/golden/bbt/f*.bf, f*.txt,
    one single-record genome each) byte for byte: bit array, header and the
    info file's counts and rates."""
    import os
    from biobloom_b200 import synth
    from tests.golden import make_golden as mg
    rng = np.random.default_rng(20240611)
    genomes = [mg.genome(rng, 20000, gc) for gc in (0.5, 0.41, 0.6)]
    genomes[2][5000:7000] = genomes[0][1000:3000]
    gold = os.path.join(os.path.dirname(__file__), "golden", "bbt")
    for i, g in enumerate(genomes):
        want_txt = open(os.path.join(gold, f"f{i}.txt")).read()
        src = [ln for ln in want_txt.splitlines() if ln.startswith("sequence_sources=")][0]
        stem = str(tmp_path / f"f{i}")
        synth.make_filter([g], stem, f"f{i}", k=25, fpr=0.075,
                          sources=src[len("sequence_sources="):].rstrip(" "))
        assert open(stem + ".txt").read() == want_txt
        assert open(stem + ".bf", "rb").read() == open(os.path.join(gold, f"f{i}.bf"), "rb").read()


@pytest.mark.parametrize("paired", [False, True])
def test_host_batch_in_slot_loads_matches_device_batch(tmp_path, paired):
    """A host batch that fits one staging slot still goes through the slots in
    about eight loads (copies overlapping kernels); results, categories and
    summary equal one device-resident call's."""
    import torch
    rng, genomes, filters = _random_case(31)
    paths = []
    for i, f in enumerate(filters):
        stem = str(tmp_path / f"s{i}")
        f.store(stem + ".bf")
        ol.write_info(stem + ".txt", f"s{i}", f.k, 0.075, f.h, 1, "x", f.m, 1, 0.1, 0, 0.1)
        paths.append(stem + ".bf")
    n = 600_000
    g = np.concatenate(genomes)
    st = rng.integers(0, len(g) - 80, n)
    seq = g[st[:, None] + np.arange(80)[None, :]].reshape(-1).copy()
    off = np.arange(n + 1, dtype=np.uint64) * np.uint64(80)
    seq2 = None
    if paired:
        st2 = rng.integers(0, len(g) - 80, n)
        seq2 = g[st2[:, None] + np.arange(80)[None, :]].reshape(-1).copy()
    with _classifier(paths) as a:
        h, h2, c = a.classify((seq, off), (seq2, off) if paired else None)
        ca, na = a.summary()
    with _classifier(paths) as d:
        t = lambda x: torch.from_numpy(x.astype(np.int64) if x.dtype == np.uint64 else x).cuda()
        dh, dh2, dc = d.classify_device(t(seq), t(off), t(seq2) if paired else None,
                                        t(off) if paired else None)
        torch.cuda.synchronize()
        cd, nd = d.summary()
    assert np.array_equal(h, dh.cpu().numpy().view(np.uint64))
    if paired:
        assert np.array_equal(h2, dh2.cpu().numpy().view(np.uint64))
    assert np.array_equal(c, dc.cpu().numpy().view(np.uint32))
    assert na == nd == n and np.array_equal(ca, cd)
    assert h.any()


def test_filter_above_2_pow_32_bits(tmp_path):
    """A filter of m > 2^32 bits (600 MB; 89% of bit positions lie above 2^32):
    the hash reduction and the word index use 64-bit arithmetic on every path,
    including the filter-major two-pass path."""
    import torch
    rng = np.random.default_rng(4242)
    m = 4_800_000_064
    genome = bytes(rng.choice(np.frombuffer(b"ACGT", dtype=np.uint8), 30000))
    f = ol.Filter.create(m, 3, 25)
    f.insert_sequence(genome)
    bits = f.bits()
    high = np.flatnonzero(bits[(1 << 32) // 8:]).size
    assert high > 0, "no set bit above 2^32"
    stem = str(tmp_path / "big")
    f.store(stem + ".bf")
    ol.write_info(stem + ".txt", "big", 25, 0.075, 3, 30000, "x", m, 30000, 0.0, 0, 0.0)
    reads = []
    for i in range(2000):
        L = int(rng.integers(60, 400))
        if i % 2:
            s = int(rng.integers(0, len(genome) - L))
            r = bytearray(genome[s:s + L])
            for j in np.flatnonzero(rng.random(L) < 0.02):
                r[j] = ord("ACGT"[int(rng.integers(0, 4))])
            reads.append(bytes(r))
        else:
            reads.append(bytes(rng.choice(np.frombuffer(b"ACGT", dtype=np.uint8), L)))
    seq, off = ol.pack_reads(reads)
    want, _ = ol.classify(seq, off, [f], 0.15, 3)
    assert 0 < int((want[:, 0] != 0).sum()) < len(reads)
    dseq = torch.tensor(np.frombuffer(seq, dtype=np.uint8), device="cuda")
    doff = torch.tensor(off.astype(np.int64), device="cuda")
    for launch in (PATHS[0], PATHS[1], PATHS[4]):
        with _classifier([stem + ".bf"], **launch) as bbc:
            hits, _, _ = bbc.classify_device(dseq, doff)
            torch.cuda.synchronize()
            assert np.array_equal(hits.cpu().numpy().view(np.uint64), want), launch
