"""The bucketed probe path (BBT_PATH_BUCKETED: probes sorted by filter
address, resolved bucket by bucket in rounds, SeqEval walked over the resolved
bits) gives the CPU oracle's hits bit for bit.  Small buckets, small
sub-batches and several phase layouts force every boundary the path has:
requests across many buckets, reads across window blocks and sub-batches,
reads decided in either phase, and reads too long for any sub-batch (the
direct kernel's)."""
import ctypes

import numpy as np
import pytest

from tests import oracle_lib as ol
from tests.test_gpu_parity import _classifier, _random_case, _random_reads, _store

pytestmark = pytest.mark.gpu

SETTINGS = [dict(bucket_shift=12, phase_split=8, phase_min=64, max_frames=40000),
            dict(bucket_shift=14, phase_split=16, phase_min=1, max_frames=1 << 20),
            dict(bucket_shift=12, phase_split=3, phase_min=1, max_frames=33000,
                 levels_per_round=1),
            dict(bucket_shift=28, phase_split=8, phase_min=64, max_frames=0)]
SET_IDS = ["b12-half", "b14-one-phase", "b12-3of16", "default"]


@pytest.fixture(scope="module", autouse=True)
def _need_gpu():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("GPU tests need a CUDA device")
    from biobloom_b200 import _lib
    _lib.lib()


def _bucketed(paths, settings, score=0.15, streak=3, **kw):
    bbc = _classifier(paths, score, streak, path=4, **kw)
    bbc.set_bucketing(**settings)
    return bbc


@pytest.mark.parametrize("settings", SETTINGS, ids=SET_IDS)
@pytest.mark.parametrize("seed,k,h,score,streak", [
    (1, 25, 0, 0.15, 3), (2, 21, 2, 0.3, 2), (3, 31, 4, 0.05, 1), (4, 17, 1, 0.9, 5),
    (5, 25, 3, 0.0, 3), (6, 25, 3, 1.0, 3), (7, 12, 3, 0.4, 0), (8, 64, 3, 0.15, 3)])
def test_random_parity(seed, k, h, score, streak, settings, tmp_path):
    rng, genomes, filters = _random_case(seed, k=k, h=h, fpr=0.2)
    paths = _store(filters, tmp_path, "b")
    reads = _random_reads(rng, genomes, 3000)
    seq, off = ol.pack_reads(reads)
    want, _ = ol.classify(seq, off, filters, score, streak)
    with _bucketed(paths, settings, score, streak) as bbc:
        hits, _, cat = bbc.classify(reads)
    assert np.array_equal(hits, want)
    _, cats = ol.summary_counts(want, len(filters))
    assert np.array_equal(cat, cats)


@pytest.mark.parametrize("settings", SETTINGS[:3], ids=SET_IDS[:3])
def test_long_reads_and_device_batches(settings, tmp_path):
    import torch
    rng, genomes, filters = _random_case(11, n_filters=2, glen=60000)
    paths = _store(filters, tmp_path, "l")
    reads = _random_reads(rng, genomes, 400, lmin=20, lmax=12000, nrate=0.001, sub=0.005)
    seq, off = ol.pack_reads(reads)
    want, _ = ol.classify(seq, off, filters, 0.15, 3)
    dseq = torch.tensor(np.frombuffer(seq, dtype=np.uint8), device="cuda")
    doff = torch.tensor(off.astype(np.int64), device="cuda")
    with _bucketed(paths, settings) as bbc:
        hits, _, _ = bbc.classify_device(dseq, doff)
        torch.cuda.synchronize()
        assert np.array_equal(hits.cpu().numpy().view(np.uint64), want)


def test_read_longer_than_a_sub_batch(tmp_path):
    """max_frames at its minimum (32768 frames): reads of 40 kb have no
    sub-batch and go to the direct kernel; the others stay bucketed."""
    rng, genomes, filters = _random_case(21, n_filters=2, glen=120000)
    paths = _store(filters, tmp_path, "o")
    reads = _random_reads(rng, genomes, 300, lmin=30, lmax=3000)
    g = genomes[0].tobytes()
    reads[17] = g[1000:41000]
    reads[150] = bytes(rng.choice(np.frombuffer(b"ACGT", dtype=np.uint8), 50000))
    seq, off = ol.pack_reads(reads)
    want, _ = ol.classify(seq, off, filters, 0.15, 3)
    with _bucketed(paths, dict(bucket_shift=12, phase_split=8, phase_min=64,
                               max_frames=32768)) as bbc:
        hits, _, _ = bbc.classify(reads)
    assert np.array_equal(hits, want)
    assert int(want[17, 0]) & 1


@pytest.mark.parametrize("incl", [False, True])
@pytest.mark.parametrize("ordered", [False, True])
def test_pairs_inclusive_and_ordered(tmp_path, incl, ordered):
    rng, genomes, filters = _random_case(31, n_filters=3, glen=40000)
    paths = _store(filters, tmp_path, "p")
    r1 = _random_reads(rng, genomes, 1500, lmin=60, lmax=300)
    r2 = _random_reads(rng, genomes, 1500, lmin=60, lmax=300)
    s1, o1 = ol.pack_reads(r1)
    s2, o2 = ol.pack_reads(r2)
    w1, _ = ol.classify(s1, o1, filters, 0.15, 3)
    w2, _ = ol.classify(s2, o2, filters, 0.15, 3)
    if ordered:
        w1, w2 = ol.ordered(w1, 3, w2, incl)
    counts, cats = ol.summary_counts(w1, 3, w2, incl)
    with _bucketed(paths, SETTINGS[0]) as bbc:
        if incl:
            bbc.setInclusive()
        if ordered:
            bbc.setOrderedFilter()
        h1, h2, cat = bbc.classify(r1, r2)
        got_counts, seen = bbc.summary()
    assert np.array_equal(h1, w1) and np.array_equal(h2, w2)
    assert np.array_equal(cat, cats)
    assert np.array_equal(got_counts, counts) and seen == 1500


@pytest.mark.parametrize("score_type,score,scoring", [
    ("simple", 40, ol.LENGTH), ("harmonic", 0.15, ol.HARMONIC), ("binomial", 100, ol.BINOMIAL)])
def test_scoring_methods(tmp_path, score_type, score, scoring):
    from biobloom_b200 import BioBloomClassifier
    rng, genomes, filters = _random_case(41, n_filters=2, glen=40000)
    paths = _store(filters, tmp_path, "s")
    reads = _random_reads(rng, genomes, 2500, lmin=20, lmax=2000)
    seq, off = ol.pack_reads(reads)
    with BioBloomClassifier(paths, score, score_type=score_type) as ref:
        want, _, _ = ref.classify(reads)  # the read-major path, itself tested against goldens
    with BioBloomClassifier(paths, score, score_type=score_type, path=4) as bbc:
        bbc.set_bucketing(**SETTINGS[0])
        hits, _, _ = bbc.classify(reads)
    assert np.array_equal(hits, want)
    if scoring == ol.LENGTH:
        w, _ = ol.classify(seq, off, filters, 40, 3, scoring=ol.LENGTH)
        assert np.array_equal(hits, w)


def test_dust_masking(tmp_path):
    rng, genomes, filters = _random_case(51, n_filters=2, glen=40000)
    paths = _store(filters, tmp_path, "d")
    reads = _random_reads(rng, genomes, 1500, lmin=60, lmax=600)
    for i in range(0, len(reads), 7):
        r = bytearray(reads[i])
        r[10:70] = b"AT" * 30 if len(r) > 80 else r[10:70]
        reads[i] = bytes(r)
    seq, off = ol.pack_reads(reads)
    with ol.dust(20, 64):
        want, _ = ol.classify(seq, off, filters, 0.15, 3)
    with _bucketed(paths, SETTINGS[0]) as bbc:
        bbc.set_dust(True, 20, 64)
        hits, _, _ = bbc.classify(reads)
    assert np.array_equal(hits, want)


def test_packed_batch(tmp_path):
    import torch
    from biobloom_b200 import _lib as L
    rng, genomes, filters = _random_case(61, n_filters=2, glen=40000)
    paths = _store(filters, tmp_path, "k")
    reads = _random_reads(rng, genomes, 2000, lmin=20, lmax=900)
    seq, off = ol.pack_reads(reads)
    want, _ = ol.classify(seq, off, filters, 0.15, 3)
    n = len(seq)
    words = np.zeros((n + 15) // 16 + 1, dtype=np.uint32)
    valid = np.zeros((n + 31) // 32 + 1, dtype=np.uint32)
    buf = np.frombuffer(seq, dtype=np.uint8)
    L.check(L.lib().bbt_pack_bases(buf.ctypes.data, n, words.ctypes.data, valid.ctypes.data,
                                   None))
    dw = torch.tensor(words.view(np.int32), device="cuda")
    dv = torch.tensor(valid.view(np.int32), device="cuda")
    do = torch.tensor(off.astype(np.int64), device="cuda")
    hits = torch.zeros((len(reads), 1), dtype=torch.int64, device="cuda")
    with _bucketed(paths, SETTINGS[0]) as bbc:
        b = L.Batch()
        b.seq, b.offsets, b.valid, b.n_reads = dw.data_ptr(), do.data_ptr(), dv.data_ptr(), len(reads)
        b.location, b.encoding = L.DEVICE, L.BASES_2BIT
        r = L.Result()
        r.hits, r.location = hits.data_ptr(), L.DEVICE
        L.check(L.lib().bbt_classify_batch(bbc._ctx, ctypes.byref(b), ctypes.byref(r), None),
                bbc._ctx)
        L.check(L.lib().bbt_sync(bbc._ctx), bbc._ctx)
    assert np.array_equal(hits.cpu().numpy().view(np.uint64), want)
