"""The bucketed miBF query (bbt_mibf_set_bucketing: every probe of a
sub-batch of reads sorted by ID-map address, read out of L2 bucket by bucket,
then the reads tallied from the resolved entries) gives the oracle's per-read
results, bit for bit.  Small buckets and small sub-batches force every
boundary the path has: requests across many buckets, reads across window
blocks and sub-batches, mates across blocks; spaced seeds and k-mer mode,
single and paired reads, every query option, the many-ID tally."""
import numpy as np
import pytest

from tests.test_mibf_gpu import (BASES, OPTS, _oracle_query, _opts, _reads, built,  # noqa: F401
                                 many_targets)

pytestmark = pytest.mark.gpu

DENSE = 2
SETTINGS = [dict(bucket_shift=12, max_frames=1 << 16), dict(bucket_shift=14, max_frames=0),
            dict(bucket_shift=23, max_frames=1 << 20)]
SET_IDS = ["b12-small-sub", "b14", "default-bucket"]


@pytest.fixture(scope="module", autouse=True)
def _need_gpu():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("GPU tests need a CUDA device")


def _open(path, o, settings):
    from biobloom_b200.mibf import MIBFClassifier
    mc = MIBFClassifier(path, score=o["score"], frame_matches=o["frame_matches"],
                        multi=o["multi"], min_nonsat=o["min_nonsat"], best_hit_agree=o["best"],
                        layout=DENSE)
    assert mc.layout == DENSE
    mc.set_bucketing(mode=1, **settings)
    return mc


@pytest.mark.parametrize("settings", SETTINGS, ids=SET_IDS)
@pytest.mark.parametrize("tag", ["ss", "km"])
@pytest.mark.parametrize("paired", [False, True])
@pytest.mark.parametrize("oi", range(len(OPTS)))
def test_bucketed_matches_oracle(built, tag, paired, oi, settings):  # noqa: F811
    targets, filters, _, names = built
    path, f = filters[tag]
    o = _opts(OPTS[oi])
    rng = np.random.default_rng(700 + oi + 10 * paired)
    reads, reads2 = _reads(rng, targets, 900, paired=paired)
    want = _oracle_query(f, names, reads, reads2, o)
    mc = _open(path, o, settings)
    got, sat = mc.classify(reads, reads2, max_hits=2)  # max_hits 2 exercises the retry
    for i, (res, s) in enumerate(want):
        assert (got[i], int(sat[i])) == (res, s), i
    counts, n = mc.summary()
    assert n == len(reads)
    nf = len(names) + 1
    assert counts[2 * (nf + 2) + 1] == sum(1 for r, _ in want if not r)
    assert counts[2 * (nf + 2)] == sum(1 for r, _ in want if len(r) > 1)
    mc.close()


@pytest.mark.parametrize("settings", SETTINGS[:2], ids=SET_IDS[:2])
def test_bucketed_device_batch_equals_direct_kernel(built, settings):  # noqa: F811
    """A device batch with bucketing on gives the direct kernel's results,
    saturation counts, summary and work counters."""
    import torch

    from biobloom_b200.classifier import pack
    from biobloom_b200.mibf import MIBFClassifier
    targets, filters, _, names = built
    path, _ = filters["ss"]
    rng = np.random.default_rng(77)
    reads, _ = _reads(rng, targets, 5000)
    seq, off = pack(reads)
    dseq = torch.from_numpy(seq.copy()).cuda()
    doff = torch.from_numpy(off.astype(np.int64)).cuda()
    out = []
    for mode in (0, 1):
        mc = MIBFClassifier(path, layout=DENSE)
        mc.set_bucketing(mode=mode, **settings)
        hits, nh, sat = mc.classify_device(dseq, doff, max_hits=mc.num_ids)
        mc.sync()
        out.append((hits.cpu().numpy(), nh.cpu().numpy(), sat.cpu().numpy(), mc.summary(),
                    mc.last_counts()))
        mc.close()
    (h0, n0, s0, (c0, r0), w0), (h1, n1, s1, (c1, r1), w1) = out
    assert np.array_equal(n0, n1) and np.array_equal(s0, s1)
    for i in range(len(reads)):
        assert np.array_equal(h0[i, :n0[i]], h1[i, :n1[i]]), i
    assert np.array_equal(c0, c1) and r0 == r1
    assert w0 == w1


@pytest.mark.parametrize("oi", [0, 2])
def test_bucketed_five_thousand_targets(many_targets, oi):  # noqa: F811
    """The bucketed query feeding the many-ID (global tally table) kernel."""
    targets, path, f, names = many_targets
    o = _opts(OPTS[oi])
    rng = np.random.default_rng(900 + oi)
    reads = []
    for _ in range(1500):
        t = int(rng.integers(0, len(targets)))
        st = int(rng.integers(0, 250))
        a = np.frombuffer(targets[t][st:st + 150], dtype=np.uint8).copy()
        reads.append(a.tobytes() if rng.random() < 0.9 else BASES[rng.integers(0, 4, 150)].tobytes())
    reads += [BASES[rng.integers(0, 4, 9000)].tobytes()]
    reads += [b"".join(targets[i] for i in range(40, 70))]
    want = _oracle_query(f, names, reads, None, o)
    mc = _open(path, o, SETTINGS[0])
    got, sat = mc.classify(reads, None, max_hits=4)
    for i, (res, s) in enumerate(want):
        assert (got[i], int(sat[i])) == (res, s), i
    mc.close()


@pytest.mark.parametrize("paired", [False, True])
def test_bucketed_reads_without_frames(built, paired):  # noqa: F811
    """Runs of reads shorter than k (whole sub-batch samples without a frame)
    between ordinary reads: every read gets its result and the summary counts
    them, as the direct kernel does."""
    targets, filters, _, names = built
    path, f = filters["ss"]
    o = _opts({})
    rng = np.random.default_rng(31 + paired)
    reads, reads2 = _reads(rng, targets, 1200, paired=paired)
    short = [BASES[rng.integers(0, 4, int(rng.integers(0, 20)))].tobytes() for _ in range(700)]
    reads = reads[:300] + short + reads[300:]
    if paired:
        reads2 = reads2[:300] + [s[::-1] for s in short] + reads2[300:]
    want = _oracle_query(f, names, reads, reads2, o)
    mc = _open(path, o, SETTINGS[0])
    got, sat = mc.classify(reads, reads2, max_hits=4)
    for i, (res, s) in enumerate(want):
        assert (got[i], int(sat[i])) == (res, s), i
    counts, n = mc.summary()
    assert n == len(reads)
    nf = len(names) + 1
    assert counts[2 * (nf + 2) + 1] == sum(1 for r, _ in want if not r)
    mc.close()


def test_bucketed_needs_the_dense_layout(built):  # noqa: F811
    from biobloom_b200 import _lib as L
    from biobloom_b200.mibf import MIBFClassifier
    _, filters, _, _ = built
    mc = MIBFClassifier(filters["ss"][0], layout=1)
    with pytest.raises(L.BBTError):
        mc.set_bucketing(mode=1)
    with pytest.raises(L.BBTError):
        mc.set_bucketing(mode=3)
    mc.set_bucketing(mode=0)
    mc.close()
