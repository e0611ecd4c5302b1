"""Edge cases at the batch boundary, against the CPU oracle: an empty batch,
reads of length 0, k - 1, k and k + 1, reads of N only, reads in which every
k-mer holds an N (no frame is evaluated), lower-case bases, and mates of
different lengths (one of them empty).  The reference gives a read with no
evaluable frame no hit (SeqEval::evalRead over an ntHashIterator that yields
nothing, Common/SeqEval.h), and counts it as no match in the summary
(ResultsManager::updateSummaryData)."""
import numpy as np
import pytest

from tests import oracle_lib as ol

pytestmark = pytest.mark.gpu

K = 25
LAUNCHES = [dict(path=1), dict(path=2), dict(path=2, steps=1), dict(path=3)]
LAUNCH_IDS = ["plain", "persistent", "persistent-full-steps", "filter-major"]


@pytest.fixture(scope="module", autouse=True)
def _need_gpu():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("GPU tests need a CUDA device")
    from biobloom_b200 import _lib
    _lib.lib()  # raises if the library is missing: no fallback


def _case(tmp_path):
    rng = np.random.default_rng(77)
    genomes = [rng.choice(np.frombuffer(b"ACGT", dtype=np.uint8), 20000) for _ in range(2)]
    filters = [ol.Filter.make([g.tobytes()], k=K, fpr=0.075) for g in genomes]
    paths = []
    for i, f in enumerate(filters):
        stem = str(tmp_path / f"e{i}")
        f.store(stem + ".bf")
        ol.write_info(stem + ".txt", f"e{i}", f.k, 0.075, f.h, 1, "x", f.m, 1, 0.1, 0, 0.1)
        paths.append(stem + ".bf")
    g0 = genomes[0].tobytes()
    n_every = bytearray(g0[100:400])
    n_every[::K - 1] = b"N" * len(n_every[::K - 1])   # every k-mer holds an N
    reads = [
        b"",                                 # no bases
        g0[0:K - 1],                         # one base short of a k-mer
        g0[1000:1000 + K],                   # exactly one frame, in the filter
        g0[2000:2000 + K + 1],               # two frames
        b"N" * 50,                           # no valid base
        bytes(n_every),                      # bases, but no valid frame
        g0[3000:3150].lower(),               # lower-case bases
        genomes[1].tobytes()[500:650],       # the other filter
        rng.choice(np.frombuffer(b"ACGT", dtype=np.uint8), 150).tobytes(),  # random
        g0[5000:5000 + 3000],                # several hash windows
    ]
    return filters, paths, reads


def _classifier(paths, **kw):
    from biobloom_b200 import BioBloomClassifier
    return BioBloomClassifier(paths, 0.15, streak_threshold=3, **kw)


@pytest.mark.parametrize("launch", LAUNCHES, ids=LAUNCH_IDS)
def test_edge_reads_match_oracle(launch, tmp_path):
    import torch
    filters, paths, reads = _case(tmp_path)
    seq, off = ol.pack_reads(reads)
    want, _ = ol.classify(seq, off, filters, 0.15, 3)
    counts, cats = ol.summary_counts(want, len(filters))
    assert want[:2].sum() == 0 and want[4:6].sum() == 0   # no evaluable frame: no hit
    assert (want[2, 0] & 1) and (want[3, 0] & 1) and (want[6, 0] & 1)
    with _classifier(paths, **launch) as bbc:
        hits, _, cat = bbc.classify(reads)
        assert np.array_equal(hits, want)
        assert np.array_equal(cat, cats)
        got_counts, n = bbc.summary()
        assert n == len(reads)
        assert np.array_equal(got_counts[:len(counts)], counts)
        dseq = torch.tensor(np.frombuffer(seq, dtype=np.uint8), device="cuda")
        doff = torch.tensor(off.astype(np.int64), device="cuda")
        dh, _, dc = bbc.classify_device(dseq, doff)
        torch.cuda.synchronize()
        assert np.array_equal(dh.cpu().numpy().view(np.uint64), want)
        assert np.array_equal(dc.cpu().numpy().astype(np.uint32), cats)


def test_empty_batch_is_a_no_op(tmp_path):
    import torch
    _, paths, _ = _case(tmp_path)
    with _classifier(paths) as bbc:
        hits, _, cat = bbc.classify([])
        assert hits.shape[0] == 0 and cat.shape[0] == 0
        dseq = torch.zeros(16, dtype=torch.uint8, device="cuda")
        doff = torch.zeros(1, dtype=torch.int64, device="cuda")
        dh, _, dc = bbc.classify_device(dseq, doff)
        torch.cuda.synchronize()
        assert dh.shape[0] == 0 and dc.shape[0] == 0
        counts, n = bbc.summary()
        assert n == 0 and not counts.any()


@pytest.mark.parametrize("launch", LAUNCHES[:2], ids=LAUNCH_IDS[:2])
def test_mates_of_different_lengths(launch, tmp_path):
    filters, paths, reads = _case(tmp_path)
    mates = list(reversed(reads))          # pairs an empty read with a long one, and so on
    seq1, off1 = ol.pack_reads(reads)
    seq2, off2 = ol.pack_reads(mates)
    w1, _ = ol.classify(seq1, off1, filters, 0.15, 3)
    w2, _ = ol.classify(seq2, off2, filters, 0.15, 3)
    counts, cats = ol.summary_counts(w1, len(filters), w2)
    with _classifier(paths, **launch) as bbc:
        h1, h2, cat = bbc.classify(reads, mates)
        assert np.array_equal(h1, w1) and np.array_equal(h2, w2)
        assert np.array_equal(cat, cats)
        got_counts, n = bbc.summary()
        assert np.array_equal(got_counts[:len(counts)], counts)
