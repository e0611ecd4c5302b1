"""bbt_open_devices: the filters on several devices, host batches split into
contiguous shards of reads (one per device) and classified concurrently,
results in batch order, summary counters added up.  One GPU is enough to
check it: the same device listed twice gives two contexts that each take a
shard.  Hits, categories, summaries and the file pipeline's summary.tsv must
equal the single-device ones (and the reference CLI's for the fixtures)."""
import os
import subprocess
import tempfile

import numpy as np
import pytest

from tests import oracle_lib as ol
from tests.fixtures import filter_paths, golden, read_fastx

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module", autouse=True)
def _need_gpu():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("GPU tests need a CUDA device")
    from biobloom_b200 import _lib
    _lib.lib()


@pytest.mark.parametrize("devices", [[0, 0], [0, 0, 0]])
def test_split_batches_equal_one_device(devices):
    from biobloom_b200 import BioBloomClassifier
    r1 = [s for _, s in read_fastx(golden("reads_1.fq.gz"))]
    r2 = [s for _, s in read_fastx(golden("reads_2.fq.gz"))]
    with BioBloomClassifier(filter_paths(), 0.15) as one:
        w1, w2, wc = one.classify(r1, r2)
        wcounts, wseen = one.summary()
        wtsv = one.summary_tsv()
    with BioBloomClassifier(filter_paths(), 0.15, devices=devices) as many:
        h1, h2, cat = many.classify(r1, r2)
        counts, seen = many.summary()
        assert many.summary_tsv() == wtsv
        many.setInclusive()
        many.reset_summary()
        many.classify(r1, r2)
        _, seen2 = many.summary()
    assert np.array_equal(h1, w1) and np.array_equal(h2, w2) and np.array_equal(cat, wc)
    assert np.array_equal(counts, wcounts) and seen == wseen == seen2


def test_file_pipeline_and_cli_on_two_contexts():
    from biobloom_b200 import BioBloomClassifier
    with tempfile.TemporaryDirectory() as tmp:
        prefix = os.path.join(tmp, "pe")
        with BioBloomClassifier(filter_paths(), 0.15, prefix=prefix, devices=[0, 0]) as bbc:
            bbc.filterPair(golden("reads_1.fq.gz"), golden("reads_2.fq.gz"))
        with open(prefix + "_summary.tsv") as f, open(golden("expected_summary_pe.tsv")) as g:
            assert f.read() == g.read()
        cli = os.path.join(ROOT, "biobloom_b200", "bin", "biobloomcategorizer")
        p = subprocess.run([cli, "--devices=0,0", "-p", os.path.join(tmp, "se"), "-f",
                            " ".join(filter_paths()), golden("reads_se.fa.gz")],
                           capture_output=True, text=True)
        assert p.returncode == 0, p.stderr
        with open(os.path.join(tmp, "se_summary.tsv")) as f, \
                open(golden("expected_summary_se.tsv")) as g:
            assert f.read() == g.read()


def test_scoring_and_packed_batches_split(tmp_path):
    import ctypes
    from biobloom_b200 import BioBloomClassifier
    from biobloom_b200 import _lib as L
    from tests.test_gpu_parity import _random_case, _random_reads, _store
    rng, genomes, filters = _random_case(71, n_filters=3, glen=40000)
    paths = _store(filters, tmp_path, "m")
    reads = _random_reads(rng, genomes, 3001, lmin=20, lmax=800)
    seq, off = ol.pack_reads(reads)
    want, _ = ol.classify(seq, off, filters, 0.15, 3)
    with BioBloomClassifier(paths, 0.15) as one:
        _, _, _, wscores, _ = one.classify(reads, scores=True)
    n = len(seq)
    words = np.zeros((n + 15) // 16 + 1, dtype=np.uint32)
    valid = np.zeros((n + 31) // 32 + 1, dtype=np.uint32)
    buf = np.frombuffer(seq, dtype=np.uint8)
    L.check(L.lib().bbt_pack_bases(buf.ctypes.data, n, words.ctypes.data, valid.ctypes.data,
                                   None))
    with BioBloomClassifier(paths, 0.15, devices=[0, 0]) as bbc:
        _, _, _, scores, _ = bbc.classify(reads, scores=True)
        assert np.array_equal(scores.view(np.uint64), wscores.view(np.uint64))
        hits = np.zeros((len(reads), 1), dtype=np.uint64)
        b = L.Batch()
        b.seq, b.offsets, b.valid, b.n_reads = (words.ctypes.data, off.ctypes.data,
                                                valid.ctypes.data, len(reads))
        b.location, b.encoding = L.HOST, L.BASES_2BIT
        r = L.Result()
        r.hits, r.location = hits.ctypes.data, L.HOST
        L.check(L.lib().bbt_classify_batch(bbc._ctx, ctypes.byref(b), ctypes.byref(r), None),
                bbc._ctx)
    assert np.array_equal(hits, want)
