"""bbt_classify_noalloc, the entry point for callers that cannot call
cudaMalloc (their device memory is owned by another allocator or a fixed
pool, or cudaMalloc's device-wide synchronization is not acceptable where they
run): through the C ABI it must give exactly the hits of the ordinary entry
point, bbt_classify_batch, on two calls in a row (the second call finds the
first call's contents in the shared scratch array), and reject more filters
than its stated maximum.

This file is collected last so that a run stopping at the first failure has
run every other test first; it passes alone in a fresh process as well."""
import ctypes

import numpy as np
import pytest

from tests import oracle_lib as ol
from tests.fixtures import filter_paths, golden, read_fastx

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def setup():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("this test needs a CUDA device")
    from biobloom_b200 import _lib as L
    L.lib()  # no fallback: raises if the library is missing
    # filters uploaded by the caller (the test allocates; the entry point does not)
    filters = [ol.Filter.load(p) for p in filter_paths()]
    dev_words = [torch.tensor(f.bits(), device="cuda") for f in filters]
    views = (L.FilterView * len(filters))()
    for v, f, w in zip(views, filters, dev_words):
        v.words, v.m, v.h, v.k = w.data_ptr(), f.m, f.h, f.k
    r1 = [s for _, s in read_fastx(golden("reads_1.fq.gz"))]
    r2 = [s for _, s in read_fastx(golden("reads_2.fq.gz"))]
    rng = np.random.default_rng(5)
    extra = [rng.choice(np.frombuffer(b"ACGTN", dtype=np.uint8), int(n)).tobytes()
             for n in rng.integers(0, 3000, 64)]
    return L, torch, filters, dev_words, views, r1 + extra, r2 + extra


def _to_device(torch, reads):
    seq, off = ol.pack_reads(reads)
    return (torch.tensor(np.frombuffer(seq or b"\0", dtype=np.uint8), device="cuda"),
            torch.tensor(off.astype(np.int64), device="cuda"))


def _noalloc(L, torch, views, nf, seq, off, seq2=None, off2=None, score=0.15, scoring=0):
    n = off.numel() - 1
    words = (nf + 63) // 64
    hits = torch.full((n, words), -1, dtype=torch.int64, device="cuda")
    hits2 = torch.full((n, words), -1, dtype=torch.int64, device="cuda") if seq2 is not None \
        else None
    p = L.Params()
    L.lib().bbt_default_params(ctypes.byref(p))
    p.score = score
    p.scoring = scoring
    b = L.Batch()
    b.seq, b.offsets, b.n_reads, b.location = seq.data_ptr(), off.data_ptr(), n, L.DEVICE
    if seq2 is not None:
        b.seq2, b.offsets2 = seq2.data_ptr(), off2.data_ptr()
    stream = torch.cuda.current_stream()
    rc = L.lib().bbt_classify_noalloc(views, nf, ctypes.byref(p), ctypes.byref(b),
                                      ctypes.c_void_p(hits.data_ptr()),
                                      ctypes.c_void_p(hits2.data_ptr() if hits2 is not None
                                                      else 0),
                                      ctypes.c_void_p(stream.cuda_stream))
    L.check(rc)
    torch.cuda.synchronize()
    return hits, hits2


def test_noalloc_matches_classify_batch_twice(setup):
    L, torch, filters, dev_words, views, r1, r2 = setup
    from biobloom_b200 import BioBloomClassifier
    s1, o1 = _to_device(torch, r1)
    s2, o2 = _to_device(torch, r2)
    with BioBloomClassifier(filter_paths(), 0.15) as bbc:
        want1, want2, _ = bbc.classify_device(s1, o1, s2, o2)
        wse, _, _ = bbc.classify_device(s1, o1)
        torch.cuda.synchronize()
    for _ in range(2):  # two calls in a row share the scratch array
        h1, h2 = _noalloc(L, torch, views, len(filters), s1, o1, s2, o2)
        assert torch.equal(h1, want1) and torch.equal(h2, want2)
        hse, _ = _noalloc(L, torch, views, len(filters), s1, o1)
        assert torch.equal(hse, wse)


def test_noalloc_rejects_too_many_filters(setup):
    L, torch, filters, dev_words, views, r1, r2 = setup
    many = (L.FilterView * 65)()
    for i in range(65):
        many[i] = views[i % len(filters)]
    s1, o1 = _to_device(torch, r1[:4])
    p = L.Params()
    L.lib().bbt_default_params(ctypes.byref(p))
    b = L.Batch()
    b.seq, b.offsets, b.n_reads, b.location = s1.data_ptr(), o1.data_ptr(), 4, L.DEVICE
    hits = torch.zeros((4, 2), dtype=torch.int64, device="cuda")
    rc = L.lib().bbt_classify_noalloc(many, 65, ctypes.byref(p), ctypes.byref(b),
                                      ctypes.c_void_p(hits.data_ptr()), None, None)
    assert rc == -1
    assert b"at most" in L.lib().bbt_last_error(None) or b"between 1 and 64" in \
        L.lib().bbt_last_error(None)


def test_noalloc_integer_harmonic_score_is_a_match_length(setup):
    """As the ordinary entry point does (BioBloomCategorizer.cpp:423-430 reads
    an integer score > 1 as a minimum match length, whatever -S says), a
    harmonic score of 40 classifies by LENGTH; scores of 2^32 and more are
    refused before any conversion."""
    L, torch, filters, dev_words, views, r1, r2 = setup
    from biobloom_b200 import BioBloomClassifier
    s1, o1 = _to_device(torch, r1)
    with BioBloomClassifier(filter_paths(), 40, score_type="harmonic") as bbc:
        want, _, _ = bbc.classify_device(s1, o1)
        torch.cuda.synchronize()
    for _ in range(2):
        got, _ = _noalloc(L, torch, views, len(filters), s1, o1, score=40, scoring=2)
        assert torch.equal(got, want)
    with pytest.raises(Exception):
        _noalloc(L, torch, views, len(filters), s1, o1, score=2.0 ** 32, scoring=2)
