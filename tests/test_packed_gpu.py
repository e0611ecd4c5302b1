"""2-bit packed batches (BBT_BASES_2BIT: code words + validity bits) give the
same per-read hits as the ASCII batch and the CPU oracle, on every launch
path, for host and device buffers, single-end and paired, with N and
lower-case bases and reads that start at any base offset."""
import ctypes

import numpy as np
import pytest

from tests import oracle_lib as ol

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _need_gpu():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("GPU tests need a CUDA device")
    from biobloom_b200 import _lib
    _lib.lib()


def _case(seed, tmp_path, n_reads=1500):
    rng = np.random.default_rng(seed)
    genomes = [bytes(rng.choice(np.frombuffer(b"ACGT", dtype=np.uint8), 40000)) for _ in range(2)]
    paths, filters = [], []
    for j, g in enumerate(genomes):
        f = ol.Filter.make([g], k=25, fpr=0.1)
        stem = str(tmp_path / f"p{j}")
        f.store(stem + ".bf")
        ol.write_info(stem + ".txt", f"p{j}", 25, 0.1, f.h, 1, "x", f.m, 1, 0.1, 0, 0.1)
        paths.append(stem + ".bf")
        filters.append(f)
    reads = []
    for i in range(n_reads):
        L = int(rng.integers(10, 700))
        g = genomes[i % 2]
        if i % 3:
            s = int(rng.integers(0, len(g) - L))
            r = bytearray(g[s:s + L])
        else:
            r = bytearray(rng.choice(np.frombuffer(b"ACGT", dtype=np.uint8), L))
        for j in np.flatnonzero(rng.random(L) < 0.01):
            r[j] = ord("N")
        for j in np.flatnonzero(rng.random(L) < 0.05):
            r[j] = r[j] | 0x20  # lower case
        reads.append(bytes(r))
    return paths, filters, reads


def _pack(seq):
    from biobloom_b200 import _lib as L
    n = len(seq)
    words = np.zeros((n + 15) // 16 + 1, dtype=np.uint32)
    valid = np.zeros((n + 31) // 32 + 1, dtype=np.uint32)
    bad = ctypes.c_uint64()
    buf = np.frombuffer(seq, dtype=np.uint8)
    L.check(L.lib().bbt_pack_bases(buf.ctypes.data, n, words.ctypes.data, valid.ctypes.data,
                                   ctypes.byref(bad)))
    return words, valid, bad.value


def test_pack_bases_layout():
    seq = b"ACGTacgtNNxT" * 7 + b"G"
    words, valid, bad = _pack(seq)
    for g, c in enumerate(seq):
        code = (int(words[g // 16]) >> (2 * (g % 16))) & 3
        ok = (int(valid[g // 32]) >> (g % 32)) & 1
        assert ok == (chr(c) in "ACGTacgt")
        if ok:
            assert code == "ACGT".index(chr(c).upper())
    assert bad == sum(1 for c in seq if chr(c) not in "ACGTacgt")


@pytest.mark.parametrize("launch", [dict(path=1), dict(path=2), dict(path=3),
                                    dict(path=2, frames_per_lane=8)],
                         ids=["plain", "persistent", "filter-major", "persistent-seg8"])
@pytest.mark.parametrize("where", ["device", "host"])
def test_packed_single_matches_ascii_and_oracle(tmp_path, launch, where):
    import torch
    from biobloom_b200 import BioBloomClassifier
    from biobloom_b200 import _lib as L
    paths, filters, reads = _case(31, tmp_path)
    seq, off = ol.pack_reads(reads)
    want, _ = ol.classify(seq, off, filters, 0.15, 3)
    words, valid, _ = _pack(seq)
    n = len(reads)
    with BioBloomClassifier(paths, 0.15, max_batch_reads=400, max_batch_bases=70000,
                            **launch) as bbc:
        ascii_hits, _, _ = bbc.classify(reads)
        assert np.array_equal(ascii_hits, want)
        b = L.Batch()
        r = L.Result()
        if where == "device":
            dw = torch.tensor(words.view(np.int32), device="cuda")
            dv = torch.tensor(valid.view(np.int32), device="cuda")
            do = torch.tensor(off.astype(np.int64), device="cuda")
            hits = torch.zeros((n, 1), dtype=torch.int64, device="cuda")
            b.seq, b.offsets, b.valid = dw.data_ptr(), do.data_ptr(), dv.data_ptr()
            b.location = r.location = L.DEVICE
            r.hits = hits.data_ptr()
        else:
            hits_np = np.zeros((n, 1), dtype=np.uint64)
            b.seq, b.offsets, b.valid = words.ctypes.data, off.ctypes.data, valid.ctypes.data
            b.location = r.location = L.HOST
            r.hits = hits_np.ctypes.data
        b.n_reads, b.encoding = n, L.BASES_2BIT
        L.check(L.lib().bbt_classify_batch(bbc._ctx, ctypes.byref(b), ctypes.byref(r), None),
                bbc._ctx)
        L.check(L.lib().bbt_sync(bbc._ctx), bbc._ctx)
        got = hits.cpu().numpy().view(np.uint64) if where == "device" else hits_np
        assert np.array_equal(got, want)


@pytest.mark.parametrize("where", ["device", "host"])
def test_packed_pairs_and_offset_start(tmp_path, where):
    """Pairs, and a batch whose offsets[0] is not on a word boundary."""
    import torch
    from biobloom_b200 import BioBloomClassifier
    from biobloom_b200 import _lib as L
    paths, filters, reads = _case(32, tmp_path, 1201)
    r1, r2 = reads[1:601], reads[601:1201]
    seq1, off1 = ol.pack_reads([reads[0]] + r1)
    seq2, off2 = ol.pack_reads([reads[0]] + r2)
    w1, _ = ol.classify(seq1, off1, filters, 0.15, 3)
    w2, _ = ol.classify(seq2, off2, filters, 0.15, 3)
    w1, w2 = w1[1:], w2[1:]
    pk1, v1, _ = _pack(seq1)
    pk2, v2, _ = _pack(seq2)
    o1 = np.ascontiguousarray(off1[1:])
    o2 = np.ascontiguousarray(off2[1:])
    n = len(r1)
    with BioBloomClassifier(paths, 0.15, max_batch_reads=250, max_batch_bases=90000) as bbc:
        b = L.Batch()
        r = L.Result()
        keep = []
        if where == "device":
            t = [torch.tensor(x.view(np.int32), device="cuda") for x in (pk1, v1, pk2, v2)]
            to = [torch.tensor(x.astype(np.int64), device="cuda") for x in (o1, o2)]
            h1 = torch.zeros((n, 1), dtype=torch.int64, device="cuda")
            h2 = torch.zeros((n, 1), dtype=torch.int64, device="cuda")
            keep += t + to
            b.seq, b.valid, b.seq2, b.valid2 = (x.data_ptr() for x in t)
            b.offsets, b.offsets2 = to[0].data_ptr(), to[1].data_ptr()
            r.hits, r.hits2 = h1.data_ptr(), h2.data_ptr()
            b.location = r.location = L.DEVICE
        else:
            h1n = np.zeros((n, 1), dtype=np.uint64)
            h2n = np.zeros((n, 1), dtype=np.uint64)
            b.seq, b.valid, b.seq2, b.valid2 = (x.ctypes.data for x in (pk1, v1, pk2, v2))
            b.offsets, b.offsets2 = o1.ctypes.data, o2.ctypes.data
            r.hits, r.hits2 = h1n.ctypes.data, h2n.ctypes.data
            b.location = r.location = L.HOST
        b.n_reads, b.encoding = n, L.BASES_2BIT
        L.check(L.lib().bbt_classify_batch(bbc._ctx, ctypes.byref(b), ctypes.byref(r), None),
                bbc._ctx)
        L.check(L.lib().bbt_sync(bbc._ctx), bbc._ctx)
        if where == "device":
            g1, g2 = h1.cpu().numpy().view(np.uint64), h2.cpu().numpy().view(np.uint64)
        else:
            g1, g2 = h1n, h2n
        assert np.array_equal(g1, w1) and np.array_equal(g2, w2)
