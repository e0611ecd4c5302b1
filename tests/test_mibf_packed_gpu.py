"""2-bit packed batches (bbt_batch BBT_BASES_2BIT: code words + validity bits)
through the miBF query give the same per-read results and summary as the
ASCII batch: host batches (through the chunk slots, chunks starting at any
base) and device batches, single-end and paired, with N runs and lower case,
with and without validity bits, on the direct kernel and the bucketed
query."""
import ctypes

import numpy as np
import pytest

from tests.test_mibf_gpu import _reads, built  # noqa: F401

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _need_gpu():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("GPU tests need a CUDA device")


def _concat(reads):
    off = np.zeros(len(reads) + 1, dtype=np.uint64)
    off[1:] = np.cumsum([len(r) for r in reads])
    return np.frombuffer(b"".join(reads), dtype=np.uint8).copy(), off


def _pack(seq):
    from biobloom_b200 import _lib as L
    n = len(seq)
    words = np.zeros((n + 15) // 16 + 1, dtype=np.uint32)
    valid = np.zeros((n + 31) // 32 + 1, dtype=np.uint32)
    bad = ctypes.c_uint64()
    L.check(L.lib().bbt_pack_bases(seq.ctypes.data, n, words.ctypes.data, valid.ctypes.data,
                                   ctypes.byref(bad)))
    return words, valid, bad.value


def _mutate(rng, reads):
    out = []
    for r in reads:
        a = bytearray(r)
        for j in np.flatnonzero(rng.random(len(a)) < 0.01):
            a[j] = ord("N")
        for j in np.flatnonzero(rng.random(len(a)) < 0.05):
            a[j] = a[j] | 0x20
        out.append(bytes(a))
    return out


def _run_host(mc, seq, off, seq2=None, off2=None, packed=False, with_valid=True, max_hits=64):
    from biobloom_b200 import _lib as L
    n = len(off) - 1
    keep = []
    b = L.Batch()
    if packed:
        w, v, _ = _pack(seq)
        keep += [w, v]
        b.seq, b.encoding = w.ctypes.data, L.BASES_2BIT
        b.valid = v.ctypes.data if with_valid else None
    else:
        b.seq = seq.ctypes.data
    b.offsets, b.n_reads, b.location = off.ctypes.data, n, L.HOST
    if seq2 is not None:
        if packed:
            w2, v2, _ = _pack(seq2)
            keep += [w2, v2]
            b.seq2 = w2.ctypes.data
            b.valid2 = v2.ctypes.data if with_valid else None
        else:
            b.seq2 = seq2.ctypes.data
        b.offsets2 = off2.ctypes.data
    hits = np.zeros((n, max_hits, 7), dtype=np.uint32)
    nh = np.zeros(n, dtype=np.uint32)
    sat = np.zeros(n, dtype=np.uint32)
    r = L.MibfResult()
    r.hits, r.max_hits, r.n_hits, r.sat_count, r.location = (
        hits.ctypes.data, max_hits, nh.ctypes.data, sat.ctypes.data, L.HOST)
    L.check_mibf(L.lib().bbt_mibf_classify_batch(mc._ctx, ctypes.byref(b), ctypes.byref(r),
                                                 None), mc._ctx)
    return [hits[i, :nh[i]].tolist() for i in range(n)], sat, mc.summary()


@pytest.mark.parametrize("bucketed", [0, 1])
@pytest.mark.parametrize("paired", [False, True])
@pytest.mark.parametrize("tag", ["ss", "km"])
def test_packed_host_batch_equals_ascii(built, tag, paired, bucketed):  # noqa: F811
    from biobloom_b200.mibf import MIBFClassifier
    targets, filters, _, names = built
    path, _ = filters[tag]
    rng = np.random.default_rng(50 + paired + 2 * bucketed)
    reads, reads2 = _reads(rng, targets, 1500, paired=paired)
    reads = _mutate(rng, reads)
    seq, off = _concat(reads)
    seq2 = off2 = None
    if paired:
        seq2, off2 = _concat(_mutate(rng, reads2))
    got = []
    for packed in (False, True):
        mc = MIBFClassifier(path, layout=2)
        mc.set_bucketing(mode=bucketed, bucket_shift=12, max_frames=1 << 16)
        got.append(_run_host(mc, seq, off, seq2, off2, packed=packed))
        mc.close()
    (h0, s0, (c0, n0)), (h1, s1, (c1, n1)) = got
    assert h0 == h1
    assert np.array_equal(s0, s1)
    assert np.array_equal(c0, c1) and n0 == n1


def test_packed_host_batch_without_validity_bits(built):  # noqa: F811
    """A batch of ACGT-only reads may pass valid = NULL."""
    from biobloom_b200.mibf import MIBFClassifier
    targets, filters, _, names = built
    path, _ = filters["ss"]
    rng = np.random.default_rng(61)
    reads, _ = _reads(rng, targets, 800)
    reads = [bytes(b"ACGT"[c] for c in rng.integers(0, 4, len(r))) if i % 5 == 0 else
             bytes(c if c in b"ACGT" else ord("A") for c in r.upper())
             for i, r in enumerate(reads)]
    seq, off = _concat(reads)
    mc = MIBFClassifier(path, layout=2)
    h0, s0, _ = _run_host(mc, seq, off)
    h1, s1, _ = _run_host(mc, seq, off, packed=True, with_valid=False)
    mc.close()
    assert h0 == h1 and np.array_equal(s0, s1)


@pytest.mark.parametrize("bucketed", [0, 1])
def test_packed_device_batch_equals_ascii(built, bucketed):  # noqa: F811
    import torch

    from biobloom_b200 import _lib as L
    from biobloom_b200.mibf import MIBFClassifier
    targets, filters, _, names = built
    path, _ = filters["ss"]
    rng = np.random.default_rng(71 + bucketed)
    reads, _ = _reads(rng, targets, 3000)
    reads = _mutate(rng, reads)
    seq, off = _concat(reads)
    words, valid, _ = _pack(seq)
    n = len(reads)
    mc = MIBFClassifier(path, layout=2)
    mc.set_bucketing(mode=bucketed, bucket_shift=12, max_frames=1 << 16)
    want, wsat = mc.classify(reads, max_hits=mc.num_ids)
    dw = torch.from_numpy(words.view(np.int32)).cuda()
    dv = torch.from_numpy(valid.view(np.int32)).cuda()
    doff = torch.from_numpy(off.astype(np.int64)).cuda()
    mh = mc.num_ids
    hits = torch.zeros((n, mh, 7), dtype=torch.int32, device="cuda")
    nh = torch.zeros(n, dtype=torch.int32, device="cuda")
    sat = torch.zeros(n, dtype=torch.int32, device="cuda")
    b = L.Batch()
    b.seq, b.offsets, b.n_reads, b.location = dw.data_ptr(), doff.data_ptr(), n, L.DEVICE
    b.encoding, b.valid = L.BASES_2BIT, dv.data_ptr()
    r = L.MibfResult()
    r.hits, r.max_hits, r.n_hits, r.sat_count, r.location = (
        hits.data_ptr(), mh, nh.data_ptr(), sat.data_ptr(), L.DEVICE)
    L.check_mibf(L.lib().bbt_mibf_classify_batch(mc._ctx, ctypes.byref(b), ctypes.byref(r),
                                                 None), mc._ctx)
    mc.sync()
    torch.cuda.synchronize()
    hits, nh, sat = hits.cpu().numpy(), nh.cpu().numpy(), sat.cpu().numpy()
    for i in range(n):
        got = [tuple(int(x) for x in hits[i, j]) for j in range(int(nh[i]))]
        assert got == want[i] and int(sat[i]) == int(wsat[i]), i
    mc.close()


@pytest.mark.parametrize("paired", [False, True])
def test_packed_host_batch_over_several_chunks(built, paired):  # noqa: F811
    """More reads than one pipeline chunk holds: later chunks start at bases
    that are not on a code-word boundary."""
    from biobloom_b200.mibf import MIBFClassifier
    targets, filters, _, names = built
    path, _ = filters["ss"]
    rng = np.random.default_rng(81 + paired)
    n = 1_300_000
    genome = np.frombuffer(b"".join(targets), dtype=np.uint8)

    def batch():
        lens = rng.integers(20, 60, n).astype(np.uint64)
        off = np.zeros(n + 1, dtype=np.uint64)
        off[1:] = np.cumsum(lens)
        starts = rng.integers(0, len(genome) - 60, n)
        idx = np.repeat(starts, lens.astype(np.int64)) + (
            np.arange(int(off[-1])) - np.repeat(off[:-1], lens.astype(np.int64)).astype(np.int64))
        seq = genome[idx].copy()
        seq[rng.random(len(seq)) < 0.005] = ord("N")
        return seq, off

    seq, off = batch()
    seq2 = off2 = None
    if paired:
        seq2, off2 = batch()
    got = []
    for packed in (False, True):
        mc = MIBFClassifier(path, layout=2)
        got.append(_run_host(mc, seq, off, seq2, off2, packed=packed, max_hits=12))
        mc.close()
    (h0, s0, (c0, n0)), (h1, s1, (c1, n1)) = got
    assert h0 == h1
    assert np.array_equal(s0, s1)
    assert np.array_equal(c0, c1) and n0 == n1
