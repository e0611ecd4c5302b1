"""miBF path on the GPU: the biobloommicategorizer CLI against the reference
CLI's golden output, the C ABI (host and device batches) against the oracle on
seeded inputs, and the GPU maker against the oracle's build, byte for byte."""
import os
import subprocess

import numpy as np
import pytest

from tests import mibf_util as mu
from tests import oracle_lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CLI = os.path.join(ROOT, "biobloom_b200", "bin", "biobloommicategorizer")
BASES = np.frombuffer(b"ACGT", dtype=np.uint8)

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("case", sorted(mu.CASES))
def test_cli_matches_reference_cli(case, tmp_path):
    prefix, args, paired = mu.CASES[case]
    if paired is None:
        inputs = [mu.g("reads_edge.fa.gz")]
    elif paired:
        inputs = ["-e", mu.g("reads_1.fq.gz"), mu.g("reads_2.fq.gz")]
    else:
        inputs = [mu.g("reads_se.fa.gz")]
    p = subprocess.run([CLI, "-p", str(tmp_path / "out"), "-f", mu.g(f"{prefix}.bf")] + args +
                       inputs, capture_output=True)
    assert p.returncode == 0, p.stderr.decode()
    with open(mu.g(f"mi_{case}.tsv"), "rb") as f:
        assert p.stdout == f.read()
    summary = (tmp_path / "out_summary.tsv").read_text()
    if paired is None:
        results, names, o, _ = mu.oracle_results(case)
        assert summary == mu.summary_text(names, results, False, o["hit_only"])
    else:
        with open(mu.g(f"mi_{case}_summary.tsv")) as f:
            assert summary == f.read()


def _genome(rng, n, gc=0.5):
    u = rng.random(n)
    return np.where(u < gc / 2, ord("C"), np.where(u < gc, ord("G"),
                    np.where(u < gc + (1 - gc) / 2, ord("A"), ord("T")))).astype(np.uint8)


def _targets(rng, n_targets=24, length=12000):
    seqs = [_genome(rng, length, float(rng.uniform(0.35, 0.65))) for _ in range(n_targets)]
    for i in range(0, n_targets - 1, 3):  # shared blocks between target pairs
        a = int(rng.integers(0, length - 3000))
        b = int(rng.integers(0, length - 3000))
        seqs[i + 1][b:b + 2000] = seqs[i][a:a + 2000]
    seqs[5][100:6100] = np.tile(_genome(rng, 40), 150)  # a repeat-rich target
    return [s.tobytes() for s in seqs]


def _reads(rng, targets, n, paired=False, long_frac=0.05):
    comp = bytes.maketrans(b"ACGTN", b"TGCAN")
    out1, out2 = [], []
    for i in range(n):
        L = int(rng.integers(1, 300))
        if rng.random() < long_frac:
            L = int(rng.integers(500, 3000))  # several staging chunks
        t = int(rng.integers(-1, len(targets)))
        if t < 0 or L > len(targets[t]) - 1:
            s = BASES[rng.integers(0, 4, L)].tobytes()
        else:
            st = int(rng.integers(0, len(targets[t]) - L))
            s = targets[t][st:st + L]
            a = np.frombuffer(s, dtype=np.uint8).copy()
            m = rng.random(L) < 0.01
            a[m] = BASES[rng.integers(0, 4, int(m.sum()))]
            if rng.random() < 0.2:
                a[rng.random(L) < 0.02] = ord("N")
            if rng.random() < 0.2:
                a[rng.random(L) < 0.3] |= 0x20
            s = a.tobytes()
            if rng.random() < 0.5:
                s = s.translate(comp)[::-1]
        out1.append(s)
        if paired:
            out2.append(BASES[rng.integers(0, 4, int(rng.integers(1, 200)))].tobytes()
                        if rng.random() < 0.3 else s[::-1].translate(comp))
    return out1, (out2 if paired else None)


@pytest.fixture(scope="module")
def built(tmp_path_factory):
    """A 24-target miBF (3 spaced seeds) and a k-mer-mode one, built by the oracle."""
    rng = np.random.default_rng(11)
    targets = _targets(rng)
    d = tmp_path_factory.mktemp("mibf")
    seeds = ["1111011101110010111011111", "1101111101001011111011011",
             "1111101011100111010111111"]
    names = [f"target{i + 1}" for i in range(len(targets))]
    out = {}
    for tag, sd in (("ss", seeds), ("km", None)):
        f = oracle_lib.MIBF.build(targets, list(range(1, len(targets) + 1)), seeds=sd, k=25, h=3,
                                  occupancy=0.5)
        f.store(str(d / tag))
        with open(d / f"{tag}_ids.txt", "w") as fh:
            for i, n in enumerate(names):
                fh.write(f"{i + 1}\t{n}\n")
        out[tag] = (str(d / f"{tag}.bf"), f)
    return targets, out, seeds, names


def _oracle_query(f, names, reads, reads2, o):
    h = f.f.h
    allowed = 0 if (o["frame_matches"] > h or f.f.nseeds == 0) else h - o["frame_matches"]
    probs, _ = f.frame_probs(len(names) + 1, allowed)
    cache = {}
    res = []
    for i, s in enumerate(reads):
        s2 = reads2[i] if reads2 is not None else None
        fc = mu.frame_count(len(s), len(s2) if s2 is not None else 0, f.f.k, s2 is not None)
        if fc == 0:
            res.append(([], 0))
            continue
        if fc not in cache:
            cache[fc] = mu.min_counts(fc, probs, o["score"])
        res.append(f.query(s, cache[fc], seq2=s2, multi=o["multi"], allowed_miss=allowed,
                           min_nonsat=o["min_nonsat"], best_agree=o["best"]))
    return res


OPTS = [
    {},
    {"multi": 3.0},
    {"frame_matches": 2, "min_nonsat": 2},
    {"frame_matches": 3, "best": True},
    {"score": 1e-3, "multi": 100.0},
]


def _opts(d):
    o = {"score": 1e-10, "multi": 1.0, "frame_matches": 1, "min_nonsat": 0, "best": False}
    o.update(d)
    return o


@pytest.mark.parametrize("layout", [1, 2])
@pytest.mark.parametrize("tag", ["ss", "km"])
@pytest.mark.parametrize("paired", [False, True])
@pytest.mark.parametrize("oi", range(len(OPTS)))
def test_abi_host_batch_matches_oracle(built, tag, paired, oi, layout):
    from biobloom_b200.mibf import MIBFClassifier
    targets, filters, _, names = built
    path, f = filters[tag]
    o = _opts(OPTS[oi])
    rng = np.random.default_rng(100 + oi + 10 * paired)
    reads, reads2 = _reads(rng, targets, 700, paired=paired)
    want = _oracle_query(f, names, reads, reads2, o)
    mc = MIBFClassifier(path, score=o["score"], frame_matches=o["frame_matches"],
                        multi=o["multi"], min_nonsat=o["min_nonsat"], best_hit_agree=o["best"],
                        layout=layout)
    assert mc.layout == layout
    got, sat = mc.classify(reads, reads2, max_hits=2)  # max_hits 2 exercises the retry
    for i, (res, s) in enumerate(want):
        assert (got[i], int(sat[i])) == (res, s), i
    counts, n = mc.summary()
    assert n == len(reads)
    nf = len(names) + 1
    assert counts[2 * (nf + 2) + 1] == sum(1 for r, _ in want if not r)
    assert counts[2 * (nf + 2)] == sum(1 for r, _ in want if len(r) > 1)
    mc.close()


@pytest.mark.parametrize("layout", [1, 2])
def test_abi_device_batch_matches_host_batch(built, layout):
    import torch
    from biobloom_b200.mibf import MIBFClassifier
    from biobloom_b200.classifier import pack
    targets, filters, _, names = built
    path, f = filters["ss"]
    rng = np.random.default_rng(5)
    reads, _ = _reads(rng, targets, 3000)
    mc = MIBFClassifier(path, layout=layout)
    want, wsat = mc.classify(reads)
    seq, off = pack(reads)
    dseq = torch.from_numpy(seq.copy()).cuda()
    doff = torch.from_numpy(off.astype(np.int64)).cuda()
    hits, nh, sat = mc.classify_device(dseq, doff, max_hits=mc.num_ids)
    mc.sync()
    torch.cuda.synchronize()
    hits, nh, sat = hits.cpu().numpy(), nh.cpu().numpy(), sat.cpu().numpy()
    for i in range(len(reads)):
        got = [tuple(int(x) for x in hits[i, j]) for j in range(int(nh[i]))]
        assert got == want[i] and int(sat[i]) == int(wsat[i]), i


def test_results_are_the_same_alone_and_in_a_batch(built):
    from biobloom_b200.mibf import MIBFClassifier
    targets, filters, _, names = built
    path, _ = filters["ss"]
    rng = np.random.default_rng(9)
    reads, _ = _reads(rng, targets, 400)
    mc = MIBFClassifier(path)
    batch, bsat = mc.classify(reads)
    for i in range(0, 400, 37):
        one, osat = mc.classify([reads[i]])
        assert one[0] == batch[i] and osat[0] == bsat[i]


@pytest.mark.parametrize("tag", ["ss", "km"])
def test_gpu_maker_matches_oracle_build(built, tag, tmp_path):
    from biobloom_b200.mibf import make_mibf
    targets, filters, seeds, names = built
    path, _ = filters[tag]
    make_mibf(str(tmp_path / "g"), targets, list(range(1, len(targets) + 1)), names,
              seeds=seeds if tag == "ss" else None, k=25, hash_num=3, occupancy=0.5)
    for ext in (".bf", ".sdsl", "_ids.txt"):
        with open(path[:-3] + ext, "rb") as a, open(str(tmp_path / "g") + ext, "rb") as b:
            assert a.read() == b.read(), ext


def test_ids_outside_the_names_file_tally_nothing(tmp_path):
    """IDs in the filter that the ID file does not name (and ID 0) count as hits
    and saturation but are never results, in both layouts."""
    import shutil
    from biobloom_b200.mibf import MIBFClassifier
    rng = np.random.default_rng(8)
    seqs = [_genome(rng, 3000).tobytes() for _ in range(6)]
    f = oracle_lib.MIBF.build(seqs, [1, 2, 3, 4, 5, 6], k=21, h=2, occupancy=0.5)
    f.store(str(tmp_path / "x"))
    with open(tmp_path / "x_ids.txt", "w") as fh:   # names only IDs 1-3
        fh.write("1\ta\n2\tb\n3\tc\n")
    reads, _ = _reads(rng, seqs, 300)
    want = _oracle_query(f, ["a", "b", "c"], reads, None, _opts({}))
    for layout in (1, 2):
        mc = MIBFClassifier(str(tmp_path / "x.bf"), layout=layout)
        got, sat = mc.classify(reads)
        assert [(g, int(s)) for g, s in zip(got, sat)] == [(r, s) for r, s in want]
        assert mc.last_counts()[2] > 0


def test_gpu_maker_multi_contig_ids(tmp_path):
    """Several sequences per ID, sequences shorter than k, and N runs."""
    from biobloom_b200.mibf import make_mibf
    rng = np.random.default_rng(21)
    seqs = [_genome(rng, int(rng.integers(10, 4000))).tobytes() for _ in range(30)]
    seqs[3] = b"ACGTN" * 40
    seqs[7] = b"ACGTACGTACGTACGT"  # k - 1 bases: no frames
    ids = [int(rng.integers(1, 9)) for _ in seqs]
    names = [f"n{i}" for i in range(1, 9)]
    seeds = ["11011111111111011", "11111011111101111"]
    f = oracle_lib.MIBF.build(seqs, ids, seeds=seeds, k=17, h=2, occupancy=0.3)
    f.store(str(tmp_path / "o"))
    make_mibf(str(tmp_path / "g"), seqs, ids, names, seeds=seeds, k=17, occupancy=0.3)
    for ext in (".bf", ".sdsl"):
        with open(str(tmp_path / "o") + ext, "rb") as a, open(str(tmp_path / "g") + ext, "rb") as b:
            assert a.read() == b.read(), ext


def _many_reads(rng, targets, n, length):
    """n reads of `length` bases: 80% substrings of the targets, 20% random."""
    genome = np.frombuffer(b"".join(targets), dtype=np.uint8)
    starts = rng.integers(0, len(genome) - length, n)
    idx = starts[:, None] + np.arange(length)[None, :]
    seq = genome[idx]
    rand = rng.random(n) < 0.2
    seq[rand] = np.frombuffer(b"ACGT", dtype=np.uint8)[rng.integers(0, 4, (int(rand.sum()),
                                                                           length))]
    off = np.arange(n + 1, dtype=np.uint64) * np.uint64(length)
    return np.ascontiguousarray(seq.reshape(-1)), off


def _abi_host(mc, seq, off, seq2, off2, max_hits):
    import ctypes

    from biobloom_b200 import _lib as L
    n = len(off) - 1
    b = L.Batch()
    b.seq, b.offsets, b.n_reads, b.location = seq.ctypes.data, off.ctypes.data, n, L.HOST
    if seq2 is not None:
        b.seq2, b.offsets2 = seq2.ctypes.data, off2.ctypes.data
    hits = np.zeros((n, max_hits, 7), dtype=np.uint32)
    nh = np.zeros(n, dtype=np.uint32)
    sat = np.zeros(n, dtype=np.uint32)
    r = L.MibfResult()
    r.hits, r.max_hits, r.n_hits, r.sat_count, r.location = (
        hits.ctypes.data, max_hits, nh.ctypes.data, sat.ctypes.data, L.HOST)
    rc = L.lib().bbt_mibf_classify_batch(mc._ctx, ctypes.byref(b), ctypes.byref(r), None)
    return rc, hits, nh, sat


@pytest.mark.parametrize("paired", [False, True])
def test_host_batch_in_chunks_matches_one_device_launch(built, paired):
    """A host batch of more than one pipeline chunk (1M reads) gives the
    results and summary of the same reads classified in one device launch;
    with too few result slots it reports the overflow, keeps n_hits exact and
    adds nothing to the summary."""
    import torch

    from biobloom_b200 import _lib as L
    from biobloom_b200.mibf import MIBFClassifier
    targets, filters, _, names = built
    path, _ = filters["ss"]
    rng = np.random.default_rng(21)
    n = 1_100_000
    seq, off = _many_reads(rng, targets, n, 40)
    seq2 = off2 = None
    if paired:
        seq2, off2 = _many_reads(rng, targets, n, 60)
    mh = 8
    a = MIBFClassifier(path)
    rc, hits, nh, sat = _abi_host(a, seq, off, seq2, off2, mh)
    assert rc == 0
    counts_a, reads_a = a.summary()
    d = MIBFClassifier(path)
    t = lambda x: torch.from_numpy(x.astype(np.int64) if x.dtype == np.uint64 else x).cuda()
    dh, dn, ds = d.classify_device(t(seq), t(off), t(seq2) if paired else None,
                                   t(off2) if paired else None, max_hits=mh)
    d.sync()
    torch.cuda.synchronize()
    dn = dn.cpu().numpy().view(np.uint32)
    assert np.array_equal(nh, dn)
    assert np.array_equal(sat, ds.cpu().numpy().view(np.uint32))
    dh = dh.cpu().numpy().view(np.uint32).reshape(n, mh, 7)
    keep = np.arange(mh)[None, :] < nh[:, None]
    assert np.array_equal(hits[keep], dh[keep])
    counts_d, reads_d = d.summary()
    assert reads_a == reads_d == n and np.array_equal(counts_a, counts_d)
    assert nh.max() > 1
    # overflow: one result slot while some reads have more
    rc, _, nh1, _ = _abi_host(a, seq, off, seq2, off2, 1)
    assert rc == L.ERR_OVERFLOW
    assert np.array_equal(nh1, nh)
    counts_b, reads_b = a.summary()
    assert reads_b == reads_a and np.array_equal(counts_b, counts_a)
    a.close()
    d.close()


@pytest.fixture(scope="module")
def many_targets(tmp_path_factory):
    """A 5000-target miBF (IDs up to 5000, above the shared-memory tally's
    1023): 5000 seeded 400 bp targets, every fourth sharing a block with the
    one before, built by the oracle."""
    rng = np.random.default_rng(77)
    targets = [_genome(rng, 400, float(rng.uniform(0.35, 0.65))) for _ in range(5000)]
    for i in range(1, 5000, 4):
        targets[i][100:220] = targets[i - 1][50:170]
    targets = [t.tobytes() for t in targets]
    d = tmp_path_factory.mktemp("mibf5k")
    names = [f"t{i + 1}" for i in range(len(targets))]
    seeds = ["1111011101110010111011111", "1101111101001011111011011",
             "1111101011100111010111111"]
    f = oracle_lib.MIBF.build(targets, list(range(1, len(targets) + 1)), seeds=seeds, k=25,
                              h=3, occupancy=0.5)
    f.store(str(d / "big"))
    with open(d / "big_ids.txt", "w") as fh:
        for i, n in enumerate(names):
            fh.write(f"{i + 1}\t{n}\n")
    return targets, str(d / "big.bf"), f, names


@pytest.mark.parametrize("layout", [1, 2])
@pytest.mark.parametrize("oi", [0, 1, 2])
def test_five_thousand_targets_match_oracle(many_targets, layout, oi):
    """More IDs than the shared-memory tally holds: per-warp tally tables in
    global memory, cleared over the IDs a read touched (or all of them after
    a long read touched more than the list holds)."""
    from biobloom_b200.mibf import MIBFClassifier
    targets, path, f, names = many_targets
    o = _opts(OPTS[oi])
    rng = np.random.default_rng(300 + oi)
    reads = []
    for _ in range(1500):  # 150 bp: one minCount row for all of them
        t = int(rng.integers(0, len(targets)))
        st = int(rng.integers(0, 250))
        a = np.frombuffer(targets[t][st:st + 150], dtype=np.uint8).copy()
        m = rng.random(150) < 0.01
        a[m] = BASES[rng.integers(0, 4, int(m.sum()))]
        reads.append(a.tobytes() if rng.random() < 0.9 else BASES[rng.integers(0, 4, 150)].tobytes())
    reads += [BASES[rng.integers(0, 4, 9000)].tobytes()]          # touches thousands of IDs
    reads += [b"".join(targets[i] for i in range(40, 70))]      # 30 targets in one read
    want = _oracle_query(f, names, reads, None, o)
    mc = MIBFClassifier(path, score=o["score"], frame_matches=o["frame_matches"],
                        multi=o["multi"], min_nonsat=o["min_nonsat"], best_hit_agree=o["best"],
                        layout=layout)
    assert mc.num_ids == 5001
    got, sat = mc.classify(reads, None, max_hits=4)
    for i, (res, s) in enumerate(want):
        assert (got[i], int(sat[i])) == (res, s), i
    assert any(len(r) for r, _ in want[:1500])
    counts, n = mc.summary()
    assert n == len(reads)
    mc.close()
