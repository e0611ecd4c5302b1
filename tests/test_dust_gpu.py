"""DUST masking (-D) on the GPU against the reference's SeqEval with
opt::dust (tests/golden/make_golden_dust.py) and against the CPU oracle on
reads built to stress the masking kernel: long homopolymers and tandem
repeats, whose pending-interval lists overflow the kernel's first pass and go
through the second.  The CLI's -D files are checked with the other modes in
test_filter_modes_gpu.py."""
import os
import sys

import numpy as np
import pytest

from tests import oracle_lib as ol
from tests.fixtures import expected_hits, filter_paths, golden, read_fastx

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))

import make_golden_dust as mgd  # noqa: E402

pytestmark = pytest.mark.gpu


def _hitsets(hits, nf):
    return [set(f for f in range(nf) if (int(h[f // 64]) >> (f % 64)) & 1) for h in hits]


def _classifier(method, score, streak):
    from biobloom_b200 import BioBloomClassifier
    if method in ("harmonic", "binomial"):
        return BioBloomClassifier(filter_paths(), float(score), streak_threshold=int(streak),
                                  score_type=method)
    return BioBloomClassifier(filter_paths(), float(score), streak_threshold=int(streak))


@pytest.mark.parametrize("name", sorted(mgd.HIT_CASES))
def test_dust_hits_match_reference(name):
    method, score, streak, paired = mgd.HIT_CASES[name]
    rows, summary = expected_hits(name)
    r1 = [s for _, s in read_fastx(golden("reads_dust.fa.gz"))]
    r2 = [s for _, s in read_fastx(golden("reads_dust_2.fa.gz"))] if paired else None
    with _classifier(method, score, streak) as bbc:
        bbc.set_dust(True, 20, 64)
        h1, h2, _ = bbc.classify(r1, r2)
        assert bbc.summary_tsv() == summary
    assert _hitsets(h1, 3) == [r[1] for r in rows]
    if paired:
        assert _hitsets(h2, 3) == [r[2] for r in rows]


@pytest.mark.parametrize("name", sorted(mgd.SCORE_CASES))
def test_dust_scores_match_reference(name):
    from biobloom_b200 import MODE_SCORES, BioBloomClassifier
    method, streak = mgd.SCORE_CASES[name]
    recs = [s for _, s in read_fastx(golden("reads_dust.fa.gz"))]
    if method == "length":
        bbc = BioBloomClassifier(filter_paths(), 40, streak_threshold=streak)
    else:
        bbc = BioBloomClassifier(filter_paths(), None, streak_threshold=streak,
                                 score_type=method)
    with bbc:
        bbc.set_dust(True)
        bbc.set_mode(MODE_SCORES)
        _, _, _, sc, _ = bbc.classify(recs, scores=True)
    want = []
    with open(golden(f"expected_scores_{name}.tsv")) as f:
        for line in f:
            want.append([int(v, 16) for v in line.rstrip("\n").split("\t")[1].split(",")])
    want = np.array(want, dtype=np.uint64)
    if method != "binomial":
        assert np.array_equal(sc.view(np.uint64), want)
    else:
        w = want.view(np.float64)
        same = sc.view(np.uint64) == want
        with np.errstate(invalid="ignore"):
            close = np.abs(sc - w) <= 1e-9 + 1e-12 * np.abs(w)
        assert np.all(same | (np.isfinite(w) & close))


def _repeat_reads(seed, n):
    """Fixture reads with long low-complexity stretches, N runs and case
    changes: many overflow the first pass's list of pending intervals."""
    rng = np.random.default_rng(seed)
    pool = [s for _, s in read_fastx(golden("reads_se.fa.gz")) if len(s) > 50]
    units = [b"A", b"C", b"AC", b"AT", b"AAG", b"GATA", b"ACGTT"]
    out = []
    for _ in range(n):
        parts = []
        for _ in range(int(rng.integers(1, 6))):
            if rng.random() < 0.5:
                u = units[int(rng.integers(len(units)))]
                rep = (u * 3000)[: int(rng.integers(10, 1500))]
                parts.append(rep.lower() if rng.random() < 0.2 else rep)
            else:
                parts.append(pool[int(rng.integers(len(pool)))])
            if rng.random() < 0.15:
                parts.append(b"N" * int(rng.integers(1, 5)))
        out.append(b"".join(parts))
    return out


@pytest.mark.parametrize("T,W", [(20, 64), (30, 32), (10, 16)])
@pytest.mark.parametrize("paired", [False, True])
def test_dust_on_repeats_matches_oracle(T, W, paired):
    from biobloom_b200 import BioBloomClassifier
    r1 = _repeat_reads(T + W, 120)
    r2 = _repeat_reads(T + W + 1, 120) if paired else None
    with BioBloomClassifier(filter_paths()) as bbc:
        bbc.set_dust(True, T, W)
        h1, h2, cat = bbc.classify(r1, r2)
        counts, _ = bbc.summary()
    filters = [ol.Filter.load(p) for p in filter_paths()]
    s1, o1 = ol.pack_reads(r1)
    with ol.dust(T, W):
        w1, _ = ol.classify(s1, o1, filters)
        w2 = None
        if paired:
            s2, o2 = ol.pack_reads(r2)
            w2, _ = ol.classify(s2, o2, filters)
    assert np.array_equal(h1, w1)
    if paired:
        assert np.array_equal(h2, w2)
    want, cats = ol.summary_counts(w1, 3, w2)
    assert np.array_equal(cat, cats) and np.array_equal(counts, want)


def test_dust_device_batch_with_offset_base_matches_host():
    import torch
    from biobloom_b200 import BioBloomClassifier
    from biobloom_b200.classifier import pack
    reads = _repeat_reads(5, 200)
    with BioBloomClassifier(filter_paths()) as bbc:
        bbc.set_dust(True)
        h, _, c = bbc.classify(reads)
        seq, off = pack(reads)
        pad = 1000  # offsets that do not start at 0
        seq_p = np.concatenate([np.full(pad, ord("A"), dtype=np.uint8), seq])
        dev = torch.device("cuda:0")
        ts = torch.from_numpy(seq_p).to(dev)
        to = torch.from_numpy((off + pad).astype(np.int64)).to(dev)
        dh, _, dc = bbc.classify_device(ts, to)
        torch.cuda.synchronize()
    assert np.array_equal(dh.cpu().numpy().view(np.uint64), h)
    assert np.array_equal(dc.cpu().numpy().astype(np.uint32), c)


def test_dust_parameters_are_checked():
    from biobloom_b200 import BBTError, BioBloomClassifier
    with BioBloomClassifier(filter_paths()) as bbc:
        with pytest.raises(BBTError):
            bbc.set_dust(True, 20, 2)
        with pytest.raises(BBTError):
            bbc.set_dust(True, 20, 5000)
        bbc.set_dust(True, 20, 64)
        bbc.set_dust(False)
