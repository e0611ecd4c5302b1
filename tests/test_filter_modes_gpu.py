"""Filtering modes on the GPU: ordered (-c), best hit (-b), with scores (-w),
exhaustive scores (bbt_classify_batch_scores), single-file paired input and
file lists.

  * the CLI's files (categorized reads, stdout, summary) against the
    reference CLI's on the same fixtures (tests/golden/make_golden_print.py);
  * per-read scores against the reference's SeqEval::evalScore
    (tests/golden/make_golden_scores.py) and against the CPU oracle on
    longer reads with N runs, for filters of one k and of mixed k;
  * hit words, categories and summaries of the modes against the oracle.

Scores of SIMPLE, HARMONIC and LENGTH are sums and quotients of exactly
representable terms in a fixed order and must match bit for bit.  BINOMIAL
scores are -10 log10 of a binomial tail whose terms are evaluated in log
space (lgamma of numbers up to the frame count, ~2^14 here): each term, and
so the tail, carries a relative error of order 1e-13 to 1e-12 in the shim
and in the kernel alike, which moves the score by 10/ln(10) times that.
They must agree within 1e-9 absolute plus 1e-12 relative (infinities
exactly), and printed with 6 significant digits within one unit in the last
printed digit.
"""
import gzip
import os
import re
import subprocess
import sys

import numpy as np
import pytest

from tests import oracle_lib as ol
from tests.fixtures import filter_paths, golden, read_fastx

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CLI = os.path.join(ROOT, "biobloom_b200", "bin", "biobloomcategorizer")
sys.path.insert(0, os.path.join(HERE, "golden"))

import make_golden_print as mgp  # noqa: E402
import make_golden_scores as mgs  # noqa: E402

pytestmark = pytest.mark.gpu

BINOMIAL_ATOL, BINOMIAL_RTOL = 1e-9, 1e-12
NUM = re.compile(r"^-?(\d+\.?\d*(e[-+]\d+)?|inf|nan)$")


def _close_text(got, want):
    """Equal line structure; numbers equal or, printed with %g, within one
    unit in the 6th significant digit."""
    gl, wl = got.split(b"\n"), want.split(b"\n")
    if len(gl) != len(wl):
        return False
    for a, b in zip(gl, wl):
        if a == b:
            continue
        ta, tb = a.split(b" "), b.split(b" ")
        if len(ta) != len(tb):
            return False
        for x, y in zip(ta, tb):
            if x == y:
                continue
            xs, ys = x.decode(), y.decode()
            if not (NUM.match(xs) and NUM.match(ys)):
                return False
            fx, fy = float(xs), float(ys)
            if abs(fx - fy) > 1.5e-5 * max(abs(fx), abs(fy)):
                return False
    return True


@pytest.mark.parametrize("case", sorted(mgp.MODE_CASES))
def test_mode_cli_outputs_match_reference(case, tmp_path):
    args, kind = mgp.MODE_CASES[case]
    filters = " ".join(os.path.join(mgp.BBT, f"f{i}.bf") for i in range(3))
    p = subprocess.run([CLI, "-p", str(tmp_path / "out"), "-f", filters] + args +
                       mgp.mode_inputs(kind, str(tmp_path)), capture_output=True)
    assert p.returncode == 0, p.stderr.decode()
    got = mgp.collect(str(tmp_path), p.stdout, summary=True)
    with gzip.open(os.path.join(mgp.BBT, f"print_{case}.txt.gz"), "rb") as f:
        want = f.read()
    if "binomial" in case:
        assert got == want or _close_text(got, want)
    else:
        assert got == want


def _expected_scores(case):
    rows = []
    with open(golden(f"expected_scores_{case}.tsv")) as f:
        for line in f:
            rows.append([int(v, 16) for v in line.rstrip("\n").split("\t")[1].split(",")])
    return np.array(rows, dtype=np.uint64).view(np.float64)


def _classifier(paths, method, streak, **kw):
    from biobloom_b200 import BioBloomClassifier
    if method == "length":
        return BioBloomClassifier(paths, 40, streak_threshold=streak, **kw)
    return BioBloomClassifier(paths, None, streak_threshold=streak,
                              score_type="simple" if method == "simple" else method, **kw)


def _assert_scores(got, want, method):
    if method != "binomial":
        assert np.array_equal(got.view(np.uint64), want.view(np.uint64))
        return
    same = got.view(np.uint64) == want.view(np.uint64)
    finite = np.isfinite(want) & np.isfinite(got)
    with np.errstate(invalid="ignore"):
        close = np.abs(got - want) <= BINOMIAL_ATOL + BINOMIAL_RTOL * np.abs(want)
    assert np.all(same | (finite & close))


@pytest.mark.parametrize("case", sorted(mgs.CASES))
def test_scores_match_reference_evalscore(case):
    from biobloom_b200 import MODE_SCORES
    method, streak = mgs.CASES[case]
    recs = read_fastx(golden("reads_se.fa.gz"))
    with _classifier(filter_paths(), method, streak) as bbc:
        bbc.set_mode(MODE_SCORES)
        _, _, _, sc, _ = bbc.classify([s for _, s in recs], scores=True)
    _assert_scores(sc, _expected_scores(case), method)


def _long_reads(seed, n):
    """Reads of 0-2500 bases: fixture reads glued together with N runs and
    single IUPAC bases between and inside them."""
    rng = np.random.default_rng(seed)
    pool = [s for _, s in read_fastx(golden("reads_se.fa.gz"))]
    pool += [s for _, s in read_fastx(golden("reads_1.fq.gz"))]
    out = []
    for i in range(n):
        parts = []
        for _ in range(int(rng.integers(1, 18))):
            s = bytearray(pool[int(rng.integers(len(pool)))])
            if len(s) and rng.random() < 0.3:
                s[int(rng.integers(len(s)))] = ord("N")
            parts.append(bytes(s))
            if rng.random() < 0.4:
                parts.append(b"N" * int(rng.integers(1, 40)))
        r = b"".join(parts)[: int(rng.integers(0, 2500))]
        out.append(r)
    return out


@pytest.mark.parametrize("method", ["simple", "harmonic", "length", "binomial"])
@pytest.mark.parametrize("mixed_k", [False, True])
@pytest.mark.parametrize("seg", [4, 8])
def test_scores_of_long_reads_match_oracle(method, mixed_k, seg):
    from biobloom_b200 import MODE_SCORES
    paths = filter_paths() + ([golden("len.bf")] if mixed_k else [])
    reads = _long_reads(11 + seg, 300)
    streak = 3
    with _classifier(paths, method, streak, frames_per_lane=seg) as bbc:
        bbc.set_mode(MODE_SCORES)
        _, _, _, sc, _ = bbc.classify(reads, scores=True)
    filters = [ol.Filter.load(p) for p in paths]
    seq, off = ol.pack_reads(reads)
    scoring = {"simple": ol.SIMPLE, "harmonic": ol.HARMONIC, "length": ol.LENGTH,
               "binomial": ol.BINOMIAL}[method]
    want = ol.classify_scores(seq, off, filters, scoring, streak)
    _assert_scores(sc, want, method)


def _oracle_mode(mode, reads, reads2, filters, inclusive, scoring=ol.SIMPLE, thr=0.15):
    seq, off = ol.pack_reads(reads)
    if mode == "besthit":
        h1, _ = ol.best_hit(ol.classify_scores(seq, off, filters, scoring, 3))
    else:
        h1, _ = ol.classify(seq, off, filters, thr, 3, scoring)
    h2 = None
    if reads2 is not None:
        s2, o2 = ol.pack_reads(reads2)
        if mode == "besthit":
            h2, _ = ol.best_hit(ol.classify_scores(s2, o2, filters, scoring, 3))
        else:
            h2, _ = ol.classify(s2, o2, filters, thr, 3, scoring)
    if mode == "ordered":
        h1, h2 = ol.ordered(h1, len(filters), h2, inclusive)
    counts, cats = ol.summary_counts(h1, len(filters), h2, inclusive=inclusive)
    return h1, h2, cats, counts


@pytest.mark.parametrize("mode", ["ordered", "besthit"])
@pytest.mark.parametrize("paired,inclusive", [(False, False), (True, False), (True, True)])
def test_mode_hits_and_summary_match_oracle(mode, paired, inclusive):
    from biobloom_b200 import MODE_BESTHIT, BioBloomClassifier
    paths = filter_paths()
    reads = _long_reads(5, 400)
    reads2 = _long_reads(6, 400) if paired else None
    with BioBloomClassifier(paths) as bbc:
        if inclusive:
            bbc.setInclusive()
        if mode == "ordered":
            bbc.setOrderedFilter()
        else:
            bbc.set_mode(MODE_BESTHIT)
        hits, hits2, cat = bbc.classify(reads, reads2)
        counts, n = bbc.summary()
    filters = [ol.Filter.load(p) for p in paths]
    h1, h2, cats, want = _oracle_mode(mode, reads, reads2, filters, inclusive)
    assert np.array_equal(hits, h1)
    if paired:
        assert np.array_equal(hits2, h2)
    assert np.array_equal(cat, cats)
    assert np.array_equal(counts, want) and n == len(reads)


def test_besthit_refuses_ordered():
    from biobloom_b200 import MODE_BESTHIT, BBTError, BioBloomClassifier
    with BioBloomClassifier(filter_paths()) as bbc:
        bbc.set_mode(MODE_BESTHIT)
        with pytest.raises(BBTError):
            bbc.setOrderedFilter()


def test_scores_on_device_equal_host_scores():
    import torch
    from biobloom_b200 import MODE_SCORES, BioBloomClassifier
    from biobloom_b200.classifier import pack
    reads = _long_reads(9, 200)
    reads2 = _long_reads(10, 200)
    with BioBloomClassifier(filter_paths(), score_type="harmonic") as bbc:
        bbc.set_mode(MODE_SCORES)
        h, h2, c, sc, sc2 = bbc.classify(reads, reads2, scores=True)
        s1, o1 = pack(reads)
        s2, o2 = pack(reads2)
        dev = torch.device("cuda:0")
        t = [torch.from_numpy(np.array(x, dtype=np.int64 if x.dtype == np.uint64 else x.dtype))
             .to(dev) for x in (s1, o1, s2, o2)]
        d1 = torch.empty((len(reads), 3), dtype=torch.float64, device=dev)
        d2 = torch.empty((len(reads), 3), dtype=torch.float64, device=dev)
        dh, dh2, dc = bbc.classify_device(t[0], t[1], t[2], t[3], scores=d1, scores2=d2)
        torch.cuda.synchronize()
    assert np.array_equal(d1.cpu().numpy().view(np.uint64), sc.view(np.uint64))
    assert np.array_equal(d2.cpu().numpy().view(np.uint64), sc2.view(np.uint64))
    assert np.array_equal(dh.cpu().numpy().view(np.uint64), h)
    assert np.array_equal(dc.cpu().numpy().astype(np.uint32), c)
