"""HARMONIC and BINOMIAL scoring (-S) on the GPU: per-read hits and
summary.tsv against the reference's own evalHarmonic / evalBinomial
(golden files of tests/golden/make_golden_modes.py), the CLI's summary against
the reference CLI's, and random reads against the oracle on every launch path,
device batches, CUDA graphs and the serving engine."""
import os
import subprocess

import numpy as np
import pytest

from tests import oracle_lib as ol
from tests.fixtures import expected_hits, filter_paths, golden, read_fastx
from tests.test_oracle_golden import MODE_CASES, mode_args

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CLI = os.path.join(ROOT, "biobloom_b200", "bin", "biobloomcategorizer")


def _sets(hits, nf):
    return [set(f for f in range(nf) if (int(h[f // 64]) >> (f % 64)) & 1) for h in hits]


@pytest.mark.parametrize("path", [1, 2, 3], ids=["plain", "persistent", "filter-major"])
@pytest.mark.parametrize("name,method,score,streak,paired", MODE_CASES)
def test_golden_modes(name, method, score, streak, paired, path):
    from biobloom_b200 import BioBloomClassifier
    rows, summary = expected_hits(name)
    with BioBloomClassifier(filter_paths(), score, streak_threshold=streak, score_type=method,
                            path=path) as bbc:
        if paired:
            r1 = read_fastx(golden("reads_1.fq.gz"))
            r2 = read_fastx(golden("reads_2.fq.gz"))
            h1, h2, _ = bbc.classify([s for _, s in r1], [s for _, s in r2])
            assert _sets(h1, 3) == [r[1] for r in rows]
            assert _sets(h2, 3) == [r[2] for r in rows]
        else:
            recs = read_fastx(golden("reads_se.fa.gz"))
            hits, _, _ = bbc.classify([s for _, s in recs])
            assert _sets(hits, 3) == [r[1] for r in rows]
        assert bbc.summary_tsv() == summary


@pytest.mark.parametrize("name,method,score,streak,paired", MODE_CASES)
def test_cli_modes_summary(name, method, score, streak, paired, tmp_path):
    filters = " ".join(filter_paths())
    args = [CLI, "-p", str(tmp_path / "o"), "-S", method, "-s", str(score), "-r", str(streak),
            "-f", filters]
    if paired:
        args += ["-e", golden("reads_1.fq.gz"), golden("reads_2.fq.gz")]
    else:
        args += [golden("reads_se.fa.gz")]
    p = subprocess.run(args, capture_output=True)
    assert p.returncode == 0, p.stderr.decode()
    with open(golden(f"expected_summary_{name}.tsv")) as f:
        assert (tmp_path / "o_summary.tsv").read_text() == f.read()


def _case(seed, k, h, glen=40000, n_filters=2):
    rng = np.random.default_rng(seed)
    acgt = np.frombuffer(b"ACGT", dtype=np.uint8)
    genomes = [rng.choice(acgt, glen) for _ in range(n_filters)]
    filters = [ol.Filter.make([g.tobytes()], k=k, fpr=0.2, h=h) for g in genomes]
    reads = []
    for _ in range(1500):
        L = int(rng.integers(1, 400)) if rng.random() < 0.95 else int(rng.integers(400, 6000))
        src = int(rng.integers(-1, n_filters))
        if src >= 0 and L < glen:
            st = int(rng.integers(0, glen - L))
            r = genomes[src][st:st + L].copy()
        else:
            r = rng.choice(acgt, L)
        m = rng.random(L) < 0.02
        r[m] = rng.choice(acgt, int(m.sum()))
        if rng.random() < 0.3:
            r[rng.random(L) < 0.03] = ord("N")
        reads.append(r.tobytes())
    return rng, filters, reads


@pytest.mark.parametrize("seed,k,h,method,score,streak", [
    (1, 25, 0, "harmonic", 0.15, 3), (2, 21, 2, "harmonic", 0.45, 1),
    (3, 17, 3, "harmonic", 0.05, 0), (4, 25, 0, "binomial", 100, 3),
    (5, 31, 2, "binomial", 20, 2), (6, 15, 4, "binomial", 60, 5)])
@pytest.mark.parametrize("launch", [dict(path=1), dict(path=2), dict(path=2, steps=2),
                                    dict(path=2, steps=3)],
                         ids=["plain", "persistent", "persistent-wide", "persistent-wide-full"])
def test_random_modes_match_oracle(seed, k, h, method, score, streak, launch, tmp_path):
    import torch
    from biobloom_b200 import BioBloomClassifier
    rng, filters, reads = _case(seed, k, h)
    paths = []
    for i, f in enumerate(filters):
        stem = str(tmp_path / f"m{i}")
        f.store(stem + ".bf")
        ol.write_info(stem + ".txt", f"m{i}", f.k, 0.2, f.h, 1, "x", f.m, 1, 0.1, 0, 0.1)
        paths.append(stem + ".bf")
    thr, scoring = mode_args(method, score)
    seq, off = ol.pack_reads(reads)
    want, _ = ol.classify(seq, off, filters, thr, streak, scoring)
    with BioBloomClassifier(paths, score, streak_threshold=streak, score_type=method,
                            **launch) as bbc:
        hits, _, _ = bbc.classify(reads)
        assert np.array_equal(hits, want)
        dseq = torch.tensor(np.frombuffer(seq, dtype=np.uint8), device="cuda")
        doff = torch.tensor(off.astype(np.int64), device="cuda")
        dh, _, _ = bbc.classify_device(dseq, doff)
        torch.cuda.synchronize()
        assert np.array_equal(dh.cpu().numpy().view(np.uint64), want)
        if launch["path"] == 2:
            gh = torch.zeros_like(dh)
            g = bbc.graph(dseq, doff, gh, reads_per_launch=300)
            s = torch.cuda.Stream()
            g.launch(s)
            s.synchronize()
            assert np.array_equal(gh.cpu().numpy().view(np.uint64), want)
            g.close()


def test_binomial_in_the_serving_engine(tmp_path):
    from biobloom_b200 import BioBloomClassifier
    from biobloom_b200.server import Server
    rng, filters, reads = _case(9, 25, 0)
    paths = []
    for i, f in enumerate(filters):
        stem = str(tmp_path / f"s{i}")
        f.store(stem + ".bf")
        ol.write_info(stem + ".txt", f"s{i}", f.k, 0.2, f.h, 1, "x", f.m, 1, 0.1, 0, 0.1)
        paths.append(stem + ".bf")
    thr, scoring = mode_args("binomial", 100)
    with BioBloomClassifier(paths, 100, score_type="binomial") as bbc:
        with Server(bbc, None, slots=3) as srv:
            parts = [reads[:10], reads[10:900], reads[900:]]
            hs = [srv.submit_bloom(p) for p in parts]
            for h in hs:
                srv.wait(h)
        for p, h in zip(parts, hs):
            seq, off = ol.pack_reads(p)
            want, _ = ol.classify(seq, off, filters, thr, 3, scoring)
            assert np.array_equal(h.hits[:h.n], want)
