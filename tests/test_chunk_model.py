"""The product's chunked SeqEval state machine (seqeval_chunk.cuh), compiled
for the host, against the oracle's sequential evalSimple / evalMinMatchLen:
same decision and same count of algorithmic probes on random reads with N
runs, lowercase bases, varied k, h, scores and streak thresholds."""
import ctypes
import os
import subprocess

import numpy as np
import pytest

from tests import oracle_lib as ol

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def model(tmp_path_factory):
    out = str(tmp_path_factory.mktemp("model") / "chunk_model.so")
    subprocess.run(["g++", "-O2", "-shared", "-fPIC", "-I", os.path.join(ROOT, "biobloom_b200",
                    "csrc"), "-I", os.path.join(ROOT, "oracle"), "-o", out,
                    os.path.join(ROOT, "tests", "native", "chunk_model.cpp"),
                    os.path.join(ROOT, "oracle", "bbt_oracle.c")], check=True)
    m = ctypes.CDLL(out)
    m.model_eval.argtypes = [ctypes.c_char_p, ctypes.c_uint64, ctypes.POINTER(ol._BF),
                             ctypes.c_double, ctypes.c_uint, ctypes.c_int,
                             ctypes.POINTER(ctypes.c_uint64)]
    return m


@pytest.mark.parametrize("seed", range(6))
def test_chunk_model_matches_oracle(model, seed):
    rng = np.random.default_rng(seed)
    L = ol.lib()
    acgt = np.frombuffer(b"ACGT", dtype=np.uint8)
    mism = 0
    for trial in range(40):
        h = int(rng.integers(1, 5))
        k = max(h, int(rng.integers(3, 40)))
        f = ol.Filter.create(64 * int(rng.integers(1, 60)), h, k)
        g = rng.choice(acgt, 3000)
        fill = rng.random()
        for p, hv in ol.kmers(g.tobytes(), h, k):
            if rng.random() < fill:
                L.oracle_bf_insert(ctypes.byref(f.bf), (ctypes.c_uint64 * 64)(*hv))
        for r in range(60):
            n = int(rng.integers(0, 400))
            st = int(rng.integers(0, 2600))
            s = g[st:st + n].copy() if rng.random() < 0.5 else rng.choice(acgt, n)
            s = s[:n]
            m = rng.random(len(s)) < rng.random() * 0.05
            s[m] = rng.choice(acgt, m.sum())
            if rng.random() < 0.3:
                m = rng.random(len(s)) < rng.random() * 0.2
                s[m] = np.frombuffer(b"NnRX", dtype=np.uint8)[rng.integers(0, 4, m.sum())]
            if rng.random() < 0.2:
                s = np.where(rng.random(len(s)) < 0.3, s | 0x20, s).astype(np.uint8)
            b = s.tobytes()
            streak = int(rng.integers(0, 6)) if rng.random() > 0.05 else int(rng.integers(30, 40))
            length = rng.random() < 0.2
            thr = float(rng.integers(2, 60)) if length else (
                float(rng.integers(0, 3)) * 0.5 if rng.random() < 0.2 else float(rng.random()))
            c1 = ctypes.c_uint64(0)
            c2 = ctypes.c_uint64(0)
            if length:
                a = L.oracle_eval_min_match_len(b, len(b), ctypes.byref(f.bf), int(thr),
                                                ctypes.byref(c1))
            else:
                a = L.oracle_eval_simple(b, len(b), ctypes.byref(f.bf), thr, streak,
                                         ctypes.byref(c1))
            m_ = model.model_eval(b, len(b), ctypes.byref(f.bf), thr, streak,
                                  ol.LENGTH if length else ol.SIMPLE, ctypes.byref(c2))
            if a != m_ or c1.value != c2.value:
                mism += 1
    assert mism == 0


@pytest.mark.parametrize("seed", range(4))
def test_sequential_walk_matches_oracle_harmonic_binomial(model, seed):
    """HARMONIC (the chunked sequential walk, seq_chunk) and BINOMIAL (the
    SIMPLE chunk machine with integer hits, both step policies) give the
    oracle's decision and algorithmic probe count."""
    rng = np.random.default_rng(100 + seed)
    L = ol.lib()
    acgt = np.frombuffer(b"ACGT", dtype=np.uint8)
    mism = 0
    for trial in range(30):
        h = int(rng.integers(1, 5))
        k = max(h, int(rng.integers(3, 40)))
        f = ol.Filter.create(64 * int(rng.integers(1, 60)), h, k)
        g = rng.choice(acgt, 3000)
        fill = rng.random()
        for p, hv in ol.kmers(g.tobytes(), h, k):
            if rng.random() < fill:
                L.oracle_bf_insert(ctypes.byref(f.bf), (ctypes.c_uint64 * 64)(*hv))
        fpr = L.oracle_bf_fpr(ctypes.byref(f.bf))
        for r in range(50):
            n = int(rng.integers(0, 500))
            st = int(rng.integers(0, 2500))
            s = g[st:st + n].copy() if rng.random() < 0.6 else rng.choice(acgt, n)
            s = s[:n]
            m = rng.random(len(s)) < rng.random() * 0.05
            s[m] = rng.choice(acgt, m.sum())
            if rng.random() < 0.3:
                m = rng.random(len(s)) < rng.random() * 0.2
                s[m] = ord("N")
            b = s.tobytes()
            streak = int(rng.integers(0, 6))
            c1 = ctypes.c_uint64(0)
            c2 = ctypes.c_uint64(0)
            if rng.random() < 0.5:
                thr = float(rng.random())
                a = L.oracle_eval_harmonic(b, len(b), ctypes.byref(f.bf), thr, streak,
                                           ctypes.byref(c1))
                mode = ol.HARMONIC
            else:
                thr = 10.0 ** (-float(rng.uniform(1, 100)) / 10.0)
                a = L.oracle_eval_binomial(b, len(b), ctypes.byref(f.bf), thr, fpr, streak,
                                           ctypes.byref(c1))
                mode = ol.BINOMIAL
            m_ = model.model_eval(b, len(b), ctypes.byref(f.bf), thr, streak, mode,
                                  ctypes.byref(c2))
            if a != m_ or c1.value != c2.value:
                mism += 1
    assert mism == 0


@pytest.mark.parametrize("seed", range(4))
def test_score_walk_matches_oracle(model, seed):
    """The scoring kernels' chunked walk (score_chunk) against the oracle's
    evalScore restatement, bit for bit, for all four scoring methods."""
    model.model_score.restype = ctypes.c_double
    model.model_score.argtypes = [ctypes.c_char_p, ctypes.c_uint64, ctypes.POINTER(ol._BF),
                                  ctypes.c_int, ctypes.c_uint, ctypes.c_double]
    rng = np.random.default_rng(200 + seed)
    L = ol.lib()
    acgt = np.frombuffer(b"ACGT", dtype=np.uint8)
    bad = 0
    for trial in range(25):
        h = int(rng.integers(1, 5))
        k = max(h, int(rng.integers(3, 40)))
        f = ol.Filter.create(64 * int(rng.integers(1, 60)), h, k)
        g = rng.choice(acgt, 3000)
        fill = rng.random()
        for p, hv in ol.kmers(g.tobytes(), h, k):
            if rng.random() < fill:
                L.oracle_bf_insert(ctypes.byref(f.bf), (ctypes.c_uint64 * 64)(*hv))
        fpr = L.oracle_bf_fpr(ctypes.byref(f.bf))
        for r in range(40):
            n = int(rng.integers(0, 500))
            st = int(rng.integers(0, 2500))
            s = g[st:st + n].copy() if rng.random() < 0.6 else rng.choice(acgt, n)
            s = s[:n]
            m = rng.random(len(s)) < rng.random() * 0.05
            s[m] = rng.choice(acgt, m.sum())
            if rng.random() < 0.3:
                m = rng.random(len(s)) < rng.random() * 0.2
                s[m] = ord("N")
            b = s.tobytes()
            streak = int(rng.integers(0, 6))
            for mode in (ol.SIMPLE, ol.LENGTH, ol.HARMONIC, ol.BINOMIAL):
                want = L.oracle_eval_score(b, len(b), ctypes.byref(f.bf), mode, streak, fpr)
                got = model.model_score(b, len(b), ctypes.byref(f.bf), mode, streak, fpr)
                if np.float64(want).view(np.uint64) != np.float64(got).view(np.uint64):
                    bad += 1
    assert bad == 0
