"""ctypes access to the CPU oracle (oracle/_build/liboracle.so).

Test infrastructure only: tests/, __graft_entry__.smoke() and bench.py's
CPU-baseline leg use this module to compare results with; the product path
never does.
"""
import ctypes
import os
import subprocess

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_PATH = os.path.join(ROOT, "oracle", "_build", "liboracle.so")

SIMPLE = 0
LENGTH = 1
HARMONIC = 2
BINOMIAL = 3


class _BF(ctypes.Structure):
    _fields_ = [("m", ctypes.c_uint64), ("h", ctypes.c_uint), ("k", ctypes.c_uint),
                ("dfpr", ctypes.c_double), ("n_entry", ctypes.c_uint64),
                ("t_entry", ctypes.c_uint64), ("bits", ctypes.POINTER(ctypes.c_uint8))]


class _Itr(ctypes.Structure):
    _fields_ = [("seq", ctypes.c_char_p), ("len", ctypes.c_size_t), ("k", ctypes.c_uint),
                ("h", ctypes.c_uint), ("pos", ctypes.c_size_t), ("fh", ctypes.c_uint64),
                ("rh", ctypes.c_uint64), ("hv", ctypes.c_uint64 * 64)]


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            subprocess.run(["make", "-C", os.path.join(ROOT, "oracle")], check=True,
                           capture_output=True)
        L = ctypes.CDLL(LIB_PATH)
        P = ctypes.POINTER
        u64, u32, dbl, sz = ctypes.c_uint64, ctypes.c_uint, ctypes.c_double, ctypes.c_size_t
        L.oracle_nt_forward.restype = u64
        L.oracle_nt_forward.argtypes = [ctypes.c_char_p, u32]
        L.oracle_nt_reverse.restype = u64
        L.oracle_nt_reverse.argtypes = [ctypes.c_char_p, u32]
        L.oracle_nt_extra.restype = u64
        L.oracle_nt_extra.argtypes = [u64, u32, u32]
        L.oracle_ntitr_init.argtypes = [P(_Itr), ctypes.c_char_p, sz, u32, u32]
        L.oracle_ntitr_next.argtypes = [P(_Itr)]
        L.oracle_bf_create.argtypes = [P(_BF), u64, u32, u32]
        L.oracle_bf_free.argtypes = [P(_BF)]
        L.oracle_bf_contains.argtypes = [P(_BF), P(u64), P(u64)]
        L.oracle_bf_insert.argtypes = [P(_BF), P(u64)]
        L.oracle_bf_store.argtypes = [P(_BF), ctypes.c_char_p]
        L.oracle_bf_load.argtypes = [P(_BF), ctypes.c_char_p]
        L.oracle_calc_optimal_size.restype = u64
        L.oracle_calc_optimal_size.argtypes = [u64, dbl, u32]
        L.oracle_calc_optimal_hash_num.restype = u32
        L.oracle_calc_optimal_hash_num.argtypes = [dbl]
        L.oracle_make_filter.argtypes = [P(_BF), P(ctypes.c_char_p), P(u64), sz, u32, dbl,
                                         u32, P(u64), P(u64)]
        L.oracle_write_info.argtypes = [ctypes.c_char_p, ctypes.c_char_p, u32, dbl, u32, u64,
                                        ctypes.c_char_p, u64, u64, dbl, u64, dbl]
        L.oracle_eval_simple.argtypes = [ctypes.c_char_p, sz, P(_BF), dbl, u32, P(u64)]
        L.oracle_eval_min_match_len.argtypes = [ctypes.c_char_p, sz, P(_BF), u32, P(u64)]
        L.oracle_eval_harmonic.argtypes = [ctypes.c_char_p, sz, P(_BF), dbl, u32, P(u64)]
        L.oracle_eval_binomial.argtypes = [ctypes.c_char_p, sz, P(_BF), dbl, dbl, u32, P(u64)]
        L.oracle_bf_fpr.restype = dbl
        L.oracle_bf_fpr.argtypes = [P(_BF)]
        L.oracle_calc_min_count.restype = u32
        L.oracle_calc_min_count.argtypes = [u32, dbl, dbl]
        L.oracle_classify.argtypes = [ctypes.c_char_p, P(u64), sz, P(P(_BF)), u32, dbl, u32,
                                      ctypes.c_int, P(u64), P(u64)]
        L.oracle_sdust.restype = ctypes.c_int
        L.oracle_sdust.argtypes = [ctypes.c_char_p, sz, ctypes.c_int, ctypes.c_int, P(u64),
                                   ctypes.c_int, P(ctypes.c_int)]
        L.oracle_set_dust.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int]
        L.oracle_binom_sf.restype = dbl
        L.oracle_binom_sf.argtypes = [u32, dbl, u32]
        L.oracle_eval_score.restype = dbl
        L.oracle_eval_score.argtypes = [ctypes.c_char_p, sz, P(_BF), ctypes.c_int, u32, dbl]
        L.oracle_classify_scores.argtypes = [ctypes.c_char_p, P(u64), sz, P(P(_BF)), u32,
                                             ctypes.c_int, u32, P(dbl)]
        L.oracle_best_hit.restype = dbl
        L.oracle_best_hit.argtypes = [P(dbl), u32, P(u64)]
        L.oracle_ordered.argtypes = [P(u64), P(u64), u32, ctypes.c_int]
        L.oracle_update_summary.restype = u32
        L.oracle_update_summary.argtypes = [P(u64), u32, P(u64)]
        L.oracle_update_summary_pair.restype = u32
        L.oracle_update_summary_pair.argtypes = [P(u64), u32, P(u64), P(u64), ctypes.c_int]
        L.oracle_summary_tsv.restype = sz
        L.oracle_summary_tsv.argtypes = [P(u64), u32, P(ctypes.c_char_p), u64, ctypes.c_char_p,
                                         sz]
        _lib = L
    return _lib


def _u64p(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64))


class Filter:
    """A Bloom filter held by the oracle."""

    def __init__(self):
        self.bf = _BF()
        self._owned = False

    @classmethod
    def create(cls, m, h, k):
        f = cls()
        if lib().oracle_bf_create(ctypes.byref(f.bf), m, h, k):
            raise MemoryError
        f._owned = True
        return f

    @classmethod
    def load(cls, path):
        f = cls()
        rc = lib().oracle_bf_load(ctypes.byref(f.bf), path.encode())
        if rc:
            raise IOError(f"oracle_bf_load({path}) = {rc}")
        f._owned = True
        return f

    @classmethod
    def make(cls, seqs, k=25, fpr=0.075, h=0):
        f = cls()
        arr = (ctypes.c_char_p * len(seqs))(*seqs)
        lens = np.array([len(s) for s in seqs], dtype=np.uint64)
        exp = ctypes.c_uint64()
        red = ctypes.c_uint64()
        if lib().oracle_make_filter(ctypes.byref(f.bf), arr, _u64p(lens), len(seqs), k, fpr, h,
                                    ctypes.byref(exp), ctypes.byref(red)):
            raise MemoryError
        f._owned = True
        f.expected_entries = exp.value
        f.redundant = red.value
        return f

    def __del__(self):
        if getattr(self, "_owned", False) and _lib is not None:
            _lib.oracle_bf_free(ctypes.byref(self.bf))

    @property
    def m(self):
        return self.bf.m

    @property
    def h(self):
        return self.bf.h

    @property
    def k(self):
        return self.bf.k

    def bits(self):
        return np.ctypeslib.as_array(self.bf.bits, shape=(self.bf.m // 8,)).copy()

    def store(self, path):
        if lib().oracle_bf_store(ctypes.byref(self.bf), path.encode()):
            raise IOError(path)

    def insert_sequence(self, seq):
        for _, hv in kmers(seq, self.h, self.k):
            arr = (ctypes.c_uint64 * 64)(*hv)
            lib().oracle_bf_insert(ctypes.byref(self.bf), arr)

    def contains_kmer(self, kmer):
        for _, hv in kmers(kmer, self.h, self.k):
            arr = (ctypes.c_uint64 * 64)(*hv)
            return bool(lib().oracle_bf_contains(ctypes.byref(self.bf), arr, None))
        return False


def write_info(path, fid, k, fpr, h, expected, sources, size, num_entries, approx_fpr,
               redundant, redundant_fpr):
    lib().oracle_write_info(path.encode(), fid.encode(), k, fpr, h, expected, sources.encode(),
                            size, num_entries, approx_fpr, redundant, redundant_fpr)


def kmers(seq, h, k):
    """(pos, hashes) of every valid k-mer, via the oracle's iterator."""
    it = _Itr()
    buf = ctypes.create_string_buffer(seq, len(seq))
    lib().oracle_ntitr_init(ctypes.byref(it), buf, len(seq), h, k)
    out = []
    while it.pos != 2**64 - 1:
        out.append((it.pos, list(it.hv[:max(h, 1)])))
        lib().oracle_ntitr_next(ctypes.byref(it))
    return out


def pack_reads(seqs):
    """Concatenate byte strings; returns (bytes, uint64 offsets)."""
    off = np.zeros(len(seqs) + 1, dtype=np.uint64)
    off[1:] = np.cumsum([len(s) for s in seqs])
    return b"".join(seqs), off


def classify(seq_bytes, offsets, filters, threshold=0.15, streak=3, scoring=SIMPLE,
             count_probes=False):
    """Per-read hit bitmasks (n x words uint64) and the algorithmic probe count."""
    n = len(offsets) - 1
    nf = len(filters)
    words = (nf + 63) // 64
    hits = np.zeros((n, words), dtype=np.uint64)
    arr = (ctypes.POINTER(_BF) * nf)(*[ctypes.pointer(f.bf) for f in filters])
    probes = ctypes.c_uint64(0)
    off = np.ascontiguousarray(offsets, dtype=np.uint64)
    lib().oracle_classify(seq_bytes, _u64p(off), n, arr, nf, threshold, streak, scoring,
                          _u64p(hits), ctypes.byref(probes) if count_probes else None)
    return hits, probes.value


def sdust(seq, T=20, W=64):
    """Masked intervals [(start, finish)] of one sequence (Common/sdust.c) and
    the largest number of pending perfect intervals held at once."""
    cap = len(seq) + 16
    buf = np.zeros(cap, dtype=np.uint64)
    mp = ctypes.c_int(0)
    n = lib().oracle_sdust(seq, len(seq), T, W, _u64p(buf), cap, ctypes.byref(mp))
    return [(int(v) >> 32, int(v) & 0xffffffff) for v in buf[:n]], mp.value


class dust:
    """Context manager: the oracle's evaluations mask low-complexity frames
    (-D) inside the block."""

    def __init__(self, T=20, W=64):
        self.T, self.W = T, W

    def __enter__(self):
        lib().oracle_set_dust(1, self.T, self.W)
        return self

    def __exit__(self, *a):
        lib().oracle_set_dust(0, 20, 64)


def classify_scores(seq_bytes, offsets, filters, scoring=SIMPLE, streak=3):
    """SeqEval::evalScore of every read against every filter: (n, nf) float64."""
    n = len(offsets) - 1
    nf = len(filters)
    out = np.zeros((n, nf), dtype=np.float64)
    arr = (ctypes.POINTER(_BF) * nf)(*[ctypes.pointer(f.bf) for f in filters])
    off = np.ascontiguousarray(offsets, dtype=np.uint64)
    lib().oracle_classify_scores(seq_bytes, _u64p(off), n, arr, nf, scoring, streak,
                                 out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
    return out


def best_hit(scores):
    """evaluateReadBestHit over (n, nf) scores: hit words (n, words) and the
    largest score per read."""
    n, nf = scores.shape
    words = (nf + 63) // 64
    hits = np.zeros((n, words), dtype=np.uint64)
    best = np.zeros(n, dtype=np.float64)
    for i in range(n):
        row = np.ascontiguousarray(scores[i])
        h = np.zeros(words, dtype=np.uint64)
        best[i] = lib().oracle_best_hit(row.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), nf,
                                        _u64p(h))
        hits[i] = h
    return hits, best


def ordered(hits, nf, hits2=None, inclusive=False):
    """evaluateReadOrdered(Pair) from STD hit words; returns new arrays."""
    h1 = np.array(hits, dtype=np.uint64, copy=True)
    h2 = None if hits2 is None else np.array(hits2, dtype=np.uint64, copy=True)
    for i in range(len(h1)):
        r1 = np.ascontiguousarray(h1[i])
        r2 = None if h2 is None else np.ascontiguousarray(h2[i])
        lib().oracle_ordered(_u64p(r1), None if r2 is None else _u64p(r2), nf, int(inclusive))
        h1[i] = r1
        if h2 is not None:
            h2[i] = r2
    return h1, h2


def summary_counts(hits, nf, hits2=None, inclusive=False):
    counts = np.zeros(2 * (nf + 2) + 2, dtype=np.uint64)
    cats = np.zeros(len(hits), dtype=np.uint32)
    for i in range(len(hits)):
        row = np.ascontiguousarray(hits[i])
        if hits2 is None:
            cats[i] = lib().oracle_update_summary(_u64p(counts), nf, _u64p(row))
        else:
            row2 = np.ascontiguousarray(hits2[i])
            cats[i] = lib().oracle_update_summary_pair(_u64p(counts), nf, _u64p(row), _u64p(row2),
                                                       int(inclusive))
    return counts, cats


def summary_tsv(counts, ids, read_count):
    nf = len(ids)
    arr = (ctypes.c_char_p * nf)(*[i.encode() for i in ids])
    cap = 1 << 20
    buf = ctypes.create_string_buffer(cap)
    n = lib().oracle_summary_tsv(_u64p(np.ascontiguousarray(counts, dtype=np.uint64)), nf, arr,
                                 read_count, buf, cap)
    return buf.raw[:n].decode()


# ---------------------------------------------------------------- miBF oracle

class _MIBF(ctypes.Structure):
    _fields_ = [("m", ctypes.c_uint64), ("h", ctypes.c_uint), ("k", ctypes.c_uint),
                ("nseeds", ctypes.c_uint), ("seeds", (ctypes.c_char * 256) * 16),
                ("bv", ctypes.POINTER(ctypes.c_uint64)),
                ("rank_word", ctypes.POINTER(ctypes.c_uint64)),
                ("ids", ctypes.POINTER(ctypes.c_uint16)), ("pop", ctypes.c_uint64)]


class _QRes(ctypes.Structure):
    _fields_ = [("id", ctypes.c_uint16), ("nonSatFrameCount", ctypes.c_uint32),
                ("solidCount", ctypes.c_uint32), ("count", ctypes.c_uint32),
                ("nonSatCount", ctypes.c_uint32), ("totalNonSatCount", ctypes.c_uint32),
                ("totalCount", ctypes.c_uint32)]


_mibf_sig_done = False


def _mibf_lib():
    global _mibf_sig_done
    L = lib()
    if not _mibf_sig_done:
        P = ctypes.POINTER
        L.oracle_mibf_build.argtypes = [P(_MIBF), P(ctypes.c_char_p), P(ctypes.c_uint64),
                                        P(ctypes.c_uint16), ctypes.c_size_t,
                                        P(ctypes.c_char_p), ctypes.c_uint, ctypes.c_uint,
                                        ctypes.c_uint, ctypes.c_double]
        L.oracle_mibf_free.argtypes = [P(_MIBF)]
        L.oracle_mibf_store.argtypes = [P(_MIBF), ctypes.c_char_p]
        L.oracle_mibf_load.argtypes = [P(_MIBF), ctypes.c_char_p]
        L.oracle_mibf_frame_probs.restype = ctypes.c_double
        L.oracle_mibf_frame_probs.argtypes = [P(_MIBF), P(ctypes.c_double), ctypes.c_uint,
                                              ctypes.c_uint]
        L.oracle_mibf_query.restype = ctypes.c_uint
        L.oracle_mibf_query.argtypes = [P(_MIBF), ctypes.c_char_p, ctypes.c_size_t,
                                        ctypes.c_char_p, ctypes.c_size_t, P(ctypes.c_uint32),
                                        ctypes.c_uint, ctypes.c_double, ctypes.c_uint,
                                        ctypes.c_uint, ctypes.c_int, P(_QRes), ctypes.c_uint,
                                        P(ctypes.c_uint32), P(ctypes.c_uint64)]
        L.oracle_binom_upper_quantile.restype = ctypes.c_uint
        L.oracle_binom_upper_quantile.argtypes = [ctypes.c_uint, ctypes.c_double,
                                                  ctypes.c_double]
        L.oracle_st_hash.restype = ctypes.c_uint64
        L.oracle_st_hash.argtypes = [ctypes.c_char_p, ctypes.c_uint, ctypes.c_char_p]
        _mibf_sig_done = True
    return L


class MIBF:
    """A multi-index Bloom filter held by the oracle."""

    def __init__(self):
        self.f = _MIBF()
        self._owned = False

    @classmethod
    def build(cls, seqs, ids, seeds=None, k=25, h=3, occupancy=0.5):
        L = _mibf_lib()
        o = cls()
        arr = (ctypes.c_char_p * len(seqs))(*seqs)
        lens = np.array([len(s) for s in seqs], dtype=np.uint64)
        idv = np.array(ids, dtype=np.uint16)
        sarr = (ctypes.c_char_p * max(1, len(seeds or [])))(*[s.encode() for s in seeds or []])
        kk = len(seeds[0]) if seeds else k
        rc = L.oracle_mibf_build(ctypes.byref(o.f), arr, _u64p(lens),
                                 idv.ctypes.data_as(ctypes.POINTER(ctypes.c_uint16)), len(seqs),
                                 sarr, len(seeds or []), kk, h, occupancy)
        if rc:
            raise RuntimeError(f"oracle_mibf_build = {rc}")
        o._owned = True
        return o

    @classmethod
    def load(cls, path):
        o = cls()
        rc = _mibf_lib().oracle_mibf_load(ctypes.byref(o.f), path.encode())
        if rc:
            raise IOError(f"oracle_mibf_load({path}) = {rc}")
        o._owned = True
        return o

    def __del__(self):
        if getattr(self, "_owned", False) and _lib is not None:
            _lib.oracle_mibf_free(ctypes.byref(self.f))

    def store(self, prefix):
        if _mibf_lib().oracle_mibf_store(ctypes.byref(self.f), prefix.encode()):
            raise IOError(prefix)

    def frame_probs(self, nids, allowed_miss):
        probs = np.zeros(nids, dtype=np.float64)
        sat = _mibf_lib().oracle_mibf_frame_probs(
            ctypes.byref(self.f), probs.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), nids,
            allowed_miss)
        return probs, sat

    def bits(self):
        return np.ctypeslib.as_array(self.f.bv, shape=(self.f.m // 64,)).copy()

    def ids(self):
        return np.ctypeslib.as_array(self.f.ids, shape=(self.f.pop,)).copy()

    def query(self, seq, min_count, seq2=None, multi=1.0, allowed_miss=2, min_nonsat=0,
              best_agree=False):
        L = _mibf_lib()
        nids = len(min_count)
        mc = np.ascontiguousarray(min_count, dtype=np.uint32)
        out = (_QRes * max(1, nids))()
        sat = ctypes.c_uint32()
        n = L.oracle_mibf_query(ctypes.byref(self.f), seq, len(seq), seq2,
                                len(seq2) if seq2 is not None else 0,
                                mc.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)), nids, multi,
                                allowed_miss, min_nonsat, int(best_agree), out, max(1, nids),
                                ctypes.byref(sat), None)
        res = [(r.id, r.nonSatFrameCount, r.solidCount, r.count, r.nonSatCount,
                r.totalNonSatCount, r.totalCount) for r in out[:n]]
        return res, sat.value


def binom_upper_quantile(n, p, q):
    return _mibf_lib().oracle_binom_upper_quantile(n, p, q)


# ------------------------------------------------- workload generator (CPU arm)

class ReadParams(ctypes.Structure):
    """oracle_read_params: the field layout of the product's bbt_synth_read_params."""
    _fields_ = [("len_min", ctypes.c_uint32), ("len_max", ctypes.c_uint32),
                ("long_frac", ctypes.c_double), ("long_min", ctypes.c_uint32),
                ("long_max", ctypes.c_uint32), ("sub_rate", ctypes.c_double),
                ("n_rate", ctypes.c_double), ("frag_min", ctypes.c_uint32),
                ("frag_max", ctypes.c_uint32)]


_synth_sig_done = False


def _synth_lib():
    global _synth_sig_done
    L = lib()
    if not _synth_sig_done:
        P = ctypes.POINTER
        u64, u32, dbl, vp = ctypes.c_uint64, ctypes.c_uint32, ctypes.c_double, ctypes.c_void_p
        L.oracle_synth_genome.argtypes = [u64, u64, dbl, dbl, u32, u32, dbl, dbl, vp]
        L.oracle_synth_read_lengths.argtypes = [u64, P(ReadParams), u64, vp]
        L.oracle_synth_reads.argtypes = [u64, vp, vp, u32, vp, P(ReadParams), u64, vp, vp, vp,
                                         vp]
        L.oracle_make_filter_par.argtypes = [P(_BF), P(ctypes.c_char_p), P(u64), ctypes.c_size_t,
                                             u32, dbl, u32, P(u64), P(u64)]
        _synth_sig_done = True
    return L


def _vp(a):
    return ctypes.c_void_p(a.ctypes.data) if a is not None else None


def synth_genome(seed, length, gc=0.5, repeat_frac=0.0, rep_min=0, rep_max=0, div_min=0.0,
                 div_max=0.0):
    out = np.empty(int(length), dtype=np.uint8)
    if _synth_lib().oracle_synth_genome(seed, int(length), gc, repeat_frac, rep_min, rep_max,
                                        div_min, div_max, _vp(out)):
        raise ValueError("oracle_synth_genome: bad arguments")
    return out


def read_params(len_min=150, len_max=None, long_frac=0.0, long_min=0, long_max=0, sub_rate=0.0,
                n_rate=0.0, frag_min=0, frag_max=0):
    return ReadParams(len_min, len_max if len_max is not None else len_min, long_frac, long_min,
                      long_max, sub_rate, n_rate, frag_min, frag_max)


def synth_reads(seed, refs, ref_frac, n_reads, params, paired=False):
    """(seq1, off, seq2 or None, src), as the product's synth.reads."""
    L = _synth_lib()
    off = np.empty(n_reads + 1, dtype=np.uint64)
    if L.oracle_synth_read_lengths(seed, ctypes.byref(params), n_reads, _vp(off)):
        raise ValueError("oracle_synth_read_lengths: bad arguments")
    total = int(off[-1])
    s1 = np.empty(max(total, 1), dtype=np.uint8)
    s2 = np.empty(max(total, 1), dtype=np.uint8) if paired else None
    src = np.empty(n_reads, dtype=np.uint32)
    if refs:
        cat = np.concatenate(refs) if len(refs) > 1 else np.ascontiguousarray(refs[0])
        roff = np.zeros(len(refs) + 1, dtype=np.uint64)
        roff[1:] = np.cumsum([len(r) for r in refs])
    else:
        cat = np.zeros(1, dtype=np.uint8)
        roff = np.zeros(1, dtype=np.uint64)
    frac = np.asarray(ref_frac, dtype=np.float64)
    if L.oracle_synth_reads(seed, _vp(cat), _vp(roff), len(refs), _vp(frac),
                            ctypes.byref(params), n_reads, _vp(off), _vp(s1), _vp(s2),
                            _vp(src)):
        raise ValueError("oracle_synth_reads: a reference is shorter than a fragment")
    return s1, off, s2, src


def make_filter_par(seqs, k=25, fpr=0.075, h=0):
    """Filter from uint8 arrays, built by the oracle's OpenMP threads (same bit
    array as Filter.make)."""
    L = _synth_lib()
    f = Filter()
    ptrs = (ctypes.c_char_p * len(seqs))(*[ctypes.cast(s.ctypes.data, ctypes.c_char_p)
                                           for s in seqs])
    lens = np.array([len(s) for s in seqs], dtype=np.uint64)
    exp = ctypes.c_uint64()
    red = ctypes.c_uint64()
    if L.oracle_make_filter_par(ctypes.byref(f.bf), ptrs, _u64p(lens), len(seqs), k, fpr, h,
                                ctypes.byref(exp), ctypes.byref(red)):
        raise MemoryError
    f._owned = True
    f.expected_entries = exp.value
    f.redundant = red.value
    return f
