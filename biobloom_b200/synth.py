"""Seeded synthetic genomes, reads and filters (wrappers of the bbt_synth_*
and bbt_make_filter entry points of libbbt.so)."""
import ctypes

import numpy as np

from . import _lib as L


def _vp(a):
    return ctypes.c_void_p(a.ctypes.data) if a is not None else None


def genome(seed, length, gc=0.5, repeat_frac=0.0, rep_min=0, rep_max=0, div_min=0.0,
           div_max=0.0):
    """A random genome (uint8 ASCII array) with optional repeat families."""
    out = np.empty(int(length), dtype=np.uint8)
    L.check(L.lib().bbt_synth_genome(seed, int(length), gc, repeat_frac, rep_min, rep_max,
                                     div_min, div_max, _vp(out)))
    return out


def read_params(len_min=150, len_max=None, long_frac=0.0, long_min=0, long_max=0, sub_rate=0.0,
                n_rate=0.0, frag_min=0, frag_max=0):
    p = L.SynthReadParams()
    p.len_min = len_min
    p.len_max = len_max if len_max is not None else len_min
    p.long_frac, p.long_min, p.long_max = long_frac, long_min, long_max
    p.sub_rate, p.n_rate = sub_rate, n_rate
    p.frag_min, p.frag_max = frag_min, frag_max
    return p


def reads(seed, refs, ref_frac, n_reads, params, paired=False):
    """Reads drawn from refs (list of uint8 arrays) with ref_frac[j] of the
    reads from refs[j] and the rest uniform random.
    Returns (seq1, off, seq2 or None, src)."""
    lib = L.lib()
    off = np.empty(n_reads + 1, dtype=np.uint64)
    L.check(lib.bbt_synth_read_lengths(seed, ctypes.byref(params), n_reads, _vp(off)))
    total = int(off[-1])
    s1 = np.empty(max(total, 1), dtype=np.uint8)
    s2 = np.empty(max(total, 1), dtype=np.uint8) if paired else None
    src = np.empty(n_reads, dtype=np.uint32)
    if refs:
        cat = np.concatenate(refs)
        roff = np.zeros(len(refs) + 1, dtype=np.uint64)
        roff[1:] = np.cumsum([len(r) for r in refs])
    else:
        cat = np.zeros(1, dtype=np.uint8)
        roff = np.zeros(1, dtype=np.uint64)
    frac = np.asarray(ref_frac, dtype=np.float64)
    L.check(lib.bbt_synth_reads(seed, _vp(cat), _vp(roff), len(refs), _vp(frac),
                                ctypes.byref(params), n_reads, _vp(off), _vp(s1), _vp(s2),
                                _vp(src)))
    return s1, off, s2, src


def make_filter(seqs, stem, filter_id, k=25, fpr=0.075, hash_num=0, entries=0, device=0,
                sources=""):
    """Build <stem>.bf / <stem>.txt on the GPU from a list of uint8 arrays."""
    cat = np.concatenate(seqs) if len(seqs) > 1 else np.ascontiguousarray(seqs[0])
    off = np.zeros(len(seqs) + 1, dtype=np.uint64)
    off[1:] = np.cumsum([len(s) for s in seqs])
    L.check(L.lib().bbt_make_filter(ctypes.c_void_p(cat.ctypes.data),
                                    off.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64)),
                                    len(seqs), k, fpr, hash_num, entries, stem.encode(),
                                    filter_id.encode(), sources.encode(), device))
    return stem + ".bf"
