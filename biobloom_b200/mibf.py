"""Python mirror of MIBFClassifier (BioBloomCategorizer/MIBFClassifier.hpp)
over the miBF C ABI of libbbt.so (include/bbt_mibf.h).

    mc = MIBFClassifier("targets.bf")                 # targets_ids.txt, targets.sdsl
    mc.filter(["reads.fq"], prefix="out")             # records to stdout, out_summary.tsv
    mc.filterPair("r1.fq", "r2.fq", prefix="out")
    results, sat = mc.classify([b"ACGT...", ...])     # in-memory batch

Every classification runs on the GPU; there is no CPU fallback.
``MIBFClassifier(..., host_only=True)`` loads only the host-side parts (names,
frame probabilities, minCount, record formatting) and needs no GPU.
"""
import ctypes
import math

import numpy as np

from . import _lib as L
from .classifier import _ptr, pack

HIT_FIELDS = ("id", "nonSatFrameCount", "solidCount", "count", "nonSatCount",
              "totalNonSatCount", "totalCount")
_HIT_DTYPE = np.dtype([(f, np.uint32) for f in HIT_FIELDS])


def min_fpr_to_score(min_fpr):
    """-s N of biobloommicategorizer: score = 10^(-N/10) (BioBloomMICategorizer.cpp:168-173)."""
    return math.pow(10.0, -(float(min_fpr) / 10.0))


class MIBFClassifier:
    def __init__(self, filter_file, *, score=1e-10, frame_matches=1, multi=1.0, streak=3,
                 min_nonsat=0, best_hit_agree=False, hit_only=False, device=0,
                 host_only=False, layout=L.MIBF_LAYOUT_AUTO):
        lib = L.lib()
        p = L.MibfParams()
        lib.bbt_mibf_default_params(ctypes.byref(p))
        p.score = float(score)
        p.frame_matches = int(frame_matches)
        p.multi_thresh = float(multi)
        p.streak = int(streak)
        p.min_nonsat = int(min_nonsat)
        p.best_hit_agree = int(bool(best_hit_agree))
        p.hit_only = int(bool(hit_only))
        p.device = int(device)
        p.layout = int(layout)
        ctx = ctypes.c_void_p()
        opener = lib.bbt_mibf_open_host if host_only else lib.bbt_mibf_open
        L.check_mibf(opener(str(filter_file).encode(), ctypes.byref(p), ctypes.byref(ctx)))
        self._ctx = ctx
        self.params = p
        self.host_only = host_only
        self.num_ids = lib.bbt_mibf_num_ids(ctx)
        self.names = [lib.bbt_mibf_id_name(ctx, i).decode() for i in range(self.num_ids)]
        m, h, k, ns = ctypes.c_uint64(), ctypes.c_uint(), ctypes.c_uint(), ctypes.c_uint()
        lib.bbt_mibf_info(ctx, ctypes.byref(m), ctypes.byref(h), ctypes.byref(k), ctypes.byref(ns))
        self.m, self.h, self.k, self.n_seeds = m.value, h.value, k.value, ns.value
        self.layout = None if host_only else lib.bbt_mibf_layout(ctx)

    # -- host-side pieces ------------------------------------------------------
    def frame_probs(self):
        probs = np.zeros(self.num_ids, dtype=np.float64)
        rate = ctypes.c_double()
        L.check_mibf(L.lib().bbt_mibf_frame_probs(
            self._ctx, probs.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), ctypes.byref(rate)),
            self._ctx)
        return probs, rate.value

    def min_counts(self, frame_count):
        """getMinCount for every ID (index 0 unused)."""
        probs, _ = self.frame_probs()
        return [0] + [L.lib().bbt_mibf_min_count(frame_count, float(probs[i]), self.params.score,
                                                 self.num_ids) for i in range(1, self.num_ids)]

    def format_record(self, name, comment, seq, qual, hits, sat_count, out_type=L.MIBF_OUT_TSV):
        """formatOutStr for one read; hits = list of 7-tuples in HIT_FIELDS order."""
        arr = (L.MibfHit * max(1, len(hits)))()
        for i, t in enumerate(hits):
            for f, v in zip(HIT_FIELDS, t):
                setattr(arr[i], f, int(v))
        n = ctypes.c_size_t()
        args = [self._ctx, out_type, name.encode(), comment.encode() if comment else None,
                seq if seq is not None else None, qual if qual is not None else None, arr,
                len(hits), int(sat_count)]
        L.check_mibf(L.lib().bbt_mibf_format_record(*args, None, 0, ctypes.byref(n)), self._ctx)
        buf = ctypes.create_string_buffer(n.value + 1)
        L.check_mibf(L.lib().bbt_mibf_format_record(*args, buf, n.value + 1, ctypes.byref(n)),
                     self._ctx)
        return buf.raw[:n.value].decode()

    # -- classification --------------------------------------------------------
    def classify(self, reads, reads2=None, max_hits=8):
        """Classify host reads (list of bytes, or (uint8 array, uint64 offsets)).
        Returns (results, sat_count): results[i] is the list of 7-tuples
        (HIT_FIELDS) of read (pair) i in result order."""
        seq, off = pack(reads) if isinstance(reads, list) else reads
        seq = np.ascontiguousarray(seq, dtype=np.uint8)
        off = np.ascontiguousarray(off, dtype=np.uint64)
        n = len(off) - 1
        b = L.Batch()
        b.seq, b.offsets, b.n_reads, b.location = _ptr(seq), _ptr(off), n, L.HOST
        if reads2 is not None:
            seq2, off2 = pack(reads2) if isinstance(reads2, list) else reads2
            seq2 = np.ascontiguousarray(seq2, dtype=np.uint8)
            off2 = np.ascontiguousarray(off2, dtype=np.uint64)
            if len(off2) - 1 != n:
                raise ValueError("mate arrays differ in length")
            b.seq2, b.offsets2 = _ptr(seq2), _ptr(off2)
        mh = max(1, min(int(max_hits), self.num_ids))
        while True:
            hits = np.zeros((max(n, 1), mh), dtype=_HIT_DTYPE)
            nh = np.zeros(max(n, 1), dtype=np.uint32)
            sat = np.zeros(max(n, 1), dtype=np.uint32)
            r = L.MibfResult()
            r.hits, r.max_hits, r.n_hits, r.sat_count, r.location = (
                _ptr(hits), mh, _ptr(nh), _ptr(sat), L.HOST)
            rc = L.lib().bbt_mibf_classify_batch(self._ctx, ctypes.byref(b), ctypes.byref(r), None)
            if rc == L.ERR_OVERFLOW and mh < self.num_ids:
                mh = self.num_ids
                continue
            L.check_mibf(rc, self._ctx)
            break
        out = []
        for i in range(n):
            out.append([tuple(int(x) for x in hits[i, j]) for j in range(int(nh[i]))])
        return out, sat[:n].copy()

    def classify_device(self, seq, off, seq2=None, off2=None, max_hits=8, stream=None, out=None):
        """Classify reads resident on the GPU (torch uint8 / int64 tensors).
        Enqueued on `stream` (default: the current stream).  Returns
        (hits [n, max_hits, 7] int32 tensor, n_hits, sat_count); `out` may
        pass those three tensors in to be filled."""
        import torch
        n = off.numel() - 1
        dev = seq.device
        if out is not None:
            hits, nh, sat = out
            max_hits = hits.shape[1]
        else:
            hits = torch.zeros((max(n, 1), max_hits, 7), dtype=torch.int32, device=dev)
            nh = torch.zeros(max(n, 1), dtype=torch.int32, device=dev)
            sat = torch.zeros(max(n, 1), dtype=torch.int32, device=dev)
        b = L.Batch()
        b.seq, b.offsets, b.n_reads, b.location = seq.data_ptr(), off.data_ptr(), n, L.DEVICE
        if seq2 is not None:
            b.seq2, b.offsets2 = seq2.data_ptr(), off2.data_ptr()
        r = L.MibfResult()
        r.hits, r.max_hits, r.n_hits, r.sat_count, r.location = (
            hits.data_ptr(), max_hits, nh.data_ptr(), sat.data_ptr(), L.DEVICE)
        s = stream if stream is not None else torch.cuda.current_stream(dev)
        L.check_mibf(L.lib().bbt_mibf_classify_batch(self._ctx, ctypes.byref(b), ctypes.byref(r),
                                                     ctypes.c_void_p(s.cuda_stream)), self._ctx)
        return hits[:n], nh[:n], sat[:n]

    def sync(self):
        L.check_mibf(L.lib().bbt_mibf_sync(self._ctx), self._ctx)

    def set_bucketing(self, mode=None, bucket_shift=0, max_frames=0):
        """Bucketed query of the dense layout (bbt_mibf_set_bucketing): mode 0
        off, 1 on, 2 automatic (None keeps it); 0 keeps the other settings."""
        m = getattr(self, "_bk_mode", 0) if mode is None else mode
        L.check_mibf(L.lib().bbt_mibf_set_bucketing(self._ctx, m, bucket_shift, max_frames),
                     self._ctx)
        self._bk_mode = m

    def last_kernel_ms(self):
        return L.lib().bbt_mibf_last_kernel_ms(self._ctx)

    def last_counts(self):
        """(frames visited, values probed, probes that hit) of the last batch."""
        out = (ctypes.c_uint64 * 3)()
        L.check_mibf(L.lib().bbt_mibf_last_counts(self._ctx, out), self._ctx)
        return tuple(int(x) for x in out)

    # -- file pipeline ---------------------------------------------------------
    def filter(self, input_files, prefix="", out_type=L.MIBF_OUT_TSV, out_path=None):
        """MIBFClassifier::filter: records to out_path (default stdout) and
        <prefix>_summary.tsv."""
        files = [str(f).encode() for f in input_files]
        arr = (ctypes.c_char_p * len(files))(*files)
        return self._with_out(out_path, lambda fp: L.lib().bbt_mibf_filter_files(
            self._ctx, arr, len(files), prefix.encode(), out_type, fp))

    def filterPair(self, file1, file2, prefix="", out_type=L.MIBF_OUT_TSV, out_path=None):
        return self._with_out(out_path, lambda fp: L.lib().bbt_mibf_filter_pair_files(
            self._ctx, str(file1).encode(), str(file2).encode(), prefix.encode(), out_type, fp))

    def _with_out(self, out_path, fn):
        libc = ctypes.CDLL(None)
        libc.fopen.restype = ctypes.c_void_p
        libc.fopen.argtypes = [ctypes.c_char_p, ctypes.c_char_p]
        libc.fclose.argtypes = [ctypes.c_void_p]
        fp = libc.fopen(str(out_path).encode(), b"wb") if out_path else None
        if out_path and not fp:
            raise OSError(f"cannot write {out_path}")
        try:
            L.check_mibf(fn(ctypes.c_void_p(fp) if fp else None), self._ctx)
        finally:
            if fp:
                libc.fclose(fp)

    # -- summary (ResultsManager<ID>) -------------------------------------------
    def summary(self):
        counts = np.zeros(2 * (self.num_ids + 2) + 2, dtype=np.uint64)
        reads = ctypes.c_uint64()
        L.check_mibf(L.lib().bbt_mibf_summary(self._ctx, counts.ctypes.data_as(
            ctypes.POINTER(ctypes.c_uint64)), ctypes.byref(reads)), self._ctx)
        return counts, reads.value

    def summary_tsv(self, read_count=None):
        if read_count is None:
            read_count = self.summary()[1]
        n = ctypes.c_size_t()
        L.check_mibf(L.lib().bbt_mibf_summary_tsv(self._ctx, int(read_count), None, 0,
                                                  ctypes.byref(n)), self._ctx)
        buf = ctypes.create_string_buffer(n.value + 1)
        L.check_mibf(L.lib().bbt_mibf_summary_tsv(self._ctx, int(read_count), buf, n.value + 1,
                                                  ctypes.byref(n)), self._ctx)
        return buf.value.decode()

    def reset_summary(self):
        L.check_mibf(L.lib().bbt_mibf_reset_summary(self._ctx), self._ctx)

    def close(self):
        if getattr(self, "_ctx", None):
            L.lib().bbt_mibf_close(self._ctx)
            self._ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


def make_mibf(prefix, seqs, seq_ids, names, seeds=None, k=25, hash_num=3, occupancy=0.5,
              device=0):
    """Build a miBF on the GPU (bbt_mibf_make) from host sequences; seq_ids[i]
    is sequence i's 1-based target ID, names[id - 1] its name."""
    buf, off = pack(list(seqs))
    sid = np.ascontiguousarray(seq_ids, dtype=np.uint16)
    nm = [n.encode() for n in names]
    narr = (ctypes.c_char_p * len(nm))(*nm)
    seeds = list(seeds or [])
    sarr = (ctypes.c_char_p * max(1, len(seeds)))(*[s.encode() for s in seeds])
    kk = len(seeds[0]) if seeds else int(k)
    L.check_mibf(L.lib().bbt_mibf_make(_ptr(buf), _ptr(off), _ptr(sid), len(seqs), narr, len(nm),
                                       sarr, len(seeds), kk, int(hash_num), float(occupancy),
                                       L.HOST, str(prefix).encode(), int(device)))
