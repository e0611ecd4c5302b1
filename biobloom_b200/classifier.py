"""Python mirror of BioBloomClassifier (BioBloomCategorizer/BioBloomClassifier.h:47-98)
over the C ABI of libbbt.so.

    bbc = BioBloomClassifier(["a.bf", "b.bf"], 0.15, "out")
    bbc.filter(["reads.fq"])                 # writes out_summary.tsv
    bbc.filterPair("r1.fq", "r2.fq")         # paired (intersection of mates)
    bbc.filterPrint(["reads.fq"], "fq")      # also out_<filter>.fq per category
    hits, hits2, cats = bbc.classify([b"ACGT...", ...])  # in-memory batch

Every call goes through the CUDA path; there is no CPU fallback.
"""
import ctypes

import numpy as np

from . import _lib as L


def _ptr(a):
    return ctypes.c_void_p(a.ctypes.data)


def pack(seqs):
    """Concatenate byte strings into (uint8 array, uint64 offsets)."""
    off = np.zeros(len(seqs) + 1, dtype=np.uint64)
    if seqs:
        off[1:] = np.cumsum([len(s) for s in seqs])
    buf = np.frombuffer(b"".join(seqs) or b"\0", dtype=np.uint8)
    return buf, off


class BioBloomClassifier:
    def __init__(self, filter_paths, score_threshold=None, prefix="", postfix="", *,
                 streak_threshold=3, device=0, path=L.PATH_AUTO, warps_per_block=0,
                 frames_per_lane=0, max_batch_reads=0, max_batch_bases=0, l2_fetch_bytes=0,
                 score_type="simple", devices=None, steps=L.STEPS_DECISION):
        """score_type: "simple", "harmonic" or "binomial" (-S); for binomial the
        score is the -s value, the minimum -10*log10(FPR) of a match [100].
        devices: a list of GPU ordinals to load the filters on (bbt_open_devices;
        host batches and files are split across them); default: `device` alone."""
        lib = L.lib()
        p = L.Params()
        lib.bbt_default_params(ctypes.byref(p))
        if score_threshold is None:
            score_threshold = 100 if score_type == "binomial" else 0.15
        p.score = float(score_threshold)
        p.streak_threshold = int(streak_threshold)
        p.device = int(device)
        p.path = int(path)
        p.warps_per_block = int(warps_per_block)
        p.frames_per_lane = int(frames_per_lane)
        p.max_batch_reads = int(max_batch_reads)
        p.max_batch_bases = int(max_batch_bases)
        p.l2_fetch_bytes = int(l2_fetch_bytes)
        # BioBloomCategorizer.cpp:414-441: binomial scores are -10*log10(FPR);
        # otherwise an integer score > 1 is a minimum match length
        if score_type == "binomial":
            p.scoring = L.SCORE_BINOMIAL
            p.score = 10.0 ** (-(float(score_threshold) / 10.0))
        elif int(score_threshold) > 1:
            p.score = float(int(score_threshold))
            p.scoring = L.SCORE_LENGTH
        elif score_type == "harmonic":
            p.scoring = L.SCORE_HARMONIC
        paths = [str(x).encode() for x in filter_paths]
        arr = (ctypes.c_char_p * len(paths))(*paths)
        ctx = ctypes.c_void_p()
        if devices:
            devs = (ctypes.c_int * len(devices))(*[int(d) for d in devices])
            L.check(lib.bbt_open_devices(arr, len(paths), ctypes.byref(p), devs, len(devices),
                                         ctypes.byref(ctx)))
        else:
            L.check(lib.bbt_open(arr, len(paths), ctypes.byref(p), ctypes.byref(ctx)))
        self._ctx = ctx
        self.params = p
        self.prefix = prefix
        self.postfix = postfix
        self.n_filters = lib.bbt_num_filters(ctx)
        self.words = (self.n_filters + 63) // 64
        self.filter_ids = [lib.bbt_filter_id(ctx, i).decode() for i in range(self.n_filters)]
        self._inclusive = False
        self.mode = L.MODE_STD
        if steps:
            self.set_steps(steps)

    # -- reference-style configuration -------------------------------------
    def setInclusive(self):
        """-i: a pair counts for a filter when either mate hits (union);
        BioBloomClassifier::setInclusive (BioBloomClassifier.h:77-79)."""
        L.check(L.lib().bbt_set_inclusive(self._ctx, 1), self._ctx)
        self._inclusive = True

    def setOrderedFilter(self):
        """-c: only the first filter (in load order) that a read passes counts;
        BioBloomClassifier::setOrderedFilter (BioBloomClassifier.h:67-75),
        which refuses best-hit mode."""
        if self.mode == L.MODE_BESTHIT:
            raise L.BBTError(-1,
                             "Best Hit mode and Ordered mode detected. Not yet supported.")
        self.set_mode(L.MODE_ORDERED)

    def setStdout(self, inverse=False):
        """-d (-n): the file pipelines print the first filter's reads (all
        others) to stdout; BioBloomClassifier::setStdout (BioBloomClassifier.h:81-83)."""
        L.check(L.lib().bbt_set_stdout(self._ctx, 1, int(bool(inverse))), self._ctx)

    def set_dust(self, on=True, T=20, W=64):
        """-D (-T, -W): SDUST masking of low-complexity frames before every
        evaluation (opt::dust, Common/SDust.hpp)."""
        L.check(L.lib().bbt_set_dust(self._ctx, int(bool(on)), int(T), int(W)), self._ctx)

    def set_mode(self, mode):
        """opt::mode: MODE_STD, MODE_ORDERED (-c), MODE_BESTHIT (-b) or
        MODE_SCORES (-w)."""
        L.check(L.lib().bbt_set_mode(self._ctx, int(mode)), self._ctx)
        self.mode = int(mode)

    def set_launch(self, path=0, warps_per_block=0, frames_per_lane=0):
        L.check(L.lib().bbt_set_launch(self._ctx, path, warps_per_block, frames_per_lane),
                self._ctx)

    def set_bucketing(self, bucket_shift=0, phase_split=0, phase_min=0, max_frames=0,
                      levels_per_round=0):
        """Settings of the bucketed path (bbt_set_bucketing; 0 keeps one)."""
        L.check(L.lib().bbt_set_bucketing(self._ctx, bucket_shift, phase_split, phase_min,
                                          max_frames, levels_per_round), self._ctx)

    def set_schedule(self, long_bases=0):
        """Persistent kernel read order: reads of at least long_bases bases
        first (0 = index order)."""
        L.check(L.lib().bbt_set_schedule(self._ctx, int(long_bases)), self._ctx)

    def autotune(self, seq, off, seq2=None, off2=None):
        """Time the kernel configurations on a device-resident sample and keep
        the fastest (bbt_autotune); returns the chosen configuration."""
        b = L.Batch()
        b.seq, b.offsets, b.n_reads, b.location = (seq.data_ptr(), off.data_ptr(),
                                                   off.numel() - 1, L.DEVICE)
        if seq2 is not None:
            b.seq2, b.offsets2 = seq2.data_ptr(), off2.data_ptr()
        t = L.Tune()
        L.check(L.lib().bbt_autotune(self._ctx, ctypes.byref(b), ctypes.byref(t)), self._ctx)
        return {"path": t.path, "warps_per_block": t.warps_per_block,
                "frames_per_lane": t.frames_per_lane, "long_bases": t.long_bases,
                "reads_per_launch": t.reads_per_launch, "reads_per_s": t.reads_per_s,
                "steps": t.steps}

    def set_steps(self, steps):
        """Steps of the persistent path (bbt_set_steps): STEPS_DECISION sized to
        the read's decision, STEPS_FULL full 32-frame steps, STEPS_WIDE and
        STEPS_WIDE_FULL the same with two frames per lane (up to 64 frames)."""
        L.check(L.lib().bbt_set_steps(self._ctx, int(steps)), self._ctx)

    def graph(self, seq, off, hits, seq2=None, off2=None, hits2=None, category=None,
              reads_per_launch=0):
        """A CUDA graph classifying this device batch into these result tensors
        (bbt_graph_create); call .launch(stream) to run it."""
        return ClassifyGraph(self, seq, off, hits, seq2, off2, hits2, category, reads_per_launch)

    def set_counting(self, on=True):
        L.check(L.lib().bbt_set_counting(self._ctx, int(on)), self._ctx)

    # -- file pipeline (BioBloomClassifier::filter / filterPair) -----------
    def filter(self, input_files, read_status=None):
        files = [str(f).encode() for f in input_files]
        arr = (ctypes.c_char_p * len(files))(*files)
        L.check(L.lib().bbt_filter_files(self._ctx, arr, len(files), self.prefix.encode(),
                                          read_status.encode() if read_status else None),
                self._ctx)

    def filterPair(self, file1, file2, read_status=None):
        L.check(L.lib().bbt_filter_pair_files(self._ctx, str(file1).encode(), str(file2).encode(),
                                              self.prefix.encode(),
                                              read_status.encode() if read_status else None),
                self._ctx)

    def filterPrint(self, input_files, output_type, read_status=None):
        """Also write each read to "<prefix>_<category>.<output_type><postfix>"
        (output_type "fa" or "fq"); BioBloomClassifier::filterPrint."""
        files = [str(f).encode() for f in input_files]
        arr = (ctypes.c_char_p * len(files))(*files)
        L.check(L.lib().bbt_filter_files_print(self._ctx, arr, len(files), self.prefix.encode(),
                                                output_type.encode(), self.postfix.encode(),
                                                read_status.encode() if read_status else None),
                self._ctx)

    def filterPairPrint(self, file1, file2, output_type=None, read_status=None):
        """filterPairPrint(file1, file2, type), or filterPairPrint(file, type)
        for one file of name-matched mates when output_type is None."""
        if output_type is None:
            L.check(L.lib().bbt_filter_smart_pairs_print(
                self._ctx, str(file1).encode(), self.prefix.encode(), str(file2).encode(),
                self.postfix.encode(), read_status.encode() if read_status else None), self._ctx)
            return
        L.check(L.lib().bbt_filter_pair_files_print(
            self._ctx, str(file1).encode(), str(file2).encode(), self.prefix.encode(),
            output_type.encode(), self.postfix.encode(),
            read_status.encode() if read_status else None), self._ctx)

    def filterSmartPair(self, file, read_status=None):
        """filterPair(file): mates matched by name in one file
        (BioBloomClassifier.cpp:463-564)."""
        L.check(L.lib().bbt_filter_smart_pairs(self._ctx, str(file).encode(),
                                               self.prefix.encode(),
                                               read_status.encode() if read_status else None),
                self._ctx)

    def filterPairList(self, files1, files2, read_status=None):
        """filterPair(vector, vector): file i of files2 holds the mates of file
        i of files1 (BioBloomClassifier.cpp:731-806)."""
        if len(files1) != len(files2):
            raise ValueError("file lists differ in length")
        a = (ctypes.c_char_p * len(files1))(*[str(f).encode() for f in files1])
        b = (ctypes.c_char_p * len(files2))(*[str(f).encode() for f in files2])
        L.check(L.lib().bbt_filter_pair_file_lists(self._ctx, a, b, len(files1),
                                                   self.prefix.encode(),
                                                   read_status.encode() if read_status else None),
                self._ctx)

    # -- in-memory batches ---------------------------------------------------
    def classify(self, reads, reads2=None, scores=False):
        """Classify host reads (list of bytes or (uint8 array, uint64 offsets)).
        Returns (hits, hits2, category) as numpy arrays; hits2 is None for
        single-end input.  scores=True also returns SeqEval::evalScore of
        every read against every filter: (hits, hits2, category, scores,
        scores2), scores n x n_filters float64."""
        seq, off = pack(reads) if isinstance(reads, list) else reads
        seq = np.ascontiguousarray(seq, dtype=np.uint8)
        off = np.ascontiguousarray(off, dtype=np.uint64)
        n = len(off) - 1
        b = L.Batch()
        b.seq, b.offsets, b.n_reads, b.location = _ptr(seq), _ptr(off), n, L.HOST
        hits = np.zeros((n, self.words), dtype=np.uint64)
        cat = np.zeros(n, dtype=np.uint32)
        r = L.Result()
        r.hits, r.category, r.location = _ptr(hits), _ptr(cat), L.HOST
        hits2 = None
        if reads2 is not None:
            seq2, off2 = pack(reads2) if isinstance(reads2, list) else reads2
            seq2 = np.ascontiguousarray(seq2, dtype=np.uint8)
            off2 = np.ascontiguousarray(off2, dtype=np.uint64)
            if len(off2) - 1 != n:
                raise ValueError("mate arrays differ in length")
            b.seq2, b.offsets2 = _ptr(seq2), _ptr(off2)
            hits2 = np.zeros((n, self.words), dtype=np.uint64)
            r.hits2 = _ptr(hits2)
        if scores:
            sc = np.zeros((n, self.n_filters), dtype=np.float64)
            sc2 = np.zeros((n, self.n_filters), dtype=np.float64) if reads2 is not None else None
            L.check(L.lib().bbt_classify_batch_scores(
                self._ctx, ctypes.byref(b), ctypes.byref(r), _ptr(sc),
                _ptr(sc2) if sc2 is not None else None, None), self._ctx)
            return hits, hits2, cat, sc, sc2
        L.check(L.lib().bbt_classify_batch(self._ctx, ctypes.byref(b), ctypes.byref(r), None),
                self._ctx)
        return hits, hits2, cat

    def classify_device(self, seq, off, seq2=None, off2=None, hits=None, hits2=None,
                        category=None, stream=None, scores=None, scores2=None):
        """Classify reads resident on the GPU (torch uint8 / int64 tensors).
        Enqueued on `stream` (a torch.cuda.Stream, default: the current
        stream); returns (hits, hits2, category) tensors.  scores / scores2
        (float64 tensors of n x n_filters, optional) receive evalScore."""
        import torch
        n = off.numel() - 1
        dev = seq.device
        if hits is None:
            hits = torch.empty((n, self.words), dtype=torch.int64, device=dev)
        if category is None:
            category = torch.empty(n, dtype=torch.int32, device=dev)
        b = L.Batch()
        b.seq, b.offsets, b.n_reads, b.location = seq.data_ptr(), off.data_ptr(), n, L.DEVICE
        r = L.Result()
        r.hits, r.category, r.location = hits.data_ptr(), category.data_ptr(), L.DEVICE
        if seq2 is not None:
            if hits2 is None:
                hits2 = torch.empty((n, self.words), dtype=torch.int64, device=dev)
            b.seq2, b.offsets2 = seq2.data_ptr(), off2.data_ptr()
            r.hits2 = hits2.data_ptr()
        s = stream if stream is not None else torch.cuda.current_stream(dev)
        if scores is not None:
            L.check(L.lib().bbt_classify_batch_scores(
                self._ctx, ctypes.byref(b), ctypes.byref(r), ctypes.c_void_p(scores.data_ptr()),
                ctypes.c_void_p(scores2.data_ptr()) if scores2 is not None else None,
                ctypes.c_void_p(s.cuda_stream)), self._ctx)
            return hits, hits2, category
        L.check(L.lib().bbt_classify_batch(self._ctx, ctypes.byref(b), ctypes.byref(r),
                                           ctypes.c_void_p(s.cuda_stream)), self._ctx)
        return hits, hits2, category

    def last_stats(self):
        st = L.Stats()
        L.check(L.lib().bbt_last_stats(self._ctx, ctypes.byref(st)), self._ctx)
        return {"reads": st.reads, "frames": st.frames, "probes_issued": st.probes_issued,
                "probes_algorithmic": st.probes_algorithmic, "kernel_ms": st.kernel_ms,
                "classify_ms": st.classify_ms, "kernels": st.kernels}

    # -- summary (ResultsManager) ---------------------------------------------
    def summary(self):
        counts = np.zeros(2 * (self.n_filters + 2) + 2, dtype=np.uint64)
        reads = ctypes.c_uint64()
        L.check(L.lib().bbt_summary(self._ctx, counts.ctypes.data_as(
            ctypes.POINTER(ctypes.c_uint64)), ctypes.byref(reads)), self._ctx)
        return counts, reads.value

    def summary_tsv(self):
        n = ctypes.c_size_t()
        L.check(L.lib().bbt_summary_tsv(self._ctx, None, 0, ctypes.byref(n)), self._ctx)
        buf = ctypes.create_string_buffer(n.value + 1)
        L.check(L.lib().bbt_summary_tsv(self._ctx, buf, n.value + 1, ctypes.byref(n)), self._ctx)
        return buf.value.decode()

    def reset_summary(self):
        L.check(L.lib().bbt_reset_summary(self._ctx), self._ctx)

    def sync(self):
        L.check(L.lib().bbt_sync(self._ctx), self._ctx)

    def close(self):
        if getattr(self, "_ctx", None):
            L.lib().bbt_close(self._ctx)
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


class ClassifyGraph:
    """bbt_graph_*: a captured classification of fixed device buffers."""

    def __init__(self, bbc, seq, off, hits, seq2, off2, hits2, category, reads_per_launch):
        self._bbc = bbc
        self._keep = (seq, off, hits, seq2, off2, hits2, category)
        b = L.Batch()
        b.seq, b.offsets, b.n_reads, b.location = (seq.data_ptr(), off.data_ptr(),
                                                   off.numel() - 1, L.DEVICE)
        r = L.Result()
        r.hits, r.location = hits.data_ptr(), L.DEVICE
        if seq2 is not None:
            b.seq2, b.offsets2 = seq2.data_ptr(), off2.data_ptr()
            r.hits2 = hits2.data_ptr()
        if category is not None:
            r.category = category.data_ptr()
        g = ctypes.c_void_p()
        L.check(L.lib().bbt_graph_create(bbc._ctx, ctypes.byref(b), ctypes.byref(r),
                                         int(reads_per_launch), ctypes.byref(g)), bbc._ctx)
        self._g = g

    @property
    def launches(self):
        n = ctypes.c_uint64()
        L.check(L.lib().bbt_graph_launches(self._g, ctypes.byref(n)), self._bbc._ctx)
        return n.value

    def launch(self, stream=None):
        s = ctypes.c_void_p(stream.cuda_stream) if stream is not None else None
        L.check(L.lib().bbt_graph_launch(self._g, s), self._bbc._ctx)

    def close(self):
        if getattr(self, "_g", None):
            L.lib().bbt_graph_destroy(self._g)
            self._g = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
