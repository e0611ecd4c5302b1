"""ctypes binding of libbbt.so (the C ABI declared in include/bbt.h).

The library is built in-tree by biobloom_b200.build_native; importing this
module never falls back to anything else: if the library is missing or cannot
be loaded, LibraryMissing is raised.
"""
import ctypes
import os

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "lib", "libbbt.so")

BBT_OK = 0
BBT_ERR = {-1: "ARG", -2: "IO", -3: "FORMAT", -4: "CUDA", -5: "NOMEM", -6: "UNSUPPORTED",
           -7: "TIMEOUT", -8: "NODEVICE", -9: "OVERFLOW"}
ERR_OVERFLOW = -9
MIBF_OUT_TSV, MIBF_OUT_FASTA, MIBF_OUT_FASTQ = 0, 1, 2
MIBF_LAYOUT_AUTO, MIBF_LAYOUT_RANK, MIBF_LAYOUT_DENSE = 0, 1, 2
SCORE_SIMPLE, SCORE_LENGTH, SCORE_HARMONIC, SCORE_BINOMIAL = 0, 1, 2, 3
HOST, DEVICE = 0, 1
BASES_ASCII, BASES_2BIT = 0, 1
PATH_AUTO, PATH_PLAIN, PATH_PERSISTENT, PATH_FILTER_MAJOR, PATH_BUCKETED = 0, 1, 2, 3, 4
STEPS_DECISION, STEPS_FULL, STEPS_WIDE, STEPS_WIDE_FULL = 0, 1, 2, 3
MODE_STD, MODE_ORDERED, MODE_BESTHIT, MODE_SCORES = 0, 1, 2, 3


class LibraryMissing(RuntimeError):
    pass


class BBTError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"bbt error {code} ({BBT_ERR.get(code, '?')}): {msg}")
        self.code = code


class Params(ctypes.Structure):
    _fields_ = [("score", ctypes.c_double), ("streak_threshold", ctypes.c_uint),
                ("scoring", ctypes.c_int), ("inclusive", ctypes.c_int), ("device", ctypes.c_int),
                ("path", ctypes.c_int), ("warps_per_block", ctypes.c_uint32),
                ("frames_per_lane", ctypes.c_uint32), ("max_batch_bases", ctypes.c_uint64),
                ("max_batch_reads", ctypes.c_uint64), ("l2_fetch_bytes", ctypes.c_uint32)]


class Batch(ctypes.Structure):
    _fields_ = [("seq", ctypes.c_void_p), ("offsets", ctypes.c_void_p), ("seq2", ctypes.c_void_p),
                ("offsets2", ctypes.c_void_p), ("n_reads", ctypes.c_uint64),
                ("location", ctypes.c_int), ("encoding", ctypes.c_int),
                ("valid", ctypes.c_void_p), ("valid2", ctypes.c_void_p)]


class Result(ctypes.Structure):
    _fields_ = [("hits", ctypes.c_void_p), ("hits2", ctypes.c_void_p),
                ("category", ctypes.c_void_p), ("location", ctypes.c_int)]


class Stats(ctypes.Structure):
    _fields_ = [("reads", ctypes.c_uint64), ("frames", ctypes.c_uint64),
                ("probes_issued", ctypes.c_uint64), ("probes_algorithmic", ctypes.c_uint64),
                ("kernel_ms", ctypes.c_double), ("classify_ms", ctypes.c_double),
                ("kernels", ctypes.c_uint64)]


class FilterView(ctypes.Structure):
    _fields_ = [("words", ctypes.c_void_p), ("m", ctypes.c_uint64), ("h", ctypes.c_uint),
                ("k", ctypes.c_uint)]


class Tune(ctypes.Structure):
    _fields_ = [("path", ctypes.c_int), ("warps_per_block", ctypes.c_int),
                ("frames_per_lane", ctypes.c_int), ("long_bases", ctypes.c_uint64),
                ("reads_per_launch", ctypes.c_uint64), ("reads_per_s", ctypes.c_double),
                ("steps", ctypes.c_int)]


class SynthReadParams(ctypes.Structure):
    _fields_ = [("len_min", ctypes.c_uint32), ("len_max", ctypes.c_uint32),
                ("long_frac", ctypes.c_double), ("long_min", ctypes.c_uint32),
                ("long_max", ctypes.c_uint32), ("sub_rate", ctypes.c_double),
                ("n_rate", ctypes.c_double), ("frag_min", ctypes.c_uint32),
                ("frag_max", ctypes.c_uint32)]


class MibfParams(ctypes.Structure):
    _fields_ = [("score", ctypes.c_double), ("frame_matches", ctypes.c_uint),
                ("multi_thresh", ctypes.c_double), ("streak", ctypes.c_uint),
                ("min_nonsat", ctypes.c_uint), ("best_hit_agree", ctypes.c_int),
                ("hit_only", ctypes.c_int), ("device", ctypes.c_int),
                ("max_batch_bases", ctypes.c_uint64), ("max_batch_reads", ctypes.c_uint64),
                ("layout", ctypes.c_int)]


class MibfHit(ctypes.Structure):
    _fields_ = [("id", ctypes.c_uint32), ("nonSatFrameCount", ctypes.c_uint32),
                ("solidCount", ctypes.c_uint32), ("count", ctypes.c_uint32),
                ("nonSatCount", ctypes.c_uint32), ("totalNonSatCount", ctypes.c_uint32),
                ("totalCount", ctypes.c_uint32)]


class MibfResult(ctypes.Structure):
    _fields_ = [("hits", ctypes.c_void_p), ("max_hits", ctypes.c_uint32),
                ("n_hits", ctypes.c_void_p), ("sat_count", ctypes.c_void_p),
                ("location", ctypes.c_int)]


class ServerParams(ctypes.Structure):
    _fields_ = [("mem_budget", ctypes.c_uint64), ("slots", ctypes.c_uint32),
                ("chunk_reads", ctypes.c_uint64), ("max_frames", ctypes.c_uint32)]


class Request(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_int), ("seq", ctypes.c_void_p), ("offsets", ctypes.c_void_p),
                ("seq2", ctypes.c_void_p), ("offsets2", ctypes.c_void_p),
                ("n_reads", ctypes.c_uint64), ("hits", ctypes.c_void_p), ("hits2", ctypes.c_void_p),
                ("category", ctypes.c_void_p), ("mi_hits", ctypes.c_void_p),
                ("mi_max_hits", ctypes.c_uint32), ("mi_n_hits", ctypes.c_void_p),
                ("mi_sat", ctypes.c_void_p)]


class RequestStats(ctypes.Structure):
    _fields_ = [("status", ctypes.c_int), ("t_submit", ctypes.c_double),
                ("t_admit", ctypes.c_double), ("t_done", ctypes.c_double),
                ("device_bytes", ctypes.c_uint64), ("slot", ctypes.c_uint32)]


REQ_BLOOM, REQ_MIBF = 0, 1

_lib = None


def lib():
    """Load libbbt.so (raises LibraryMissing if it is not built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise LibraryMissing(f"{LIB_PATH} is not built; run biobloom_b200.build_native.build()")
    try:
        L = ctypes.CDLL(LIB_PATH)
    except OSError as e:
        raise LibraryMissing(f"cannot load {LIB_PATH}: {e}") from e
    P = ctypes.POINTER
    vp, u64, i32, u32, dbl, cp = (ctypes.c_void_p, ctypes.c_uint64, ctypes.c_int, ctypes.c_uint,
                                  ctypes.c_double, ctypes.c_char_p)
    sig = {
        "bbt_default_params": (None, [P(Params)]),
        "bbt_open": (i32, [P(cp), i32, P(Params), P(vp)]),
        "bbt_open_devices": (i32, [P(cp), i32, P(Params), P(ctypes.c_int), i32, P(vp)]),
        "bbt_close": (i32, [vp]),
        "bbt_last_error": (cp, [vp]),
        "bbt_num_filters": (i32, [vp]),
        "bbt_filter_id": (cp, [vp, i32]),
        "bbt_classify_batch": (i32, [vp, P(Batch), P(Result), vp]),
        "bbt_sync": (i32, [vp]),
        "bbt_summary": (i32, [vp, P(u64), P(u64)]),
        "bbt_reset_summary": (i32, [vp]),
        "bbt_summary_tsv": (i32, [vp, ctypes.c_char_p, ctypes.c_size_t, P(ctypes.c_size_t)]),
        "bbt_filter_files": (i32, [vp, P(cp), i32, cp, cp]),
        "bbt_filter_pair_files": (i32, [vp, cp, cp, cp, cp]),
        "bbt_filter_files_print": (i32, [vp, P(cp), i32, cp, cp, cp, cp]),
        "bbt_filter_pair_files_print": (i32, [vp, cp, cp, cp, cp, cp, cp]),
        "bbt_filter_pair_file_lists": (i32, [vp, P(cp), P(cp), i32, cp, cp]),
        "bbt_filter_smart_pairs": (i32, [vp, cp, cp, cp]),
        "bbt_filter_smart_pairs_print": (i32, [vp, cp, cp, cp, cp, cp]),
        "bbt_set_stdout": (i32, [vp, i32, i32]),
        "bbt_set_mode": (i32, [vp, i32]),
        "bbt_set_dust": (i32, [vp, i32, u32, u32]),
        "bbt_classify_batch_scores": (i32, [vp, P(Batch), P(Result), vp, vp, vp]),
        "bbt_last_stats": (i32, [vp, P(Stats)]),
        "bbt_set_counting": (i32, [vp, i32]),
        "bbt_set_launch": (i32, [vp, i32, i32, i32]),
        "bbt_set_steps": (i32, [vp, i32]),
        "bbt_set_inclusive": (i32, [vp, i32]),
        "bbt_set_schedule": (i32, [vp, u64]),
        "bbt_autotune": (i32, [vp, P(Batch), P(Tune)]),
        "bbt_graph_create": (i32, [vp, P(Batch), P(Result), u64, P(vp)]),
        "bbt_graph_launch": (i32, [vp, vp]),
        "bbt_graph_launches": (i32, [vp, P(u64)]),
        "bbt_graph_destroy": (i32, [vp]),
        "bbt_classify_noalloc": (i32, [P(FilterView), i32, P(Params), P(Batch), vp, vp, vp]),
        "bbt_make_filter": (i32, [vp, P(u64), u64, u32, dbl, u32, u64, cp, cp, cp, i32]),
        "bbt_measure_gather": (i32, [i32, u64, u64, i32, i32, P(dbl)]),
        "bbt_pack_bases": (i32, [vp, u64, vp, vp, P(u64)]),
        "bbt_set_bucketing": (i32, [vp, u32, u32, u32, u64, u32]),
        "bbt_synth_genome": (i32, [u64, u64, dbl, dbl, ctypes.c_uint32, ctypes.c_uint32, dbl, dbl,
                                   vp]),
        "bbt_synth_read_lengths": (i32, [u64, P(SynthReadParams), u64, vp]),
        "bbt_synth_reads": (i32, [u64, vp, vp, ctypes.c_uint32, vp, P(SynthReadParams), u64, vp,
                                  vp, vp, vp]),
        "bbt_server_create": (i32, [vp, vp, P(ServerParams), P(vp)]),
        "bbt_server_submit": (i32, [vp, P(Request), P(u64)]),
        "bbt_server_wait": (i32, [vp, u64, dbl, P(RequestStats)]),
        "bbt_server_load": (i32, [vp, P(u64), P(u64), P(u64)]),
        "bbt_server_destroy": (i32, [vp]),
        "bbt_server_last_error": (cp, [vp]),
        "bbt_mibf_default_params": (None, [P(MibfParams)]),
        "bbt_mibf_open": (i32, [cp, P(MibfParams), P(vp)]),
        "bbt_mibf_open_host": (i32, [cp, P(MibfParams), P(vp)]),
        "bbt_mibf_close": (i32, [vp]),
        "bbt_mibf_last_error": (cp, [vp]),
        "bbt_mibf_num_ids": (u32, [vp]),
        "bbt_mibf_layout": (i32, [vp]),
        "bbt_mibf_id_name": (cp, [vp, u32]),
        "bbt_mibf_info": (i32, [vp, P(u64), P(u32), P(u32), P(u32)]),
        "bbt_mibf_frame_probs": (i32, [vp, P(dbl), P(dbl)]),
        "bbt_mibf_classify_batch": (i32, [vp, P(Batch), P(MibfResult), vp]),
        "bbt_mibf_sync": (i32, [vp]),
        "bbt_mibf_set_bucketing": (i32, [vp, i32, u32, u64]),
        "bbt_mibf_last_kernel_ms": (dbl, [vp]),
        "bbt_mibf_last_counts": (i32, [vp, P(u64)]),
        "bbt_mibf_summary": (i32, [vp, P(u64), P(u64)]),
        "bbt_mibf_reset_summary": (i32, [vp]),
        "bbt_mibf_summary_tsv": (i32, [vp, u64, ctypes.c_char_p, ctypes.c_size_t,
                                       P(ctypes.c_size_t)]),
        "bbt_mibf_filter_files": (i32, [vp, P(cp), i32, cp, i32, vp]),
        "bbt_mibf_filter_pair_files": (i32, [vp, cp, cp, cp, i32, vp]),
        "bbt_mibf_min_count": (u32, [u32, dbl, dbl, u32]),
        "bbt_mibf_format_record": (i32, [vp, i32, cp, cp, cp, cp, P(MibfHit), ctypes.c_uint32,
                                         ctypes.c_uint32, ctypes.c_char_p, ctypes.c_size_t,
                                         P(ctypes.c_size_t)]),
        "bbt_mibf_make": (i32, [vp, vp, vp, u64, P(cp), u32, P(cp), u32, u32, u32, dbl, i32,
                                cp, i32]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


def check(rc, ctx=None):
    if rc != BBT_OK:
        msg = lib().bbt_last_error(ctx)
        raise BBTError(rc, msg.decode() if msg else "")
    return rc


def check_mibf(rc, ctx=None):
    if rc != BBT_OK:
        msg = lib().bbt_mibf_last_error(ctx)
        raise BBTError(rc, msg.decode() if msg else "")
    return rc
