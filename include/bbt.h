/*
 * bbt.h -- C ABI of the B200 read-classification library (libbbt.so).
 *
 * This is the drop-in boundary for BioBloom Tools' classification path.  The
 * reference has no FFI: its boundary is the BioBloomClassifier class and the
 * biobloomcategorizer CLI.  Each entry point below names the reference
 * interface it replaces (paths are relative to the biobloom project).
 *
 * Conventions
 *   - Every function returns an int status: BBT_OK (0) or a negative BBT_ERR_*.
 *     The text of the last error is available from bbt_last_error(ctx) (or
 *     bbt_last_error(NULL) for errors raised before a context exists).  The
 *     reference prints and exit(1)s instead (e.g. BioBloomClassifier.cpp:54-57).
 *   - The caller owns every host buffer; a context owns its device memory.
 *   - A context is used from one host thread at a time.
 *   - Streams are passed as void* (a cudaStream_t, or NULL for the context's
 *     own stream).
 *   - Sequences are ASCII bases; A, C, G, T in either case are valid bases,
 *     every other byte ends the k-mers that cover it, as ntHashIterator does.
 */
#ifndef BBT_H
#define BBT_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---- */
#define BBT_OK 0
#define BBT_ERR_ARG (-1)          /* invalid argument */
#define BBT_ERR_IO (-2)           /* file cannot be opened / read / written */
#define BBT_ERR_FORMAT (-3)       /* malformed .bf / .txt / FASTA / FASTQ */
#define BBT_ERR_CUDA (-4)         /* CUDA runtime error */
#define BBT_ERR_NOMEM (-5)        /* host or device allocation failed */
#define BBT_ERR_UNSUPPORTED (-6)  /* option combination not implemented */
#define BBT_ERR_TIMEOUT (-7)      /* a bounded device wait gave up */
#define BBT_ERR_NODEVICE (-8)     /* no CUDA device is usable */

/* ---- scoring methods (opt::ScoringMethod, Common/Options.h:75) ---- */
#define BBT_SCORE_SIMPLE 0
#define BBT_SCORE_LENGTH 1
#define BBT_SCORE_HARMONIC 2   /* -S harmonic: score in [0, 1] */
#define BBT_SCORE_BINOMIAL 3   /* -S binomial: score = minimum FPR of a match,
                                  10^(-s/10) (BioBloomCategorizer.cpp:418-420) */

/* ---- where batch buffers live ---- */
#define BBT_HOST 0
#define BBT_DEVICE 1

/* ---- kernel paths ---- */
#define BBT_PATH_AUTO 0        /* persistent work-stealing path, tuned */
#define BBT_PATH_PLAIN 1       /* one warp per read, one launch per batch */
#define BBT_PATH_PERSISTENT 2  /* persistent work-stealing kernel, read-major */
#define BBT_PATH_FILTER_MAJOR 3 /* persistent, (filter, read) items in filter order */
#define BBT_PATH_BUCKETED 4    /* probes sorted by filter address (filters far above L2) */

typedef struct bbt_ctx bbt_ctx;

/*
 * Classification parameters.  Mirrors the options the reference reads from
 * opt:: inside BioBloomClassifier (BioBloomCategorizer/Options.cpp:14-36,
 * Common/Options.cpp:7-9) plus the device-side knobs of this library.
 */
typedef struct {
	double score;               /* -s: threshold in [0,1], or an integer > 1 for
	                               LENGTH scoring (BioBloomCategorizer.cpp:416-441) */
	unsigned streak_threshold;  /* -r (Common/Options.cpp:9), default 3 */
	int scoring;                /* BBT_SCORE_*; set from score by bbt_default_params
	                               semantics when score > 1 */
	int inclusive;              /* -i (BioBloomClassifier.h:77-79) */
	int device;                 /* CUDA device ordinal */
	int path;                   /* BBT_PATH_* */
	uint32_t warps_per_block;   /* 0 = tuned */
	uint32_t frames_per_lane;   /* probe chains in flight per lane (1, 2 or 4); 0 = tuned */
	uint64_t max_batch_bases;   /* device staging capacity per batch (bases); 0 = default */
	uint64_t max_batch_reads;   /* device staging capacity per batch (reads); 0 = default */
	uint32_t l2_fetch_bytes;    /* L2 fetch granularity for this process's context
	                               (cudaLimitMaxL2FetchGranularity): 32, 64 or 128;
	                               0 = 32, one DRAM sector per Bloom probe */
} bbt_params;

/* Fill p with the reference's defaults (score 0.15, streak 3, SIMPLE). */
void bbt_default_params(bbt_params *p);

/*
 * Load filters and upload them to device memory once.
 * Replaces BioBloomClassifier::BioBloomClassifier / loadFilters
 * (BioBloomClassifier.cpp:21-28, 950-971): for each "<x>.bf" the sidecar
 * "<x>.txt" (same stem) supplies the filter id.
 */
int bbt_open(const char *const *bf_paths, int n_filters, const bbt_params *params,
		bbt_ctx **out);
int bbt_close(bbt_ctx *ctx);
const char *bbt_last_error(const bbt_ctx *ctx);

/*
 * bbt_open on several GPUs: the filters are loaded on every device in
 * `devices` (replicas; params->device is ignored).  Host batches
 * (bbt_classify_batch with BBT_HOST buffers, and so the bbt_filter_* file
 * pipeline and the CLI) are split into contiguous shards of reads, one per
 * device, classified concurrently and written back in batch order; the
 * summary counters of the devices are added up by bbt_summary.  Device
 * batches run on the first device.  Setters apply to every device.  A device
 * may be listed twice (two contexts on one GPU).  The reference's only
 * parallelism is OpenMP threads (-t); this replaces it across GPUs.
 */
int bbt_open_devices(const char *const *bf_paths, int n_filters, const bbt_params *params,
		const int *devices, int n_devices, bbt_ctx **out);

int bbt_num_filters(const bbt_ctx *ctx);
/* Filter id of filter i (BloomFilterInfo::getFilterID, BloomFilterInfo.cpp:141). */
const char *bbt_filter_id(const bbt_ctx *ctx, int i);

/* Base encodings of a batch (bbt_batch.encoding). */
#define BBT_BASES_ASCII 0      /* one byte per base, as in FASTA / FASTQ */
#define BBT_BASES_2BIT 1       /* 2-bit codes + validity bits (below) */

/*
 * A batch of reads.  Single-end: seq/offsets hold n_reads reads
 * (read i = bases offsets[i] .. offsets[i+1] of seq).  Paired: seq2/offsets2
 * hold the mates, read i of seq pairs with read i of seq2, and n_reads counts
 * pairs.
 *
 * encoding BBT_BASES_ASCII (0, the default of a zeroed struct): seq holds one
 * byte per base.  BBT_BASES_2BIT: seq points to uint32 words with base g at
 * bits 2 (g % 16) .. 2 (g % 16) + 1 of word g / 16 (A/a = 0, C/c = 1, G/g = 2,
 * T/t = 3), 4 times fewer bytes to copy; valid (valid2 for seq2) holds bit
 * g % 32 of word g / 32 = 1 when base g is one of ACGTacgt (any other base is
 * skipped by the k-mer iterator, as an N is), or is NULL when every base is.
 * The word arrays must be 4-byte aligned; bbt_pack_bases fills them.
 * Offsets count bases in either encoding.
 */
typedef struct {
	const char *seq;
	const uint64_t *offsets;   /* n_reads + 1 entries, offsets[0] may be > 0 */
	const char *seq2;          /* NULL for single-end */
	const uint64_t *offsets2;
	uint64_t n_reads;
	int location;              /* BBT_HOST or BBT_DEVICE for all the arrays */
	int encoding;              /* BBT_BASES_ASCII or BBT_BASES_2BIT */
	const uint32_t *valid;     /* BBT_BASES_2BIT: validity bits of seq, or NULL */
	const uint32_t *valid2;    /* BBT_BASES_2BIT: validity bits of seq2, or NULL */
} bbt_batch;

/*
 * Pack n ASCII bases into the BBT_BASES_2BIT form: words (n + 15) / 16 uint32,
 * valid (n + 31) / 32 uint32 (may be NULL when the caller knows every base is
 * ACGTacgt).  *n_invalid (optional) receives the number of other bases; when
 * it is 0 the batch may pass valid = NULL.  Host memory, all host threads.
 * No counterpart in the reference, which keeps reads as strings.
 */
int bbt_pack_bases(const char *ascii, uint64_t n, uint32_t *words, uint32_t *valid,
		uint64_t *n_invalid);

/*
 * Per-read results.  hits/hits2 (optional): words = (n_filters + 63) / 64
 * uint64 per read, bit f set when SeqEval accepted the read for filter f
 * (evaluateReadStd, BioBloomClassifier.cpp:1182-1189).  category (optional):
 * per read (or pair) the index ResultsManager::updateSummaryData returns
 * (ResultsManager.hpp:66-189): the filter index for a unique hit, n_filters for
 * noMatch, n_filters + 1 for multiMatch.
 */
typedef struct {
	uint64_t *hits;
	uint64_t *hits2;
	uint32_t *category;
	int location;              /* BBT_HOST or BBT_DEVICE */
} bbt_result;

/*
 * Classify one batch and add it to the context's summary counters.
 * Replaces the per-read loop of BioBloomClassifier::filter / filterPair
 * (BioBloomClassifier.cpp:33-100, 217-303).  With BBT_HOST buffers the call
 * copies inputs in and results out and returns when they are in place (the
 * reads go through two device staging slots in about eight loads, each load's
 * copies overlapping the kernels of the one before; pinned host arrays
 * overlap best, results bound for pageable memory are staged through pinned
 * buffers); with BBT_DEVICE buffers it enqueues on `stream` and returns
 * (results are ready when the stream reaches that point).
 */
int bbt_classify_batch(bbt_ctx *ctx, const bbt_batch *batch, bbt_result *result,
		void *stream);

/* Wait for all work the context enqueued. */
int bbt_sync(bbt_ctx *ctx);

/*
 * Summary counters (ResultsManager.hpp:250-261): counts must hold
 * 2 * (n_filters + 2) + 2 uint64: aboveThreshold[n_filters + 2],
 * unique[n_filters + 2], multiMatch, noMatch; *reads = reads (or pairs) seen.
 */
int bbt_summary(bbt_ctx *ctx, uint64_t *counts, uint64_t *reads);
int bbt_reset_summary(bbt_ctx *ctx);
/* summary.tsv text (ResultsManager::getResultsSummary, ResultsManager.hpp:191-237).
 * Writes at most cap bytes including the NUL; *len receives the full length. */
int bbt_summary_tsv(bbt_ctx *ctx, char *buf, size_t cap, size_t *len);

/*
 * File pipeline: parse FASTA/FASTQ (gzip or plain) into pinned, double-
 * buffered batches, classify, and write "<prefix>_summary.tsv" and, if
 * read_status is non-NULL, a per-read "<name>\t<category>" file.
 * Replaces BioBloomClassifier::filter (BioBloomClassifier.cpp:33-100) and
 * filterPair(file1, file2) (BioBloomClassifier.cpp:217-303).
 */
int bbt_filter_files(bbt_ctx *ctx, const char *const *files, int n_files,
		const char *prefix, const char *read_status);
int bbt_filter_pair_files(bbt_ctx *ctx, const char *file1, const char *file2,
		const char *prefix, const char *read_status);

/*
 * The same pipelines, also writing every read (pair) to a file of its category
 * (--fa / --fq, with -g for gzip): "<prefix>_<filterID>.<out_type><postfix>"
 * per filter, then "_noMatch" and "_multiMatch" (pairs: "_1" / "_2" before
 * the extension); records are ">name comment\nseq\n" or
 * "@name comment\nseq\n+\nqual\n" in input order.  out_type: "fa" or "fq";
 * postfix: "" or ".gz".  In BESTHIT and SCORES modes (bbt_set_mode) records
 * carry scores after the comment, each as " %g": SCORES on multiMatch records
 * every filter's score; BESTHIT the read's best score, except on multiMatch
 * records of FASTA files and of pairs, which repeat it once per best filter
 * (BioBloomClassifier.h:144-209, 291-411).  Replaces
 * BioBloomClassifier::filterPrint (BioBloomClassifier.cpp:108-203) and
 * filterPairPrint (:311-450).
 */
int bbt_filter_files_print(bbt_ctx *ctx, const char *const *files, int n_files,
		const char *prefix, const char *out_type, const char *postfix, const char *read_status);
int bbt_filter_pair_files_print(bbt_ctx *ctx, const char *file1, const char *file2,
		const char *prefix, const char *out_type, const char *postfix, const char *read_status);

/*
 * Pairs from a list of file pairs (-e -l): files2[i] holds the mates of
 * files1[i]; each pair of files is read until either ends, and one summary
 * covers them all.  Replaces BioBloomClassifier::filterPair(vector, vector)
 * (BioBloomClassifier.cpp:731-806; list parsing BioBloomCategorizer.cpp:
 * 482-497).
 */
int bbt_filter_pair_file_lists(bbt_ctx *ctx, const char *const *files1,
		const char *const *files2, int n_pairs, const char *prefix, const char *read_status);

/*
 * Pairs from one file (-e with a single input): a record's header is its name
 * without the last two characters when the name ends in '1' or '2'; the first
 * record of a header waits until the next record with that header arrives,
 * which completes the pair (the waiting record is mate 1) and frees the
 * header.  Records that never pair are not counted.  Records are written with
 * the shortened header.  Replaces BioBloomClassifier::filterPair(file) and
 * filterPairPrint(file, type) (BioBloomClassifier.cpp:463-564, 571-729).
 */
int bbt_filter_smart_pairs(bbt_ctx *ctx, const char *file, const char *prefix,
		const char *read_status);
int bbt_filter_smart_pairs_print(bbt_ctx *ctx, const char *file, const char *prefix,
		const char *out_type, const char *postfix, const char *read_status);

/* -d / -n: the file pipelines also print, as FASTQ on stdout, each read (both
 * mates of a pair) whose category is the first filter (inverse: every other
 * category; BESTHIT adds the read's best score to the first filter's reads).  Replaces BioBloomClassifier::setStdout and printSingle /
 * printPair (BioBloomClassifier.h:81-83, 115-142, 211-247). */
int bbt_set_stdout(bbt_ctx *ctx, int on, int inverse);

/* Pairs count for a filter when either mate hits (-i; union of the mates' hit
 * lists) instead of both (intersection, the default).
 * Replaces BioBloomClassifier::setInclusive (BioBloomClassifier.h:77-79). */
int bbt_set_inclusive(bbt_ctx *ctx, int inclusive);

/*
 * Filtering mode (opt::mode, BioBloomCategorizer/Options.h:22-24), chosen in
 * the reference by -c, -b and -w (BioBloomCategorizer.cpp:276-318, 460-464):
 *   BBT_MODE_STD      every filter SeqEval::evalRead accepts
 *                     (evaluateReadStd, BioBloomClassifier.cpp:1182-1189);
 *   BBT_MODE_ORDERED  -c: only the first such filter in load order; pairs take
 *                     the first filter both mates pass, or either mate with -i
 *                     (evaluateReadOrdered / evaluateReadOrderedPair,
 *                     BioBloomClassifier.cpp:1145-1180; setOrderedFilter,
 *                     BioBloomClassifier.h:67-75);
 *   BBT_MODE_BESTHIT  -b: no threshold; the filters whose SeqEval::evalScore is
 *                     the largest, if that is above 0 (evaluateReadBestHit,
 *                     BioBloomClassifier.cpp:1194-1218);
 *   BBT_MODE_SCORES   -w: STD hits, and evalScore of every filter for the
 *                     multiMatch output (evaluateReadScore, :1224-1237).
 * Pairs outside ORDERED evaluate each mate alone, as in STD.  The hit words
 * of bbt_result carry the mode's hits.  BESTHIT and ORDERED cannot be combined
 * (the setting replaces the previous one).
 */
#define BBT_MODE_STD 0
#define BBT_MODE_ORDERED 1
#define BBT_MODE_BESTHIT 2
#define BBT_MODE_SCORES 3
int bbt_set_mode(bbt_ctx *ctx, int mode);

/*
 * -D / -T / -W: SDUST low-complexity masking (Common/sdust.c through
 * Common/SDust.hpp; options BioBloomCategorizer.cpp:323-337, defaults T = 20,
 * W = 64 in Common/Options.cpp:36-38).  Every evaluation then treats a frame
 * whose first base lies in a masked interval of its read as a miss that is not
 * probed, in all scoring methods and modes.  W must be in [3, 1024].  Calls
 * with masking wait for their stream before returning; the serving engine and
 * CUDA graphs refuse it.
 */
int bbt_set_dust(bbt_ctx *ctx, int on, unsigned T, unsigned W);

/*
 * bbt_classify_batch that also returns evalScore (Common/SeqEval.h:534-560)
 * of every read against every filter: scores (scores2 for the mates) hold
 * n_reads x n_filters doubles, read-major, in result->location memory.  The
 * score of the scoring method in use: SIMPLE and HARMONIC sums divided by
 * len - k + 1, the final match length for LENGTH, -10 log10 of the binomial
 * tail for BINOMIAL.  Any mode; the hit words and summary follow the mode.
 */
int bbt_classify_batch_scores(bbt_ctx *ctx, const bbt_batch *batch, bbt_result *result,
		double *scores, double *scores2, void *stream);

/* Kernel path and launch shape (BBT_PATH_*, warps per block 4 or 8, frames
 * per lane when hashing 4 or 8); 0 keeps the current value.  Used by the
 * tuner; no reference counterpart (the reference's only knob is -t threads,
 * BioBloomCategorizer.cpp:243-249). */
int bbt_set_launch(bbt_ctx *ctx, int path, int warps_per_block, int frames_per_lane);

/* Read order of the persistent kernel: reads of at least long_bases bases are
 * started first (longest-processing-first scheduling, so that a long read does
 * not start last and hold the end of the launch); 0 = index order.  Results do
 * not depend on it.  No reference counterpart. */
int bbt_set_schedule(bbt_ctx *ctx, uint64_t long_bases);

/* Settings of the bucketed path (BBT_PATH_BUCKETED): each round's requests
 * are resolved one bucket of 2^bucket_shift filter bits at a time (a bucket
 * should fit L2: the default 27 = 16 MB); a read's frames are resolved in two
 * phases split at phase_split / 16 of its frames (default 4; 16 = one phase),
 * the first covering at least min(frames, phase_min) frames (default 64); at
 * most max_frames frames per sub-batch (default 2^30; scratch: about
 * 8.4 + 7 x levels_per_round bytes per frame); each round tests
 * levels_per_round hash levels (1 to 64, default 1: the first round levels
 * [0, L), the next [L, 2L), ...; a frame requests a round's levels only when
 * it passed all earlier ones).  0 keeps a setting.  Results do not depend on
 * them.  No reference counterpart. */
int bbt_set_bucketing(bbt_ctx *ctx, unsigned bucket_shift, unsigned phase_split,
		unsigned phase_min, uint64_t max_frames, unsigned levels_per_round);

/*
 * Autotuner: time every kernel configuration on a device-resident sample
 * (path plain / persistent / persistent long-first / filter-major when the
 * filters fit in L2; 4 or 8 warps per block; 4 or 8 frames per lane; the
 * persistent path with either step size of bbt_set_steps), keep
 * the fastest, then pick the reads per launch (64k, 256k, 1M or the whole
 * sample) for it, and leave the context set to the result.  The summary
 * counters are left as they were.  No reference counterpart (the reference's
 * only knob is -t).
 */
typedef struct {
	int path;
	int warps_per_block;
	int frames_per_lane;
	uint64_t long_bases;        /* bbt_set_schedule value */
	uint64_t reads_per_launch;  /* 0 = whole batches (no split was faster) */
	double reads_per_s;         /* on the sample */
	int steps;                  /* bbt_set_steps value (BBT_STEPS_*) */
} bbt_tune;
int bbt_autotune(bbt_ctx *ctx, const bbt_batch *sample, bbt_tune *out);

/* Steps of the persistent path.  Each step of a warp probes up to 32 frames
 * of a read, one per lane, or up to 64 with two frames per lane (WIDE: twice
 * the filter reads in flight, for filters in HBM where the kernel waits on
 * them).  With SIMPLE and BINOMIAL scoring, DECISION steps are sized to the
 * frames that could still decide the read (fewer probes: filters in HBM) and
 * FULL steps are always full (fewer steps and instructions: filters held in
 * L2).  BBT_STEPS_DECISION is the default; bbt_autotune tries all four.
 * Results do not depend on it.  No reference counterpart. */
#define BBT_STEPS_DECISION 0
#define BBT_STEPS_FULL 1
#define BBT_STEPS_WIDE 2
#define BBT_STEPS_WIDE_FULL 3
int bbt_set_steps(bbt_ctx *ctx, int steps);

/*
 * CUDA graph of the classification of one device batch in launches of
 * reads_per_launch reads (0 = one launch), captured once and replayed by
 * bbt_graph_launch: the launch sequence (work-counter resets, read order,
 * classification and summary kernels per launch) costs one graph launch.  The
 * graph is bound to the batch's and results' device pointers: refill those
 * buffers between launches.  Summary counters are updated at each launch.
 * Plain and persistent paths only (the filter-major path reads block sums on
 * the host).  Create it after a warm-up call with the same sizes.
 */
typedef struct bbt_graph bbt_graph;
int bbt_graph_create(bbt_ctx *ctx, const bbt_batch *batch, const bbt_result *result,
		uint64_t reads_per_launch, bbt_graph **out);
int bbt_graph_launch(bbt_graph *g, void *stream);
int bbt_graph_launches(const bbt_graph *g, uint64_t *launches);
int bbt_graph_destroy(bbt_graph *g);

/* Count filter words read and frames hashed in the following batches
 * (diagnostics; costs atomics).  No reference counterpart. */
int bbt_set_counting(bbt_ctx *ctx, int on);

/* Counters of the batches classified since counting was switched on (see
 * bbt_set_counting), and the device time of the last batch. */
typedef struct {
	uint64_t reads;
	uint64_t frames;              /* frames hashed */
	uint64_t probes_issued;       /* filter words read by the kernel */
	uint64_t probes_algorithmic;  /* filter words the sequential reference reads:
	                                 BloomFilter::contains bit tests up to the first
	                                 clear bit, for the frames SeqEval visits */
	double kernel_ms;             /* device time of the last batch (all kernels) */
	double classify_ms;           /* device time of the last batch's classification
	                                 kernels (without the summary kernel) */
	uint64_t kernels;             /* kernels the last batch launched */
} bbt_stats;
int bbt_last_stats(bbt_ctx *ctx, bbt_stats *out);

/*
 * Build a Bloom filter on the device and write "<stem>.bf" and "<stem>.txt".
 * Replaces BloomFilterGenerator::generate + BloomFilterInfo sizing
 * (BioBloomMaker/BloomFilterGenerator.cpp:54-73, BloomFilterGenerator.h:108-188,
 * Common/BloomFilterInfo.h:57-76, BioBloomMaker.cpp:360-373,427-543).
 * Sequences (host memory) are seq[offsets[i] .. offsets[i+1]); hash_num 0
 * picks calcOptimalHashNum(fpr).  entries 0 = sum of (len - k + 1).
 */
int bbt_make_filter(const char *seq, const uint64_t *offsets, uint64_t n_seqs,
		unsigned k, double fpr, unsigned hash_num, uint64_t entries,
		const char *stem, const char *filter_id, const char *sources, int device);

/*
 * Classification that allocates no memory, for callers that cannot call
 * cudaMalloc: their device memory belongs to another allocator (a framework's
 * caching allocator, a pool reserved up front with a fixed budget), or they run
 * where cudaMalloc / cudaFree, which can synchronize the whole device, are not
 * acceptable.  No counterpart in the reference.
 *
 * The caller passes device pointers: the filters' bit arrays (bbt_filter_view,
 * as bbt_open would load them from .bf files), the reads (batch->location must
 * be BBT_DEVICE) and the hit words (hits, and hits2 for pairs; same layout as
 * bbt_result).  Results are the same as bbt_classify_batch's hits; no summary
 * counters are kept.  The call is enqueued on `stream` on device
 * params->device.
 *
 * Limits and sharing: at most BBT_NOALLOC_MAX_FILTERS filters (more is
 * rejected with BBT_ERR_ARG).  The kernel's scratch (filter table and work
 * counter) is one small array of device memory per GPU that lives as long as
 * the library is loaded; every call on that GPU shares it, so calls that
 * overlap on the GPU race and must be issued one after another.  Each call
 * looks up the array's device address (cudaGetSymbolAddress) and copies the
 * filter table into it with cudaMemcpyAsync on `stream`.
 */
#define BBT_NOALLOC_MAX_FILTERS 64
typedef struct {
	const void *words;   /* device pointer to the m/8-byte bit array */
	uint64_t m;          /* size in bits, a multiple of 64 */
	unsigned h;          /* hash functions */
	unsigned k;          /* k-mer size */
} bbt_filter_view;
int bbt_classify_noalloc(const bbt_filter_view *filters, int n_filters,
		const bbt_params *params, const bbt_batch *batch, uint64_t *hits,
		uint64_t *hits2, void *stream);

/* ---- machine ceilings ---- */

/* Random 4-byte gathers per second into a table of table_bytes (allocated by
 * the call) on `device`: n_gathers per launch, median of reps launches after
 * one warm-up launch.  position_stream = 1 reads the 32-bit bit positions from
 * device memory (4 bytes per gather, evict-first; table of at most 512 MB),
 * 0 generates them in the kernel.  No counterpart in the reference: it states
 * the ceilings Bloom probes run against (a table inside L2 or in HBM). */
int bbt_measure_gather(int device, uint64_t table_bytes, uint64_t n_gathers,
		int position_stream, int reps, double *gathers_per_s);

/* ---- synthetic workloads (host only; no GPU needed) ---- */

typedef struct {
	uint32_t len_min, len_max;    /* log-uniform length range (equal = fixed) */
	double long_frac;             /* fraction of long reads */
	uint32_t long_min, long_max;  /* log-uniform range of long reads */
	double sub_rate;              /* substitution rate */
	double n_rate;                /* rate of N bases */
	uint32_t frag_min, frag_max;  /* paired: fragment length range */
} bbt_synth_read_params;

/* Random genome: uniform bases at GC fraction gc, then repeat families. */
int bbt_synth_genome(uint64_t seed, uint64_t len, double gc, double repeat_frac,
		uint32_t rep_min, uint32_t rep_max, double div_min, double div_max,
		char *out);
/* Read lengths: out_off[0..n_reads] (prefix sums). */
int bbt_synth_read_lengths(uint64_t seed, const bbt_synth_read_params *p,
		uint64_t n_reads, uint64_t *out_off);
/* Reads drawn from references (ref_frac[j] of reads from reference j, the rest
 * uniform random), filled at the offsets from bbt_synth_read_lengths.  Paired
 * when out2 is non-NULL.  out_src (optional) receives the source index
 * (n_refs = random). */
int bbt_synth_reads(uint64_t seed, const char *refs, const uint64_t *ref_off,
		uint32_t n_refs, const double *ref_frac, const bbt_synth_read_params *p,
		uint64_t n_reads, const uint64_t *off, char *out1, char *out2,
		uint32_t *out_src);

#ifdef __cplusplus
}
#endif
#endif
