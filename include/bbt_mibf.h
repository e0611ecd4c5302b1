/*
 * bbt_mibf.h -- C ABI of the multi-index Bloom filter (miBF) path of
 * libbbt.so: biobloommicategorizer's classification on the GPU.
 *
 * Drop-in boundary for the reference's MIBFClassifier
 * (BioBloomCategorizer/MIBFClassifier.hpp) and its miBF data structure (the
 * btl_bloomfilter submodule's MIBloomFilter / MIBFQuerySupport, which the
 * reference tree does not hold; their semantics are fixed in this header).
 * Conventions are those of bbt.h: int status codes (BBT_OK / BBT_ERR_*), the
 * caller owns host buffers, a context owns its device memory and is used from
 * one host thread at a time, streams are passed as void*.
 *
 * Semantics shared by every entry point:
 *   Frames.  A frame is a span of k bases (k <= 32) all of which are A, C, G
 *     or T (either case).  With spaced seeds (strings of '0'/'1' of length k)
 *     each seed gives one value per frame: F = XOR over the seed's '1'
 *     positions j of rol(s(x_j), k-1-j), R = XOR of rol(s_rc(x_j), j) with
 *     ntHash's base seeds s and their complements s_rc, value = min(F, R).
 *     Without seeds (k-mer mode) the values are the canonical ntHash of the
 *     k-mer and its h-1 extra hashes.
 *   Filter.  Bit vector of m bits (a multiple of 64); value v probes bit
 *     v mod m; a set bit p owns the 16-bit ID slot rank(p) (set bits before p);
 *     an ID's low 15 bits are the target ID (0 = none), bit 15 marks a
 *     saturated slot.
 *   Files.  "<p>.bf": a text header "[BTLMIBloomFilter]" ... "[HeaderEnd]"
 *     (keys Format, BitVectorSize, HashNum, KmerSize, IDWidth, Seeds,
 *     PopCount) followed by PopCount little-endian uint16 IDs; "<p>.sdsl": the
 *     m/64 little-endian uint64 words of the bit vector; "<p>_ids.txt": one
 *     "<id>\t<name>" line per target (MIBFClassifier.hpp:52-76 reads it).
 *   Query (per read, or per pair with the frames of both mates pooled).  For
 *     each frame and value a hit gives the slot's ID and saturation.  Per ID:
 *     totalCount = hits, totalNonSatCount = unsaturated hits, count = frames
 *     with at least h - allowedMiss hits, nonSatCount = frames with at least
 *     h - allowedMiss unsaturated hits, solidCount = frames all of whose h
 *     values hit the ID, nonSatFrameCount = frames counted in count that hold
 *     no saturated hit of any ID; satCount = frames holding a saturated hit.
 *     allowedMiss = h - frameMatches (0 in k-mer mode or when frameMatches >
 *     h; MIBFClassifier.hpp:79-82).  An ID is significant when count >=
 *     minCount and (min_nonsat == 0 or nonSatCount >= min_nonsat); minCount =
 *     max(1, smallest x with P(X > x) <= score / n_targets) for X ~
 *     Binomial(frameCount, perFrameProb[id]) (getMinCount,
 *     MIBFClassifier.hpp:930-939), perFrameProb[id] = P(at least
 *     h - allowedMiss of h values hit the ID) with per-value probability
 *     (slots owned by the ID) / m.  frameCount = len - k + 1 (0 when len < k);
 *     for a pair it is read 1's frame count, or read 2's when read 1 is
 *     shorter than k (MIBFClassifier.hpp:802-803 as the C++ grammar parses
 *     it).  Significant IDs are ordered by count, nonSatCount, totalCount
 *     (descending), then ID; the result lists the first and every other with
 *     count > first.count - multi_thresh.  With best_hit_agree the result is
 *     empty unless the first also has the highest nonSatCount.
 */
#ifndef BBT_MIBF_H
#define BBT_MIBF_H

#include <stddef.h>
#include <stdint.h>

#include "bbt.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct bbt_mibf bbt_mibf;

/* Output record types of formatOutStr (MIBFClassifier.hpp:675-736). */
#define BBT_MIBF_OUT_TSV 0
#define BBT_MIBF_OUT_FASTA 1
#define BBT_MIBF_OUT_FASTQ 2

/* Device layouts of the filter (bbt_mibf_params.layout). */
#define BBT_MIBF_LAYOUT_AUTO 0   /* dense when it fits comfortably in free HBM */
#define BBT_MIBF_LAYOUT_RANK 1   /* bit vector in 32-byte rank blocks + ID array:
                                    m/7 + 2*PopCount bytes, two reads per hit */
#define BBT_MIBF_LAYOUT_DENSE 2  /* one 16-bit entry per bit: 2*m bytes, one read
                                    per probe */

/* Options of biobloommicategorizer (BioBloomMICategorizer.cpp:78-122). */
typedef struct {
	double score;            /* p-value threshold; -s N sets 10^(-N/10). [1e-10] */
	unsigned frame_matches;  /* -a [1] */
	double multi_thresh;     /* -m [1.0] */
	unsigned streak;         /* -r [3]; the query visits every frame either way */
	unsigned min_nonsat;     /* -c [0] */
	int best_hit_agree;      /* -b */
	int hit_only;            /* -i: for pairs, empty results are left out of the
	                            summary as well (MIBFClassifier.hpp:750-763) */
	int device;              /* CUDA device ordinal */
	uint64_t max_batch_bases;  /* staging capacity per host batch; 0 = default */
	uint64_t max_batch_reads;
	int layout;              /* BBT_MIBF_LAYOUT_*; no reference counterpart */
} bbt_mibf_params;

void bbt_mibf_default_params(bbt_mibf_params *p);

/*
 * Load "<p>.bf", "<p>.sdsl" and "<p>_ids.txt" (bf_path = "<p>.bf") and build
 * the device layout (bit vector with interleaved rank counts, ID array) once.
 * Replaces MIBFClassifier::MIBFClassifier (MIBFClassifier.hpp:49-94) and
 * MIBloomFilter's file constructor.  Names: id 0 is "repeat", then the
 * names of the ID file in order.
 */
int bbt_mibf_open(const char *bf_path, const bbt_mibf_params *params, bbt_mibf **out);
int bbt_mibf_close(bbt_mibf *ctx);
const char *bbt_mibf_last_error(const bbt_mibf *ctx);
/* The layout the context built (BBT_MIBF_LAYOUT_RANK or _DENSE). */
int bbt_mibf_layout(const bbt_mibf *ctx);
/* Targets + 1 (m_fullIDs.size()). */
unsigned bbt_mibf_num_ids(const bbt_mibf *ctx);
const char *bbt_mibf_id_name(const bbt_mibf *ctx, unsigned id);
/* Header values: bits, values per frame, span, number of seeds. */
int bbt_mibf_info(const bbt_mibf *ctx, uint64_t *m, unsigned *h, unsigned *k,
		unsigned *n_seeds);
/* perFrameProb[0..num_ids) and the fraction of saturated slots
 * (MIBloomFilter::calcFrameProbs, MIBFClassifier.hpp:87-89). */
int bbt_mibf_frame_probs(const bbt_mibf *ctx, double *probs, double *rate_saturated);

/* One significant ID of a read (MIBFQuerySupport::QueryResult). */
typedef struct {
	uint32_t id;
	uint32_t nonSatFrameCount, solidCount, count, nonSatCount, totalNonSatCount, totalCount;
} bbt_mibf_hit;

/*
 * Per-read results: n_hits[i] = number of significant IDs of read (pair) i,
 * hits[i * max_hits ..] the first min(n_hits[i], max_hits) of them in result
 * order, sat_count[i] = satCount.  When some read has more than max_hits
 * results the call returns BBT_ERR_OVERFLOW after writing everything else;
 * n_hits stays exact, so the caller can retry with a larger max_hits.
 */
#define BBT_ERR_OVERFLOW (-9)
typedef struct {
	bbt_mibf_hit *hits;
	uint32_t max_hits;
	uint32_t *n_hits;
	uint32_t *sat_count;
	int location;            /* BBT_HOST or BBT_DEVICE */
} bbt_mibf_result;

/*
 * Classify a batch (bbt_batch of bbt.h; pairs when seq2 != NULL) and add it to
 * the summary counters.  Replaces MIBFClassifier::classify (single,
 * MIBFClassifier.hpp:772-796; paired, :801-834) over every read of the batch.
 * Host buffers: returns when the results are in place; the reads go through
 * the device in chunks of up to 1M reads, each chunk's copies overlapping the
 * classification of the one before (pinned host arrays overlap best), with
 * the results and summary of a single launch.  Device buffers: runs on
 * `stream` (NULL = the context's stream) and returns when enqueued, except
 * that the first batch with a new read length waits for the minCount table.
 */
int bbt_mibf_classify_batch(bbt_mibf *ctx, const bbt_batch *batch, bbt_mibf_result *result,
		void *stream);
int bbt_mibf_sync(bbt_mibf *ctx);
/* The bucketed query of the dense layout: every probe of a sub-batch of reads
 * sorted by address and read out of L2 one bucket of 2^bucket_shift entries
 * at a time before the reads are tallied.  mode 0 off (the default: on B200
 * the direct kernel measured faster on the 500-target workload), 1 on (dense
 * layout), 2 on for batches of 2^20 reads or more over an ID map of 256 MB or
 * more; bucket_shift default 23 (16 MB); at most max_frames frames per
 * sub-batch (default 2^30; scratch about 8 h + 2 h + 1 bytes per frame);
 * 0 keeps a setting.  Results do not depend on them; the serving engine's
 * concurrent slots always take the direct kernel.  No reference counterpart. */
int bbt_mibf_set_bucketing(bbt_mibf *ctx, int mode, unsigned bucket_shift, uint64_t max_frames);
/* Device time of the query kernel of the last batch, in milliseconds (known
 * once the batch is done: after a host batch returns, or after bbt_mibf_sync). */
double bbt_mibf_last_kernel_ms(bbt_mibf *ctx);
/* Work of the last batch (waits for it): out[0] frames visited (spans of k
 * valid bases), out[1] values probed (frames x h), out[2] probes that found a
 * set bit (each of which read an ID).  No reference counterpart. */
int bbt_mibf_last_counts(bbt_mibf *ctx, uint64_t *out);

/*
 * Summary counters (ResultsManager<ID>::updateSummaryData over query results,
 * ResultsManager.hpp:40-64): counts holds 2 * (num_ids + 2) + 2 uint64:
 * aboveThreshold[num_ids + 2], unique[num_ids + 2], multiMatch, noMatch.
 */
int bbt_mibf_summary(bbt_mibf *ctx, uint64_t *counts, uint64_t *reads);
int bbt_mibf_reset_summary(bbt_mibf *ctx);
/* "<prefix>_summary.tsv" text for read_count reads
 * (ResultsManager::getResultsSummary, ResultsManager.hpp:191-237). */
int bbt_mibf_summary_tsv(bbt_mibf *ctx, uint64_t read_count, char *buf, size_t cap,
		size_t *len);

/*
 * File pipeline of biobloommicategorizer: parse FASTA/FASTQ into pinned double
 * buffered batches, classify, write one record per read (pair) to `out`
 * (a FILE*, e.g. stdout; records in input order) and "<prefix>_summary.tsv".
 * Replaces MIBFClassifier::filter (MIBFClassifier.hpp:200-407) and
 * filterPair (:409-616).  out_type: BBT_MIBF_OUT_*.
 */
int bbt_mibf_filter_files(bbt_mibf *ctx, const char *const *files, int n_files,
		const char *prefix, int out_type, void *out);
int bbt_mibf_filter_pair_files(bbt_mibf *ctx, const char *file1, const char *file2,
		const char *prefix, int out_type, void *out);

/* ---- host-side pieces (no GPU needed) ---- */

/* getMinCount (MIBFClassifier.hpp:930-939) for frame_count frames. */
unsigned bbt_mibf_min_count(unsigned frame_count, double frame_prob, double score,
		unsigned num_ids);
/* Append one record of read (name, comment, seq, qual) for results `hits`
 * (n_hits of them) to buf (formatOutStr, MIBFClassifier.hpp:675-736); names
 * from the context.  Writes at most cap bytes incl. NUL; *len = full length. */
int bbt_mibf_format_record(const bbt_mibf *ctx, int out_type, const char *name,
		const char *comment, const char *seq, const char *qual, const bbt_mibf_hit *hits,
		uint32_t n_hits, uint32_t sat_count, char *buf, size_t cap, size_t *len);
/* Load only the host parts of a miBF (names, header, ID array) for the
 * host-side entry points above; no device memory is touched. */
int bbt_mibf_open_host(const char *bf_path, const bbt_mibf_params *params, bbt_mibf **out);

/*
 * Build a miBF on the device and write "<prefix>.bf", "<prefix>.sdsl" and
 * "<prefix>_ids.txt".  Replaces MIBFGen::generate (BioBloomMaker/MIBFGen.hpp:
 * 131-430).  Sequences are seq[offsets[i] .. offsets[i+1]) with target ID
 * seq_id[i] (1-based; names[id - 1] is its name, n_names names).  seeds:
 * n_seeds strings of length k, or none for k-mer mode with hash_num values.
 * m = ceil(n * h / -ln(1 - occupancy)) rounded up to a multiple of 64,
 * n = sum of (len - k + 1).  Slot owners: of the IDs whose values land in a
 * slot, the one with the largest (p << 16 | id), p = the top 16 bits of
 * splitmix64's finalizer of (slot ^ id * 0x9e3779b97f4a7c15); then every
 * (sequence, frame) none of whose slots its ID owns marks all its slots
 * saturated.  Every step is order-free, so the file is the same on every run.
 * location: BBT_HOST or BBT_DEVICE for seq/offsets/seq_id.
 */
int bbt_mibf_make(const char *seq, const uint64_t *offsets, const uint16_t *seq_id,
		uint64_t n_seqs, const char *const *names, unsigned n_names,
		const char *const *seeds, unsigned n_seeds, unsigned k, unsigned hash_num,
		double occupancy, int location, const char *prefix, int device);

#ifdef __cplusplus
}
#endif
#endif
