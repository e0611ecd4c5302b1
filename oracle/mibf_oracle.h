/*
 * mibf_oracle.h -- CPU oracle for the multi-index Bloom filter (miBF) path
 * of biobloommicategorizer.  TEST INFRASTRUCTURE ONLY (see bbt_oracle.h).
 *
 * The miBF structures and query live in the btl_bloomfilter submodule
 * (MIBloomFilter.hpp, MIBFQuerySupport.hpp, MIBFConstructSupport.hpp,
 * vendor/stHashIterator.hpp), which is absent from the reference tree.  They are
 * restated here from the published method (Chu et al., "Multi-index Bloom
 * filters", PNAS 2020) and from what the reference's call sites show
 * (BioBloomCategorizer/MIBFClassifier.hpp:49-94, 652-796, 930-939;
 * BioBloomMaker/MIBFGen.hpp:131-430; Tests/ntHashTests.cpp).  Every choice the
 * sources leave open is fixed here and written down:
 *
 *  Spaced seeds.  A seed is a string of '0'/'1' of length k (the span); '1'
 *  positions are the care positions.  For seed s and span x[0..k):
 *    F = XOR_{j care} rol(seed(x_j), k-1-j),  R = XOR_{j care} rol(seed_rc(x_j), j)
 *  with ntHash's base seeds, and the seed's hash is min(F, R).  Then
 *  hash(s, x) = hash(reverse(s), revcomp(x)), the symmetry Tests/ntHashTests.cpp
 *  asserts.  A frame is visited when all k bases of its span are ACGT.
 *  Without seeds (k-mer mode) a frame's h values are ntHash's h hashes.
 *
 *  Bit vector and IDs.  m bits, m = n*h / -ln(1 - occupancy) rounded up to a
 *  multiple of 64 (n = sum of len-k+1).  Set bit p owns ID slot rank(p) (set
 *  bits before p).  IDs are 16-bit: 0 is EMPTY, the high bit marks saturation.
 *
 *  Construction (3 passes, MIBFGen.hpp:131-309): (1) set the bit of every
 *  frame's h values; (2) every (sequence ID, frame, value) offers its ID to the
 *  value's slot and the slot keeps the offer with the largest
 *  (priority(slot, id) << 16 | id), priority = top 16 bits of
 *  mix64(slot ^ id * 0x9e3779b97f4a7c15) -- a pseudo-random, order-free choice
 *  of owner among colliding IDs; (3) for every (sequence ID, frame) none of
 *  whose h slots is owned by that ID, all h slots get the saturation bit.
 *
 *  Query (MIBFQuerySupport::query).  For each visited frame and value v:
 *  a hit when bit v mod m is set, giving id and saturation from its slot.  Per
 *  ID over the read (pair): totalCount = hits, totalNonSatCount = unsaturated
 *  hits, count = frames with at least (h - allowedMiss) hits, nonSatCount =
 *  frames with at least (h - allowedMiss) unsaturated hits, solidCount = frames
 *  where all h values hit it, nonSatFrameCount = frames counted in count that
 *  hold no saturated hit of any ID.  satCount = frames with a saturated hit.
 *  An ID is significant when count >= minCount[id] (and nonSatCount >=
 *  minNonSat when that is > 0).  Significant IDs are ordered by count, then
 *  nonSatCount, then totalCount (descending), then ID; the result lists the
 *  first and every other with count > first.count - multiThresh.  With
 *  bestHitAgree, the result is empty when the highest nonSatCount belongs to
 *  another ID than the first.  The query visits every frame (no early exit).
 *
 *  Frame probabilities (MIBloomFilter::calcFrameProbs): with p_id = slots owned
 *  by id / m, perFrameProb[id] = P(at least h - allowedMiss of h values hit id)
 *  = sum_{j >= h-allowedMiss} C(h,j) p^j (1-p)^(h-j); the return value is the
 *  fraction of saturated slots.
 *
 *  Files.  <p>.bf: text header "[BTLMIBloomFilter]" ... "[HeaderEnd]" (keys
 *  BitVectorSize, HashNum, KmerSize, Seeds, PopCount) then the PopCount 16-bit
 *  IDs; <p>.sdsl: the m/64 64-bit words of the bit vector (raw, not sdsl's
 *  serialization); <p>_ids.txt: "<id>\t<name>" lines (MIBFGen.hpp:424-430).
 */
#ifndef MIBF_ORACLE_H
#define MIBF_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ORACLE_MIBF_MAX_SEEDS 16
#define ORACLE_MIBF_EMPTY 0
#define ORACLE_MIBF_SAT 0x8000u

typedef struct {
	uint64_t m;          /* bits, multiple of 64 */
	unsigned h;          /* values per frame (seeds, or hashes in k-mer mode) */
	unsigned k;          /* span */
	unsigned nseeds;     /* 0 = k-mer mode */
	char seeds[ORACLE_MIBF_MAX_SEEDS][256];
	uint64_t *bv;        /* m/64 words */
	uint64_t *rank_word; /* set bits before each word */
	uint16_t *ids;       /* pop entries */
	uint64_t pop;
} oracle_mibf;

/* Values of the frame at x (span k): seed hashes, or ntHash hashes. */
void oracle_mibf_values(const oracle_mibf *f, const char *x, uint64_t *out);
/* 1 if all k bases at x are ACGT. */
int oracle_mibf_frame_ok(const oracle_mibf *f, const char *x);
/* Spaced-seed hash of seed string s (length k) on span x. */
uint64_t oracle_st_hash(const char *seed, unsigned k, const char *x);

/* Build from n sequences; seq_id[i] is sequence i's ID (1-based).
 * seeds: nseeds strings of length k, or NULL/0 for k-mer mode with h hashes. */
int oracle_mibf_build(oracle_mibf *f, const char *const *seqs, const uint64_t *lens,
		const uint16_t *seq_id, size_t n, const char *const *seeds, unsigned nseeds,
		unsigned k, unsigned h, double occupancy);
void oracle_mibf_free(oracle_mibf *f);
int oracle_mibf_store(const oracle_mibf *f, const char *prefix);
int oracle_mibf_load(oracle_mibf *f, const char *bf_path);
uint64_t oracle_mibf_rank(const oracle_mibf *f, uint64_t pos);
/* perFrameProb for ids 0..nids-1; returns the fraction of saturated slots. */
double oracle_mibf_frame_probs(const oracle_mibf *f, double *probs, unsigned nids,
		unsigned allowed_miss);

typedef struct {
	uint16_t id;
	uint32_t nonSatFrameCount, solidCount, count, nonSatCount, totalNonSatCount, totalCount;
} oracle_qres;

/* Query one read, or a pair when seq2 != NULL (frames of both mates pooled).
 * Returns the number of results written (<= max_out). */
unsigned oracle_mibf_query(const oracle_mibf *f, const char *seq, size_t len,
		const char *seq2, size_t len2, const uint32_t *min_count, unsigned nids,
		double multi_thresh, unsigned allowed_miss, unsigned min_nonsat, int best_agree,
		oracle_qres *out, unsigned max_out, uint32_t *sat_count, uint64_t *lookups);

/* binomial: smallest x with P(X > x) <= q (the reference's
 * quantile(complement(...)) under integer_round_up) */
unsigned oracle_binom_upper_quantile(unsigned n, double p, double q);

#ifdef __cplusplus
}
#endif
#endif
