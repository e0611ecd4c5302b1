/*
 * bbt_oracle.h -- CPU oracle for the BioBloom Tools read-classification path.
 *
 * TEST INFRASTRUCTURE ONLY.  The GPU path's results are compared with this
 * oracle's.  Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline
 * leg may load it; the product library never links or calls it.
 *
 * What it restates (reference paths are relative to the biobloom project):
 *   - ntHash rolling canonical multi-hash and the k-mer iterator that skips
 *     k-mers containing a non-ACGT base.  The implementation lives in the
 *     btl_bloomfilter submodule (vendor/nthash.hpp, vendor/ntHashIterator.hpp),
 *     which is absent from the reference tree; this is restated from the
 *     published method (Mohamadi et al., "ntHash: recursive nucleotide
 *     hashing", Bioinformatics 2016).  Call sites: Common/SeqEval.h:50,302.
 *   - BloomFilter bit test / insert and the .bf file (btl_bloomfilter
 *     BloomFilter.hpp, also absent).  Call sites: Common/SeqEval.h:54,78,
 *     BioBloomCategorizer/BioBloomClassifier.cpp:962.
 *   - SeqEval::evalSimple (Common/SeqEval.h:37-114) and
 *     SeqEval::evalMinMatchLen (Common/SeqEval.h:295-332).
 *   - BloomFilterInfo sizing (Common/BloomFilterInfo.h:57-76) and the .txt
 *     INI sidecar (Common/BloomFilterInfo.cpp:31-53, 81-116).
 *   - ResultsManager::updateSummaryData and getResultsSummary
 *     (BioBloomCategorizer/ResultsManager.hpp:66-237).
 *
 * Parity status: the submodule's own hash values and .bf header bytes are not
 * available, so parity with filters built by upstream biobloommaker is
 * unpinned.  The oracle is pinned against the reference's own driver code
 * (SeqEval.h, ResultsManager.hpp, BioBloomClassifier.cpp) compiled from the
 * reference sources in oracle/_ref (see oracle/Makefile) and against the
 * properties the reference tests assert (Tests/BloomFilterTests.cpp,
 * Tests/SeqEvalTests.cpp).
 */
#ifndef BBT_ORACLE_H
#define BBT_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------- ntHash ---------------- */

/* 64-bit seed of a base ('A','C','G','T', either case); 0 for anything else. */
uint64_t oracle_nt_seed(unsigned char c);
/* Seed of the complementary base. */
uint64_t oracle_nt_seed_rc(unsigned char c);
/* 1 if c is one of ACGTacgt. */
int oracle_nt_valid(unsigned char c);

/* Forward / reverse-complement / canonical hash of the k-mer at s (direct). */
uint64_t oracle_nt_forward(const char *s, unsigned k);
uint64_t oracle_nt_reverse(const char *s, unsigned k);
/* Extra hash i (i >= 1) derived from the canonical hash. */
uint64_t oracle_nt_extra(uint64_t canon, unsigned k, unsigned i);

/* k-mer iterator with the ntHashIterator contract: yields, in increasing
 * position order, exactly the k-mers with no non-ACGT base; pos() of the end
 * state is SIZE_MAX. */
typedef struct {
	const char *seq;
	size_t len;
	unsigned k, h;
	size_t pos;         /* start of the current k-mer; SIZE_MAX at end */
	uint64_t fh, rh;    /* forward / reverse-complement hashes */
	uint64_t hv[64];    /* h hash values of the current k-mer */
} oracle_ntitr;

void oracle_ntitr_init(oracle_ntitr *it, const char *seq, size_t len,
		unsigned h, unsigned k);
void oracle_ntitr_next(oracle_ntitr *it);
static inline int oracle_ntitr_end(const oracle_ntitr *it)
{
	return it->pos == (size_t)-1;
}

/* ---------------- Bloom filter ---------------- */

typedef struct {
	uint64_t m;          /* size in bits */
	unsigned h;          /* hash functions */
	unsigned k;          /* k-mer size */
	double dfpr;         /* desired FPR written in the header */
	uint64_t n_entry;    /* new k-mers inserted (order dependent) */
	uint64_t t_entry;    /* total k-mers offered */
	uint8_t *bits;       /* m/8 bytes (m is padded to a multiple of 64) */
} oracle_bf;

int oracle_bf_create(oracle_bf *bf, uint64_t m, unsigned h, unsigned k);
void oracle_bf_free(oracle_bf *bf);
/* Bit test with short circuit; adds the number of bit reads to *probes. */
int oracle_bf_contains(const oracle_bf *bf, const uint64_t *hv, uint64_t *probes);
void oracle_bf_insert(oracle_bf *bf, const uint64_t *hv);
/* Returns 1 if every bit was already set before the insert. */
int oracle_bf_insert_check(oracle_bf *bf, const uint64_t *hv);
int oracle_bf_store(const oracle_bf *bf, const char *path);
int oracle_bf_load(oracle_bf *bf, const char *path);

/* BloomFilterInfo sizing (Common/BloomFilterInfo.h:57-76). */
uint64_t oracle_calc_optimal_size(uint64_t entries, double fpr, unsigned h);
unsigned oracle_calc_optimal_hash_num(double fpr);

/* Build a filter from n sequences the way biobloommaker does
 * (BioBloomMaker/BloomFilterGenerator.h:108-188): expected entries =
 * sum(len-k+1), size from calcOptimalSize, every valid k-mer inserted. */
int oracle_make_filter(oracle_bf *bf, const char *const *seqs,
		const uint64_t *lens, size_t n, unsigned k, double fpr, unsigned h,
		uint64_t *expected_entries, uint64_t *redundant);
/* Write the .txt INI sidecar (Common/BloomFilterInfo.cpp:81-116 layout). */
int oracle_write_info(const char *path, const char *filter_id, unsigned k,
		double fpr, unsigned h, uint64_t expected, const char *sources,
		uint64_t size, uint64_t num_entries, double approx_fpr,
		uint64_t redundant, double redundant_fpr);

/* ---------------- SeqEval ---------------- */

/* SeqEval::evalSimple on one read.  probes (optional) accumulates the number
 * of filter bit reads the sequential algorithm performs. */
int oracle_eval_simple(const char *seq, size_t len, const oracle_bf *bf,
		double threshold, unsigned streak_threshold, uint64_t *probes);
/* SeqEval::evalMinMatchLen (LENGTH scoring, -s N with N > 1). */
int oracle_eval_min_match_len(const char *seq, size_t len,
		const oracle_bf *bf, unsigned min_match_len, uint64_t *probes);

/* SeqEval::evalHarmonic (HARMONIC scoring, -S harmonic). */
int oracle_eval_harmonic(const char *seq, size_t len, const oracle_bf *bf,
		double threshold, unsigned streak_threshold, uint64_t *probes);
/* SeqEval::evalBinomial (BINOMIAL scoring, -S binomial): threshold is the
 * minimum FPR of a match (10^(-s/10)), fpr the filter's (set bits / m)^h. */
int oracle_eval_binomial(const char *seq, size_t len, const oracle_bf *bf,
		double threshold, double fpr, unsigned streak_threshold, uint64_t *probes);
double oracle_bf_fpr(const oracle_bf *bf);
/* Binomial(n, p): smallest x with P(X > x) <= q, summed from the top of the
 * tail (boost's quantile(complement(...)) under integer_round_up). */
unsigned oracle_binom_upper_quantile(unsigned n, double p, double q);
unsigned oracle_calc_min_count(unsigned frame_len, double bf_fpr, double min_fpr);

/* SDUST (Common/sdust.c, through Common/SDust.hpp): masked intervals of one
 * read as start << 32 | finish (finish exclusive), at most cap written;
 * returns how many there are.  max_perfect (optional): the largest number
 * of pending perfect intervals held at once. */
int oracle_sdust(const char *seq, size_t len, int T, int W, uint64_t *out, int cap,
		int *max_perfect);
/* -D: every oracle_eval_* and the batch drivers treat frames starting in a
 * masked interval as misses without a probe (off by default). */
void oracle_set_dust(int on, int T, int W);

/* ---------------- Batch driver + summary ---------------- */

/* Scoring methods, in the order of opt::ScoringMethod (Common/Options.h:35). */
enum { ORACLE_SIMPLE = 0, ORACLE_LENGTH = 1, ORACLE_HARMONIC = 2, ORACLE_BINOMIAL = 3 };

/* Classify reads against nf filters (evaluateReadStd,
 * BioBloomClassifier.cpp:1182-1189).  Reads are seq[off[i] .. off[i+1]).
 * hits: n x words uint64 bitmask (words = (nf+63)/64). */
void oracle_classify(const char *seq, const uint64_t *off, size_t n,
		const oracle_bf *const *filters, unsigned nf, double threshold,
		unsigned streak_threshold, int scoring, uint64_t *hits,
		uint64_t *probes);

/* Exhaustive scores (SeqEval::evalScore, Common/SeqEval.h:534-560) and the
 * modes built on them and on the STD hits: BESTHIT, ORDERED. */
double oracle_binom_sf(unsigned n, double p, unsigned x);
double oracle_eval_score(const char *seq, size_t len, const oracle_bf *bf, int scoring,
		unsigned streak_threshold, double fpr);
void oracle_classify_scores(const char *seq, const uint64_t *off, size_t n,
		const oracle_bf *const *filters, unsigned nf, int scoring,
		unsigned streak_threshold, double *scores);
double oracle_best_hit(const double *scores, unsigned nf, uint64_t *hits);
void oracle_ordered(uint64_t *hits1, uint64_t *hits2, unsigned nf, int inclusive);

/* Summary accounting (ResultsManager.hpp:66-189).  counts has nf+2 entries
 * of aboveThreshold then nf+2 entries of unique, then multiMatch, noMatch.
 * Returns the category index (filter, nf = noMatch, nf+1 = multiMatch). */
unsigned oracle_update_summary(uint64_t *counts, unsigned nf,
		const uint64_t *hits);
unsigned oracle_update_summary_pair(uint64_t *counts, unsigned nf,
		const uint64_t *hits1, const uint64_t *hits2, int inclusive);
/* summary.tsv text (ResultsManager.hpp:191-237); returns bytes written
 * (excluding NUL) or the size needed if cap is too small. */
size_t oracle_summary_tsv(const uint64_t *counts, unsigned nf,
		const char *const *ids, uint64_t read_count, char *out, size_t cap);

#ifdef __cplusplus
}
#endif
#endif
