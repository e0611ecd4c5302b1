/*
 * classify.cuh -- launch interface of the classification kernels
 * (classify.cu), used by the C ABI layer (api.cu).
 */
#ifndef BBT_CLASSIFY_CUH
#define BBT_CLASSIFY_CUH

#include <cuda_runtime.h>
#include <stdint.h>

#include "bbt_device.cuh"
#if defined(__CUDACC__)
#include "window.cuh"
#endif

namespace bbt {

/* Everything one classify launch needs.  Reads r in [0, n * mates): r < n is
 * read r of mate array 0, otherwise read r - n of mate array 1. */
struct ClassifyArgs {
	const uint8_t *seq[2];     /* ASCII bases, or 2-bit code words when packed */
	const uint32_t *valid[2];  /* packed: validity bits (NULL = all bases ACGT) */
	int packed;                /* bases are BBT_BASES_2BIT */
	const uint64_t *off[2];
	uint64_t off_base[2];      /* subtracted from offsets (staged batches) */
	uint64_t n;                /* reads per mate array */
	uint32_t mates;            /* 1 or 2 */
	const FilterDev *filters;  /* device array of nf filters */
	uint32_t nf;
	uint32_t words;            /* (nf + 63) / 64 */
	double score;              /* SIMPLE threshold */
	double one_minus;          /* 1.0 - score, computed on the host */
	uint32_t streak_thr;
	int scoring;               /* BBT_SCORE_* */
	uint32_t min_len;          /* LENGTH: (unsigned) round(score) */
	uint32_t kmax;             /* largest k among the filters */
	uint64_t *hits[2];         /* n x words per mate array */
	unsigned long long *work;  /* persistent: next read to take (zeroed) */
	const uint64_t *order;     /* persistent: optional order of the reads (a permutation
	                              of [0, n * mates)); NULL = index order */
	const uint32_t *bthres;    /* BINOMIAL: accept threshold of filter f for a read of
	                              n frames at bthres[f * bthres_rows + n] */
	uint64_t bthres_rows;
	const uint32_t *dust[2];   /* -D: bit g set when base g of the mate array lies in a
	                              masked low-complexity interval (dust.cu); NULL = off */
	int tight_steps;           /* SIMPLE scoring: size probe steps by the frames that could
	                              still accept the read (seqeval_chunk.cuh,
	                              simple_step_frames) instead of 32 frames per step */
	unsigned long long *probes;/* optional: filter words read */
	unsigned long long *frames;/* optional: frames hashed */
	unsigned long long *alg_probes; /* optional: words the sequential algorithm reads */
};

/* -D: the frame starting at base g of a mate array is masked (a miss that is
 * not probed, SeqEval's sduster->isLowComp test). */
__device__ __forceinline__ bool dust_low(const uint32_t *mask, uint64_t g)
{
	return mask && ((mask[g >> 5] >> (g & 31u)) & 1u);
}

#if defined(__CUDACC__)
/* The bases of the read starting at base `start` of mate array `mate`. */
__device__ __forceinline__ Bases read_bases(const ClassifyArgs &a, uint32_t mate, uint64_t start)
{
	Bases b;
	b.g0 = start;
	if (a.packed) {
		b.ascii = nullptr;
		b.words = reinterpret_cast<const uint32_t *>(a.seq[mate]);
		b.valid = a.valid[mate];
	} else {
		b.ascii = a.seq[mate];
		b.words = nullptr;
		b.valid = nullptr;
	}
	return b;
}
#endif

struct LaunchConfig {
	int path;             /* BBT_PATH_PLAIN or BBT_PATH_PERSISTENT */
	int warps_per_block;  /* 4 or 8 */
	int seg;              /* frames per lane when hashing: 4 or 8 */
	int num_sms;
	int count;            /* gather probe / frame counters */
	int steps;            /* persistent path: BBT_STEPS_* (bbt_set_steps) */
};

/* Dynamic shared memory one block needs. */
size_t classify_smem_bytes(const LaunchConfig &lc, uint32_t kmax);
cudaError_t launch_classify(const ClassifyArgs &a, const LaunchConfig &lc, cudaStream_t s);

/* Long-first read order for the persistent kernel: reads with at least
 * long_bases bases first, then the others (order within each group is not
 * specified; results do not depend on it).  counters: two zeroed words. */
cudaError_t launch_long_first(const ClassifyArgs &a, uint64_t long_bases, uint64_t *order,
		unsigned long long *counters, int num_sms, cudaStream_t s);

/* Read lengths of a batch (BINOMIAL thresholds): out has 1 + 2048 words,
 * zeroed; out[0] = the largest length, bit L of out[1..] for L < 65536. */
cudaError_t launch_length_set(const uint64_t *off0, const uint64_t *off1, uint64_t n,
		uint32_t mates, unsigned int *out, int num_sms, cudaStream_t s);

/* Categories and summary counters for n reads (or pairs when h2 != NULL):
 * counts = aboveThreshold[nf+2], unique[nf+2], multiMatch, noMatch.
 * ordered (-c): only the first filter of the read's hits (pairs: of the
 * intersection, or of the union with inclusive) counts, and the hit words
 * of both mates are rewritten to that one filter. */
cudaError_t launch_summarize(uint64_t *h1, uint64_t *h2, uint64_t n, uint32_t nf,
		uint32_t words, int inclusive, int ordered, uint32_t *category,
		unsigned long long *counts, int num_sms, cudaStream_t s);

/* Exhaustive per-filter scores (SeqEval::evalScore) of the reads of a
 * ClassifyArgs batch (score.cu).  scores[m] (optional): n x nf doubles of mate
 * array m.  besthit: also write, as a.hits, the filters of the largest score. */
struct ScoreArgs {
	double *scores[2];
	const double *fpr;   /* BINOMIAL: each filter's FPR (getFPRPrecompute) */
	int besthit;
};
cudaError_t launch_scores(const ClassifyArgs &a, const ScoreArgs &sa, const LaunchConfig &lc,
		cudaStream_t s);
/* BESTHIT hit words (a.hits) from stored scores (n x nf per mate array). */
cudaError_t launch_best_hits(const ClassifyArgs &a, double *const *scores, int num_sms,
		cudaStream_t s);

} // namespace bbt

#endif
