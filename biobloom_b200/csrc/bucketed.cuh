/*
 * bucketed.cuh -- launch interface of the bucketed probe path (bucketed.cu),
 * used by the C ABI layer (api.cu) for filters much larger than L2.
 */
#ifndef BBT_BUCKETED_CUH
#define BBT_BUCKETED_CUH

#include <cuda_runtime.h>
#include <stdint.h>

#include "classify.cuh"

namespace bbt {

/* Frames per window block: a frame's id inside its window fits 16 bits. */
constexpr uint32_t kBkWinFrames = 32768;
constexpr int kBkWinThreads = 256;
/* Phase boundaries are given in sixteenths of a read's frames. */
constexpr uint32_t kBkPhaseDen = 16;

/* A mate array's bases as 2-bit codes (16 per word, base g at bits 2 (g % 16)
 * of word g / 16) and validity bits (base g at bit g % 32 of word g / 32; NULL
 * when every base is ACGT); words past the ends read as 0. */
struct PackedBases {
	const uint32_t *words;
	uint64_t nwords;
	const uint32_t *valid;
	uint64_t nvalid;
};

struct BucketArgs {
	ClassifyArgs a;            /* the batch: offsets, scoring, DUST masks, hit words */
	PackedBases pk[2];         /* its bases, per mate array */
	FilterDev f;               /* the filter of this pass */
	uint32_t fbit;             /* its index: hit word fbit / 64, bit fbit % 64 */
	uint64_t r0, nr;           /* reads [r0, r0 + nr) of the batch's read space */
	const uint64_t *fo;        /* frame offsets of the batch's reads (n * mates + 1) */
	uint64_t fo0;              /* fo[r0] */
	uint64_t T;                /* frames of the sub-batch: fo[r0 + nr] - fo0 */
	uint32_t nblk;             /* window blocks: ceil(T / kBkWinFrames) */
	uint32_t *vbits;           /* bit t: frame t of the sub-batch holds only ACGT */
	uint32_t *hbits;           /* bit t: frame t is still a hit (all levels so far) */
	uint32_t *abits;           /* bit t: frame t requests tests in this phase */
	uint64_t *canon;           /* canonical ntHash of every requesting frame */
	uint8_t *state;            /* per read of the batch: 0 open, 1 decided */
	uint32_t ph_lo, ph_hi;     /* this phase: frames [bound(F, ph_lo), bound(F, ph_hi)) */
	uint32_t ph_min;           /* bound(F, q) >= min(F, ph_min) for q > 0 */
	uint32_t level, nlevels;   /* hash functions of this round: [level, level + nlevels)
	                              (0 = the canonical hash); a frame requests them all */
	uint32_t nbkt, bshift;     /* bucket of bit p: p >> bshift */
	uint32_t *cnt;             /* this round's requests per (bucket, window block):
	                              [nbkt][nblk] */
	uint32_t *loc;             /* their first slot in the block's region of the pool */
	uint64_t cap;              /* pool slots per window block */
	uint32_t *req_off;         /* request pool: bit offset inside the bucket */
	uint16_t *req_fid;         /*   frame id inside the window block */
	uint8_t *res;              /*   test result (1 = bit set) */
	uint32_t *btot;            /* requests of this round per window block */
	unsigned long long *issued;/* optional: requests resolved (bit tests issued) */
	unsigned long long *next;  /* resolve: next segment to take (zeroed before the launch) */
};

/* fo[i + 1] = frames of read i (n * mates reads); the caller scans it. */
cudaError_t launch_bk_frame_counts(const ClassifyArgs &a, unsigned k, uint64_t *fo_plus1,
		int num_sms, cudaStream_t s);
/* out[j] = fo[min(j * stride, total)], j < n. */
cudaError_t launch_bk_samples(const uint64_t *fo, uint64_t total, uint64_t stride, uint64_t *out,
		uint64_t n, int num_sms, cudaStream_t s);
/* ASCII bases [0, len) into 2-bit codes (len / 16 + 2 words) and validity
 * bits (len / 32 + 2 words). */
cudaError_t launch_bk_pack(const uint8_t *ascii, uint64_t len, uint32_t *words, uint32_t *valid,
		int num_sms, cudaStream_t s);
/* A phase's first round: hash the phase's frames of the open reads, set their
 * validity / hit / requesting bits, keep their canonical hashes and write
 * their level-0 requests, sorted by bucket in each block's region. */
cudaError_t launch_bk_hash(const BucketArgs &b, cudaStream_t s);
/* A later round: the previous round's results applied to the hit bits, then
 * requests of the frames still hits, levels [level, level + nlevels). */
cudaError_t launch_bk_emit(const BucketArgs &b, cudaStream_t s);
/* A round's bit tests, bucket by bucket (the bucket held in L2), one result
 * byte per request. */
cudaError_t launch_bk_resolve(const BucketArgs &b, int num_sms, cudaStream_t s);
/* The last round's results applied to the hit bits. */
cudaError_t launch_bk_apply(const BucketArgs &b, cudaStream_t s);
/* SeqEval over [0, bound(F, ph_hi)) of every open read; accepted reads set
 * their hit bit; reads decided or fully walked are closed. */
cudaError_t launch_bk_walk(const BucketArgs &b, int num_sms, cudaStream_t s);

/* Dynamic shared memory of the hashing / emitting kernels for nbkt buckets. */
size_t bk_sweep_smem(uint32_t nbkt);

} // namespace bbt

#endif
