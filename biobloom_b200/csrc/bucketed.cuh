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

struct BucketArgs {
	ClassifyArgs a;            /* the batch: bases, offsets, scoring, hit words */
	FilterDev f;               /* the filter of this pass */
	uint32_t fbit;             /* its index: hit word fbit / 64, bit fbit % 64 */
	uint64_t r0, nr;           /* reads [r0, r0 + nr) of the batch's read space */
	const uint64_t *fo;        /* frame offsets of the batch's reads (n * mates + 1) */
	uint64_t fo0;              /* fo[r0] */
	uint64_t T;                /* frames of the sub-batch: fo[r0 + nr] - fo0 */
	uint32_t nblk;             /* window blocks: ceil(T / kBkWinFrames) */
	uint32_t *vbits;           /* bit t: frame t of the sub-batch holds only ACGT */
	uint32_t *hbits;           /* bit t: frame t is still a hit (all levels so far) */
	uint8_t *state;            /* per read of the batch: 0 open, 1 decided */
	uint32_t ph_lo, ph_hi;     /* this phase: frames [bound(F, ph_lo), bound(F, ph_hi)) */
	uint32_t ph_min;           /* bound(F, q) >= min(F, ph_min) for q > 0 */
	uint32_t level, nlevels;   /* hash functions of this round: [level, level + nlevels)
	                              (0 = the canonical hash); a frame requests them all */
	uint32_t nbkt, bshift;     /* bucket of bit p: p >> bshift */
	unsigned long long *cnt;   /* this round's requests per (bucket, window): [nbkt][nblk],
	                              one more entry (0) at the end for the scan's total */
	unsigned long long *seg;   /* their exclusive scan, total at [nbkt * nblk] */
	const unsigned long long *pcnt; /* the previous round's (NULL in a phase's first round) */
	const unsigned long long *pseg;
	uint32_t *req_off;         /* request pool: bit offset inside the bucket */
	uint16_t *req_fid;         /*   frame id inside the window block */
	uint32_t *res;             /* result bit per request */
	unsigned long long *issued;/* optional: requests resolved (bit tests issued) */
};

/* fo[i + 1] = frames of read i (n * mates reads); the caller scans it. */
cudaError_t launch_bk_frame_counts(const ClassifyArgs &a, unsigned k, uint64_t *fo_plus1,
		int num_sms, cudaStream_t s);
/* out[j] = fo[min(j * stride, total)], j < n. */
cudaError_t launch_bk_samples(const uint64_t *fo, uint64_t total, uint64_t stride, uint64_t *out,
		uint64_t n, int num_sms, cudaStream_t s);
/* A round's counting sweep (applying the previous round's results first). */
cudaError_t launch_bk_count(const BucketArgs &b, cudaStream_t s);
/* A round's writing sweep: requests in bucket-major order. */
cudaError_t launch_bk_write(const BucketArgs &b, cudaStream_t s);
/* A round's bit tests, out of the bucket held in L2. */
cudaError_t launch_bk_resolve(const BucketArgs &b, int num_sms, cudaStream_t s);
/* The last round's results into hbits (b.pcnt / b.pseg = that round's). */
cudaError_t launch_bk_apply(const BucketArgs &b, cudaStream_t s);
/* SeqEval over [0, bound(F, ph_hi)) of every open read; accepted reads set
 * their hit bit; reads decided or fully walked are closed. */
cudaError_t launch_bk_walk(const BucketArgs &b, int num_sms, cudaStream_t s);

/* Shared memory of the counting / writing kernels for nbkt buckets. */
size_t bk_sweep_smem(uint32_t nbkt);

} // namespace bbt

#endif
