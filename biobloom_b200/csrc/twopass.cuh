/*
 * twopass.cuh -- launch interface of the two-pass filter-major path
 * (twopass.cu), used by api.cu.
 */
#ifndef BBT_TWOPASS_CUH
#define BBT_TWOPASS_CUH

#include <cuda_runtime.h>
#include <stdint.h>

#include "classify.cuh"

namespace bbt {

/* One sub-batch: reads t in [t0, t1) of the batch (t indexes the batch's
 * reads, mate arrays concatenated; read r = r_first + t in ClassifyArgs
 * numbering).  local / sums come from two_pass_scan; s0 is the first frame
 * slot of read t0, so slot - s0 indexes h0 (and / 32 indexes vmask). */
struct TwoPassArgs {
	uint64_t t0, t1;
	uint64_t r_first;
	const uint64_t *local;
	const unsigned long long *sums;
	uint64_t s0;
	unsigned k;
	uint64_t *h0;
	uint32_t *vmask;
	unsigned long long *work;
};

/* Padded frame offsets of every read of the batch (common k):
 * local[t] (per-1024-read block prefix) and sums[b] (exclusive block prefix,
 * sums[nb] = total). */
cudaError_t two_pass_scan(const ClassifyArgs &a, unsigned k, uint64_t *local,
		unsigned long long *sums, cudaStream_t s);
uint64_t two_pass_block_reads();
/* Hash pass, then the filter pass (classify: hits must be zeroed once per
 * batch beforehand) and / or the score pass (sa: every item's evalScore into
 * sa->scores), for one sub-batch. */
cudaError_t two_pass_sub_batch(const ClassifyArgs &a, const TwoPassArgs &p, const LaunchConfig &lc,
		cudaStream_t s, const ScoreArgs *sa = nullptr, bool classify = true);

} // namespace bbt

#endif
