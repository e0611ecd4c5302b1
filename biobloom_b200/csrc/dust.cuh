/*
 * dust.cuh -- launch interface of the SDUST masking kernels (dust.cu).
 */
#ifndef BBT_DUST_CUH
#define BBT_DUST_CUH

#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

namespace bbt {

/* Largest window (-W) the kernels accept; the window ring lives in registers
 * and local memory of each thread. */
constexpr int kDustMaxWindow = 1024;

/* One batch: reads r in [0, n * mates) as in ClassifyArgs.  mask[m]: zeroed
 * bit array over mate array m's bases (bit g = base seq[m][g]).  redo: n *
 * mates entries, redo_count / failed: zeroed counters.  scratch: pass-2
 * perfect lists, scratch_per_thread entries (dust_perfect_bytes() each) per
 * pass-2 thread. */
struct DustArgs {
	const uint8_t *seq[2];
	const uint64_t *off[2];
	uint64_t off_base[2];
	uint64_t n;
	uint32_t mates;
	int T, W;
	uint32_t *mask[2];
	uint64_t *redo;
	unsigned long long *redo_count;
	unsigned long long *failed;
	void *scratch;
	uint64_t scratch_per_thread;
};

size_t dust_perfect_bytes();
/* Pass 1: every read; reads whose perfect list outgrows the thread's own
 * array are appended to redo. */
cudaError_t launch_dust_pass1(const DustArgs &a, int num_sms, cudaStream_t s);
/* Pass 2: the reads pass 1 queued (their count is read on the device), on
 * `threads` threads (a multiple of 32) with scratch_per_thread entries
 * each; a read that outgrows even that counts in failed. */
cudaError_t launch_dust_pass2(const DustArgs &a, uint32_t threads, cudaStream_t s);

} // namespace bbt

#endif
