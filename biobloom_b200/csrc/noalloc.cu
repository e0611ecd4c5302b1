/*
 * noalloc.cu -- bbt_classify_noalloc: classification that allocates nothing.
 *
 * Who needs it: callers whose device memory is owned by someone else -- a
 * framework's caching allocator or a pool reserved up front with a fixed
 * budget -- and callers on paths where cudaMalloc / cudaFree (which can
 * synchronize the whole device) are not acceptable.  They pass device buffers
 * for the filters, the reads and the hit words; the only other device memory
 * the call uses is the small file-scope array below, which exists once per GPU
 * from the moment the library is loaded until the process exits.
 *
 * The array holds the filter descriptor table (at most
 * BBT_NOALLOC_MAX_FILTERS entries) and the work counter of the persistent
 * classify kernel.  Every call on a GPU shares it and it keeps the previous
 * call's contents, so each call rewrites the table and clears the counter
 * before its kernel runs.  Two calls whose work overlaps on the same GPU (for
 * example on two streams) race on this array and may return wrong hits; issue
 * such calls one after another.
 *
 * In host code the array's name is only a host-side stand-in, not a device
 * address.  Each call obtains the device address with cudaGetSymbolAddress,
 * with the call's GPU current, in noalloc_scratch() below.  The address is not
 * cached: after a cudaDeviceReset in the caller's process the GPU has a new
 * context, in which the array may sit at another address.  The first call on a
 * GPU also loads the library's device code there.
 */
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <string>

#include "bbt.h"
#include "classify.cuh"
#include "ctx.hpp"

namespace bbt {
namespace {

struct NoAllocLayout {
	FilterDev filters[BBT_NOALLOC_MAX_FILTERS];
	unsigned long long work;
};

constexpr size_t kScratchBytes = 4096;
static_assert(sizeof(NoAllocLayout) <= kScratchBytes, "no-alloc scratch too small");

static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

/* Device address of the scratch array on the current device. */
int noalloc_scratch(NoAllocLayout **out)
{
	void *p = nullptr;
	cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
	if (e != cudaSuccess || !p)
		return cuda_fail(nullptr, e == cudaSuccess ? cudaErrorInvalidSymbol : e,
				"cudaGetSymbolAddress(no-alloc scratch)");
	*out = reinterpret_cast<NoAllocLayout *>(p);
	return BBT_OK;
}

} // namespace
} // namespace bbt

using namespace bbt;

extern "C" int bbt_classify_noalloc(const bbt_filter_view *filters, int n_filters,
		const bbt_params *params, const bbt_batch *batch, uint64_t *hits, uint64_t *hits2,
		void *stream)
{
	if (!filters || !params || !batch || !hits)
		return fail(nullptr, BBT_ERR_ARG, "bbt_classify_noalloc: null argument");
	if (n_filters < 1 || n_filters > BBT_NOALLOC_MAX_FILTERS)
		return fail(nullptr, BBT_ERR_ARG,
				"bbt_classify_noalloc: n_filters must be between 1 and " +
				std::to_string(BBT_NOALLOC_MAX_FILTERS) + " (got " +
				std::to_string(n_filters) + ")");
	if (batch->location != BBT_DEVICE)
		return fail(nullptr, BBT_ERR_ARG, "bbt_classify_noalloc: reads must be in device memory");
	const bool paired = batch->seq2 != nullptr;
	if (!batch->seq || !batch->offsets || (paired && (!batch->offsets2 || !hits2)))
		return fail(nullptr, BBT_ERR_ARG, "bbt_classify_noalloc: missing reads, offsets or hits");
	if (batch->encoding != BBT_BASES_ASCII && batch->encoding != BBT_BASES_2BIT)
		return fail(nullptr, BBT_ERR_ARG, "bbt_classify_noalloc: unknown base encoding");
	double score = params->score;
	int scoring = params->scoring;
	if (!(score < 4294967296.0))
		return fail(nullptr, BBT_ERR_ARG, "bbt_classify_noalloc: score must be below 2^32");
	if ((scoring == BBT_SCORE_SIMPLE || scoring == BBT_SCORE_HARMONIC) && score > 1 &&
			(unsigned)score > 1) {
		/* as bbt_open: an integer score > 1 is a minimum match length */
		score = (double)(unsigned)score;
		scoring = BBT_SCORE_LENGTH;
	}
	if (scoring == BBT_SCORE_SIMPLE && (score < 0 || score > 1))
		return fail(nullptr, BBT_ERR_ARG, "bbt_classify_noalloc: score must be in [0, 1] or an integer > 1");
	if (scoring != BBT_SCORE_SIMPLE && scoring != BBT_SCORE_LENGTH)
		return fail(nullptr, BBT_ERR_UNSUPPORTED,
				"bbt_classify_noalloc: simple or length scoring only (harmonic and binomial "
				"thresholds live in context memory)");
	FilterDev table[BBT_NOALLOC_MAX_FILTERS];
	uint32_t kmax = 0;
	for (int i = 0; i < n_filters; ++i) {
		const bbt_filter_view &v = filters[i];
		if (!v.words || v.m == 0 || v.m % 64 || v.h == 0 || v.h > 64 || v.k == 0 || v.k > 255)
			return fail(nullptr, BBT_ERR_ARG, "bbt_classify_noalloc: filter " +
					std::to_string(i) + " has a null array or out-of-range m, h or k");
		table[i] = make_filter_dev(v.words, v.m, v.h, v.k);
		kmax = v.k > kmax ? v.k : kmax;
	}
	if (params->device < 0)
		return fail(nullptr, BBT_ERR_ARG, "bbt_classify_noalloc: negative device ordinal");
	if (batch->n_reads == 0)
		return BBT_OK;
	int prev = 0;
	cudaError_t e = cudaGetDevice(&prev);
	if (e != cudaSuccess)
		return cuda_fail(nullptr, e, "cudaGetDevice");
	const int dev = params->device;
	if (dev != prev && (e = cudaSetDevice(dev)) != cudaSuccess)
		return cuda_fail(nullptr, e, "cudaSetDevice");
	int rc = BBT_OK;
	NoAllocLayout *scratch = nullptr;
	cudaStream_t s = (cudaStream_t)stream;
	int sms = 0;
	if ((rc = noalloc_scratch(&scratch)) != BBT_OK)
		goto out;
	if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) {
		rc = cuda_fail(nullptr, e, "cudaDeviceGetAttribute");
		goto out;
	}
	/* the table comes from this call's stack; a copy from pageable memory is
	 * staged before cudaMemcpyAsync returns */
	if ((e = cudaMemcpyAsync(scratch->filters, table, sizeof(FilterDev) * n_filters,
			cudaMemcpyHostToDevice, s)) != cudaSuccess ||
			(e = cudaMemsetAsync(&scratch->work, 0, sizeof(unsigned long long), s)) != cudaSuccess) {
		rc = cuda_fail(nullptr, e, "no-alloc scratch set-up");
		goto out;
	}
	{
		ClassifyArgs a;
		memset(&a, 0, sizeof a);
		a.seq[0] = (const uint8_t *)batch->seq;
		a.off[0] = batch->offsets;
		a.seq[1] = (const uint8_t *)(paired ? batch->seq2 : batch->seq);
		a.off[1] = paired ? batch->offsets2 : batch->offsets;
		a.packed = batch->encoding == BBT_BASES_2BIT;
		a.valid[0] = a.packed ? batch->valid : nullptr;
		a.valid[1] = a.packed ? (paired ? batch->valid2 : batch->valid) : nullptr;
		a.n = batch->n_reads;
		a.mates = paired ? 2 : 1;
		a.filters = scratch->filters;
		a.nf = (uint32_t)n_filters;
		a.words = (a.nf + 63) / 64;
		a.score = score;
		a.one_minus = 1.0 - score;
		a.streak_thr = params->streak_threshold;
		a.scoring = scoring;
		a.min_len = (unsigned)std::round(score);
		a.kmax = kmax;
		a.hits[0] = hits;
		a.hits[1] = paired ? hits2 : nullptr;
		a.work = &scratch->work;
		LaunchConfig lc;
		lc.path = BBT_PATH_PERSISTENT;
		lc.warps_per_block = 8;
		lc.seg = params->frames_per_lane == 8 ? 8 : 4;
		lc.num_sms = sms;
		lc.count = 0;
		lc.steps = BBT_STEPS_DECISION;
		if ((e = launch_classify(a, lc, s)) != cudaSuccess)
			rc = cuda_fail(nullptr, e, "classify kernel launch");
	}
out:
	if (dev != prev)
		cudaSetDevice(prev);
	return rc;
}
