/*
 * classify.cu -- the read-classification kernels.
 *
 * One warp classifies one read at a time against every filter, replacing the
 * per-read body of BioBloomClassifier::filter (BioBloomClassifier.cpp:59-89):
 * evaluateReadStd (BioBloomClassifier.cpp:1182-1189) calls SeqEval::evalRead
 * (Common/SeqEval.h:493-524) once per filter, which walks the read's k-mers
 * with ntHashIterator and probes the filter (BloomFilter::contains).
 *
 * Per read the warp
 *   1. stages a window of up to 32*SEG frames: the bases go to shared memory
 *      and each lane hashes SEG consecutive frames (one Horner pass over k
 *      bases, then rolling), writing the canonical hash and a validity flag
 *      per frame to shared memory; windows are cached across filters with the
 *      same k;
 *   2. for each filter, walks the window 32 frames at a time: each lane probes
 *      one frame (h bit tests, stopping at the first clear bit, exactly as
 *      BloomFilter::contains), the warp ballots the hit bits and runs the
 *      SeqEval state machine over the chunk (seqeval_chunk.cuh); the filter is
 *      done when the state machine accepts or rejects.
 * Frames inside a skip window are not probed; frames after an accept/reject
 * inside the last chunk are probed speculatively (they change the bytes read,
 * never the result).
 *
 * Launch shapes: PLAIN gives each warp one read (one launch per batch);
 * PERSISTENT keeps one resident grid whose warps take reads from a global
 * counter until the batch is done, which balances reads of very different
 * lengths.  The filter-major order for several L2-sized filters is in
 * twopass.cu.
 */
#include "classify.cuh"
#include "seqeval_chunk.cuh"
#include "window.cuh"

#include "bbt.h"

namespace bbt {

namespace {

/* Valid-frame bits of frames [c, c + n) of the window (n <= 32). */
template <int SEG>
__device__ __forceinline__ uint32_t step_bits(const Window<SEG> &win, int c, int n)
{
	const int vi = c >> 5, vs = c & 31;
	uint32_t V = win.vmask[vi] >> vs;
	if (vs && vi + 1 < SEG)
		V |= win.vmask[vi + 1] << (32 - vs);
	if (n < 32)
		V &= (1u << n) - 1u;
	return V;
}

/* Build setting: a read whose frames mostly hit reads all h bits of a frame
 * at once (1) instead of the first, then the others together (0). */
#ifndef BBT_HIT_READS_ALL
#define BBT_HIT_READS_ALL 0
#endif

/* Evaluate read r against filters [f0, f1).  Returns the hit bits of those
 * filters that fall in word f0 / 64 (bit f % 64); read-major launches call it
 * with the whole filter range and write every word themselves.  WIDE: every
 * lane probes two frames per step (steps of up to 64 frames), twice the word
 * reads in flight per warp. */
template <int SEG, bool COUNT, int MODE, bool WIDE>
__device__ void classify_read(const ClassifyArgs &a, uint64_t r, uint32_t f0, uint32_t f1,
		const Window<SEG> &win, int lane, uint64_t &myword, unsigned long long &probe_acc,
		unsigned long long &frame_acc, unsigned long long &alg_acc)
{
	constexpr int W = Window<SEG>::W;
	const uint32_t mate = r >= a.n ? 1u : 0u;
	const uint64_t i = r - (mate ? a.n : 0);
	const uint64_t *off = a.off[mate];
	const uint64_t start = off[i] - a.off_base[mate];
	const uint64_t len = off[i + 1] - off[i];
	const Bases s = read_bases(a, mate, start);
	unsigned cached_k = 0;
	int64_t cached_w0 = -1;
	unsigned reads = 0;
	for (uint32_t f = f0; f < f1; ++f) {
		const FilterDev F = a.filters[f];
		const unsigned k = F.k;
		if (len < k)
			continue;
		const uint64_t frames = len - k + 1;
		SimpleState st;
		LengthState ls;
		SeqState qs;
		constexpr bool length_mode = MODE == BBT_SCORE_LENGTH;
		/* HARMONIC walks frame by frame (seq_chunk); BINOMIAL is SIMPLE's
		 * machine with integer hits (binomial_simple_init) */
		constexpr bool seq_mode = MODE == BBT_SCORE_HARMONIC;
		if (MODE == BBT_SCORE_HARMONIC)
			harmonic_init(qs, a.score, a.one_minus, frames);
		else if (MODE == BBT_SCORE_BINOMIAL)
			binomial_simple_init(st, a.bthres[f * a.bthres_rows + frames], frames);
		else if (length_mode)
			length_init(ls, a.min_len, len, (int)k);
		else
			simple_init(st, a.score, a.one_minus, frames);
		int decided = EVAL_OPEN;
		/* decision-sized steps read a frame's bits after the first together
		 * while at least half of the read's frames probed in its last step
		 * were hits (a read from the filter's reference: every bit gets read
		 * anyway, in fewer round trips), one after another otherwise (a read
		 * that is not in the filter: most frames stop at the first or second
		 * clear bit, so fewer filter reads); warp-uniform, from the step's
		 * ballots */
		bool hitting = true;
		for (uint64_t w0 = 0; w0 < frames && !decided; w0 += W) {
			const int wn = (int)min((uint64_t)W, frames - w0);
			if (cached_k != k || cached_w0 != (int64_t)w0) {
				if (cached_k != k)
					set_tables<SEG>(win, k, lane);
				hash_window<SEG>(s, w0, wn, k, win, lane);
				cached_k = k;
				cached_w0 = (int64_t)w0;
				if (COUNT)
					frame_acc += (lane == 0) ? (unsigned long long)wn : 0ull;
			}
			for (int c = 0; c < wn;) {
				/* frames [c, c + nfc) of the window this step: lane l probes
				 * frame c + l, and with WIDE also frame c + 32 + l; the
				 * machine then takes them 32 at a time, in frame order */
				constexpr int cap = WIDE ? 64 : 32;
				const int nfc = min((length_mode || seq_mode || !a.tight_steps) ? cap
						: simple_step_frames(st, cap), wn - c);
				const int n0 = min(nfc, 32);
				/* frames below this were in a skip window when the step began */
				const int32_t pf = length_mode ? INT32_MIN
						: seq_mode ? (int32_t)seq_probe_from(qs) : st.skip_until;
				auto probe_at = [&](uint32_t V, int q) {
					const int32_t p = (int32_t)w0 + q;
					return ((V >> lane) & 1u) && p >= pf &&
							!dust_low(a.dust[mate], start + (uint64_t)p);
				};
				auto advance = [&](uint32_t V, uint32_t H, int b, int n, uint32_t *alg) {
					return length_mode ? length_chunk(ls, V, H, (int64_t)w0 + b, n, alg)
							: seq_mode ? seq_chunk(qs, V, H, (int64_t)w0 + b, n, (int)k,
									a.streak_thr, alg)
							: simple_chunk(st, V, H, (int32_t)w0 + b, n, (int)k,
									(int)a.streak_thr, alg);
				};
				const uint32_t V0 = step_bits<SEG>(win, c, n0);
				const bool probe0 = probe_at(V0, c + lane);
				uint32_t alg = 0;
				if (WIDE) {
					const int n1 = nfc - n0;
					const uint32_t V1 = n1 > 0 ? step_bits<SEG>(win, c + 32, n1) : 0u;
					const bool probe1 = probe_at(V1, c + 32 + lane);
					bool hit0, hit1;
					unsigned ra = 0, rb = 0;
					contains2(F, probe0 ? win.h0[c + lane] : 0ull, probe0,
							probe1 ? win.h0[c + 32 + lane] : 0ull, probe1, hit0, hit1, ra, rb);
					reads += ra + rb;
					const uint32_t H0 = __ballot_sync(kFull, hit0);
					const uint32_t H1 = __ballot_sync(kFull, hit1);
					decided = advance(V0, H0, c, n0, COUNT ? &alg : nullptr);
					if (COUNT && ((alg >> lane) & 1u))
						alg_acc += ra;
					if (!decided && n1 > 0) {
						alg = 0;
						decided = advance(V1, H1, c + 32, n1, COUNT ? &alg : nullptr);
						if (COUNT && ((alg >> lane) & 1u))
							alg_acc += rb;
					}
				} else {
					const unsigned r0 = reads;
					unsigned sq = 0;
					const bool split = a.tight_steps && hitting;
					const bool hit = probe0 && (split
							? (BBT_HIT_READS_ALL
								? contains_all(F, win.h0[c + lane], reads, sq)
								: contains_split(F, win.h0[c + lane], reads, sq))
							: contains(F, win.h0[c + lane], reads));
					const uint32_t H = __ballot_sync(kFull, hit);
					if (a.tight_steps) {
						const uint32_t P = __ballot_sync(kFull, probe0);
						if (P)
							hitting = 2 * __popc(H) >= __popc(P);
					}
					decided = advance(V0, H, c, n0, COUNT ? &alg : nullptr);
					if (COUNT && ((alg >> lane) & 1u))
						alg_acc += split ? sq : reads - r0;
				}
				if (decided)
					break;
				c += nfc;
			}
		}
		if (decided == EVAL_ACCEPT && lane == (int)(f >> 6))
			myword |= 1ull << (f & 63);
	}
	if (COUNT)
		probe_acc += reads;
}

enum { ORDER_PLAIN = 0, ORDER_READS = 1 };

/*
 * ORDER_PLAIN:   one read per warp, all filters, grid covers the batch.
 * ORDER_READS:   persistent; warps take reads from a counter, all filters each.
 * (The filter-major order is the two-pass path in twopass.cu.)
 */
/* Blocks of 256 threads the register budget leaves room for (a build
 * setting: 4 gives each thread up to 64 registers, 32 warps per SM). */
#ifndef BBT_CLASSIFY_MIN_BLOCKS
#define BBT_CLASSIFY_MIN_BLOCKS 4
#endif
template <int SEG, int ORDER, bool COUNT, int MODE, bool WIDE>
__global__ void __launch_bounds__(256, BBT_CLASSIFY_MIN_BLOCKS) classify_kernel(ClassifyArgs a)
{
	extern __shared__ __align__(16) unsigned char smem[];
	const int lane = threadIdx.x & 31;
	const int warp = threadIdx.x >> 5;
	const Window<SEG> win = window_at<SEG>(smem + warp * window_stride<SEG>(a.kmax));
	const uint64_t total = a.n * a.mates;
	unsigned long long probe_acc = 0, frame_acc = 0, alg_acc = 0;
	if (ORDER == ORDER_READS) {
		for (;;) {
			unsigned long long r = 0;
			if (lane == 0)
				r = atomicAdd(a.work, 1ull);
			r = __shfl_sync(kFull, r, 0);
			if (r >= total)
				break;
			if (a.order)
				r = a.order[r];
			uint64_t myword = 0;
			classify_read<SEG, COUNT, MODE, WIDE>(a, r, 0, a.nf, win, lane, myword, probe_acc,
					frame_acc, alg_acc);
			const uint32_t mate = r >= a.n ? 1u : 0u;
			if (lane < (int)a.words)
				a.hits[mate][(r - (mate ? a.n : 0)) * a.words + lane] = myword;
		}
	} else {
		const uint64_t r = (uint64_t)blockIdx.x * (blockDim.x >> 5) + warp;
		if (r < total) {
			uint64_t myword = 0;
			classify_read<SEG, COUNT, MODE, WIDE>(a, r, 0, a.nf, win, lane, myword, probe_acc,
					frame_acc, alg_acc);
			const uint32_t mate = r >= a.n ? 1u : 0u;
			if (lane < (int)a.words)
				a.hits[mate][(r - (mate ? a.n : 0)) * a.words + lane] = myword;
		}
	}
	if (COUNT) {
		for (int o = 16; o; o >>= 1) {
			probe_acc += __shfl_xor_sync(kFull, probe_acc, o);
			frame_acc += __shfl_xor_sync(kFull, frame_acc, o);
			alg_acc += __shfl_xor_sync(kFull, alg_acc, o);
		}
		if (lane == 0) {
			if (a.probes)
				atomicAdd(a.probes, probe_acc);
			if (a.frames)
				atomicAdd(a.frames, frame_acc);
			if (a.alg_probes)
				atomicAdd(a.alg_probes, alg_acc);
		}
	}
}

/* ResultsManager::updateSummaryData (ResultsManager.hpp:66-189) over a batch:
 * the category of each read (pair) and block-aggregated counter updates.
 * ordered: evaluateReadOrdered / evaluateReadOrderedPair
 * (BioBloomClassifier.cpp:1145-1180) stop at the first filter, in load order,
 * that the read passes (pairs: that both mates pass, or either with -i) and
 * report that filter alone for both mates: the lowest set bit of the same
 * combined words, written back as the hit words. */
__global__ void summarize_kernel(uint64_t *__restrict__ h1, uint64_t *__restrict__ h2,
		uint64_t n, uint32_t nf, uint32_t words, int inclusive, int ordered, uint32_t *category,
		unsigned long long *counts)
{
	extern __shared__ unsigned long long sc[];
	const uint32_t ncount = 2 * (nf + 2) + 2;
	for (uint32_t j = threadIdx.x; j < ncount; j += blockDim.x)
		sc[j] = 0;
	__syncthreads();
	for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
			i += (uint64_t)gridDim.x * blockDim.x) {
		uint32_t idx = nf;
		for (uint32_t w = 0; w < words; ++w) {
			uint64_t x = h1[i * words + w];
			if (h2)
				x = inclusive ? (x | h2[i * words + w]) : (x & h2[i * words + w]);
			if (ordered) {
				x = idx == nf ? (x & (0ull - x)) : 0ull; /* the first filter only */
				h1[i * words + w] = x;
				if (h2)
					h2[i * words + w] = x;
			}
			while (x) {
				uint32_t f = w * 64 + (uint32_t)(__ffsll((long long)x) - 1);
				x &= x - 1;
				atomicAdd(&sc[f], 1ull);
				idx = idx == nf ? f : nf + 1;
			}
		}
		if (idx == nf)
			atomicAdd(&sc[2 * (nf + 2) + 1], 1ull);
		else if (idx == nf + 1)
			atomicAdd(&sc[2 * (nf + 2)], 1ull);
		else
			atomicAdd(&sc[(nf + 2) + idx], 1ull);
		if (category)
			category[i] = idx;
	}
	__syncthreads();
	for (uint32_t j = threadIdx.x; j < ncount; j += blockDim.x)
		if (sc[j])
			atomicAdd(&counts[j], sc[j]);
}

/* Warp-aggregated split of the reads into long (front of order, in counter 0)
 * and short (back of order, in counter 1). */
__global__ void long_first_kernel(ClassifyArgs a, uint64_t long_bases, uint64_t *order,
		unsigned long long *counters)
{
	const uint64_t total = a.n * a.mates;
	const int lane = threadIdx.x & 31;
	const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
	for (uint64_t base = (uint64_t)blockIdx.x * blockDim.x; base < total; base += stride) {
		const uint64_t r = base + threadIdx.x;
		bool valid = r < total, is_long = false;
		if (valid) {
			const uint32_t mate = r >= a.n ? 1u : 0u;
			const uint64_t i = r - (mate ? a.n : 0);
			is_long = a.off[mate][i + 1] - a.off[mate][i] >= long_bases;
		}
		const unsigned lm = __ballot_sync(kFull, valid && is_long);
		const unsigned sm = __ballot_sync(kFull, valid && !is_long);
		unsigned long long b0 = 0, b1 = 0;
		if (lane == 0) {
			if (lm)
				b0 = atomicAdd(counters, (unsigned long long)__popc(lm));
			if (sm)
				b1 = atomicAdd(counters + 1, (unsigned long long)__popc(sm));
		}
		b0 = __shfl_sync(kFull, b0, 0);
		b1 = __shfl_sync(kFull, b1, 0);
		const unsigned below = (1u << lane) - 1u;
		if (valid && is_long)
			order[b0 + __popc(lm & below)] = r;
		else if (valid)
			order[total - 1 - (b1 + __popc(sm & below))] = r;
	}
}

template <int SEG, int ORDER, bool C, bool WIDE>
cudaError_t launch_one(const ClassifyArgs &a, const LaunchConfig &lc, cudaStream_t s)
{
	const int threads = lc.warps_per_block * 32;
	const size_t smem = classify_smem_bytes(lc, a.kmax);
	auto kern = a.scoring == BBT_SCORE_LENGTH ? classify_kernel<SEG, ORDER, C, BBT_SCORE_LENGTH, WIDE>
	          : a.scoring == BBT_SCORE_HARMONIC ? classify_kernel<SEG, ORDER, C, BBT_SCORE_HARMONIC, WIDE>
	          : a.scoring == BBT_SCORE_BINOMIAL ? classify_kernel<SEG, ORDER, C, BBT_SCORE_BINOMIAL, WIDE>
	                                            : classify_kernel<SEG, ORDER, C, BBT_SCORE_SIMPLE, WIDE>;
	cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
			(int)smem);
	if (e != cudaSuccess)
		return e;
	uint64_t total = a.n * a.mates;
	uint64_t warps_needed = total;
	unsigned blocks;
	if (ORDER != ORDER_PLAIN) {
		int per_sm = 0;
		e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, threads, smem);
		if (e != cudaSuccess)
			return e;
		if (per_sm < 1)
			per_sm = 1;
		uint64_t need = (warps_needed + lc.warps_per_block - 1) / lc.warps_per_block;
		uint64_t full = (uint64_t)per_sm * lc.num_sms;
		blocks = (unsigned)(need < full ? need : full);
	} else {
		blocks = (unsigned)((total + lc.warps_per_block - 1) / lc.warps_per_block);
	}
	if (blocks == 0)
		return cudaSuccess;
	kern<<<blocks, threads, smem, s>>>(a);
	return cudaGetLastError();
}

template <int SEG>
cudaError_t launch_seg(const ClassifyArgs &a, const LaunchConfig &lc, cudaStream_t s)
{
	const bool C = lc.count != 0;
	const bool W = lc.steps >= BBT_STEPS_WIDE;
	switch (lc.path) {
	case BBT_PATH_PLAIN:
		return C ? launch_one<SEG, ORDER_PLAIN, true, false>(a, lc, s)
		         : launch_one<SEG, ORDER_PLAIN, false, false>(a, lc, s);
	default:
		if (W)
			return C ? launch_one<SEG, ORDER_READS, true, true>(a, lc, s)
			         : launch_one<SEG, ORDER_READS, false, true>(a, lc, s);
		return C ? launch_one<SEG, ORDER_READS, true, false>(a, lc, s)
		         : launch_one<SEG, ORDER_READS, false, false>(a, lc, s);
	}
}

} // namespace

size_t classify_smem_bytes(const LaunchConfig &lc, uint32_t kmax)
{
	const size_t per_warp = lc.seg == 8 ? window_stride<8>(kmax) : window_stride<4>(kmax);
	return per_warp * (size_t)lc.warps_per_block;
}

cudaError_t launch_classify(const ClassifyArgs &a0, const LaunchConfig &lc, cudaStream_t s)
{
	/* The persistent kernel on a filter in HBM is bound by DRAM traffic and
	 * the latency of its dependent word reads: it takes steps sized to the
	 * read's decision, which probe fewer frames, with two frames per lane
	 * (BBT_STEPS_WIDE) for twice the reads in flight.  The plain kernel, and
	 * the persistent one on a filter held in L2 (BBT_STEPS_FULL, chosen by the
	 * autotuner), are bound by the chain of steps and the instructions per
	 * step: they keep full steps, fewer of them. */
	ClassifyArgs a = a0;
	a.tight_steps = lc.path != BBT_PATH_PLAIN &&
			(lc.steps == BBT_STEPS_DECISION || lc.steps == BBT_STEPS_WIDE);
	return lc.seg == 8 ? launch_seg<8>(a, lc, s) : launch_seg<4>(a, lc, s);
}

cudaError_t launch_long_first(const ClassifyArgs &a, uint64_t long_bases, uint64_t *order,
		unsigned long long *counters, int num_sms, cudaStream_t s)
{
	const uint64_t total = a.n * a.mates;
	if (total == 0)
		return cudaSuccess;
	const uint64_t need = (total + 255) / 256;
	const uint64_t cap = (uint64_t)num_sms * 8;
	long_first_kernel<<<(unsigned)(need < cap ? need : cap), 256, 0, s>>>(a, long_bases, order,
			counters);
	return cudaGetLastError();
}

/* Read lengths of a batch: out[0] = the largest, out[1 + L / 32] bit L % 32
 * for each length L below 65536. */
__global__ void length_set_kernel(const uint64_t *off0, const uint64_t *off1, uint64_t n,
		uint32_t mates, unsigned int *out)
{
	for (uint64_t r = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; r < n * mates;
			r += (uint64_t)gridDim.x * blockDim.x) {
		const uint64_t *off = r >= n ? off1 : off0;
		const uint64_t i = r >= n ? r - n : r;
		const uint64_t l = off[i + 1] - off[i];
		const unsigned int L = l > 0xFFFFFFFFull ? 0xFFFFFFFFu : (unsigned int)l;
		atomicMax(out, L);
		if (L < 65536u)
			atomicOr(out + 1 + (L >> 5), 1u << (L & 31));
	}
}

cudaError_t launch_length_set(const uint64_t *off0, const uint64_t *off1, uint64_t n,
		uint32_t mates, unsigned int *out, int num_sms, cudaStream_t s)
{
	if (n == 0)
		return cudaSuccess;
	const uint64_t need = (n * mates + 255) / 256;
	const uint64_t cap = (uint64_t)num_sms * 4;
	length_set_kernel<<<(unsigned)(need < cap ? need : cap), 256, 0, s>>>(off0, off1, n, mates,
			out);
	return cudaGetLastError();
}

cudaError_t launch_summarize(uint64_t *h1, uint64_t *h2, uint64_t n, uint32_t nf,
		uint32_t words, int inclusive, int ordered, uint32_t *category,
		unsigned long long *counts, int num_sms, cudaStream_t s)
{
	if (n == 0)
		return cudaSuccess;
	const int threads = 256;
	uint64_t need = (n + threads - 1) / threads;
	uint64_t cap = (uint64_t)num_sms * 4;
	unsigned blocks = (unsigned)(need < cap ? need : cap);
	size_t smem = sizeof(unsigned long long) * (2 * (nf + 2) + 2);
	summarize_kernel<<<blocks, threads, smem, s>>>(h1, h2, n, nf, words, inclusive, ordered,
			category, counts);
	return cudaGetLastError();
}

} // namespace bbt
