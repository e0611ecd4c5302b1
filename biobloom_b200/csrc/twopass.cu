/*
 * twopass.cu -- filter-major classification in two passes, for several
 * filters that each fit in L2.
 *
 * Evaluating a read against F filters (BioBloomClassifier::evaluateReadStd,
 * BioBloomClassifier.cpp:1182-1189) gives F independent SeqEval runs over the
 * same k-mers.  The single-pass kernels walk reads and probe all F filters in
 * turn, so all filters are live at once and every probe goes to DRAM (an
 * isolated probe costs a 128-byte line fill on this GPU).  Here the work is
 * reordered without changing any result:
 *
 *   scan:        padded frame count of each read (multiple of 32) -> offsets
 *   hash pass:   each read is hashed once; the canonical hash of every frame
 *                and one validity word per 32 frames go to a global scratch
 *   filter pass: persistent warps take (filter, read) items in filter order,
 *                so the whole GPU probes one filter at a time and that filter
 *                stays resident in L2; each item replays SeqEval over the
 *                stored hashes and ORs its bit into the read's hit word.
 *
 * The scratch holds a sub-batch of reads; the host splits a batch at 1024-read
 * blocks so that each sub-batch's frames fit (one small device-to-host read of
 * the per-block frame totals per batch).
 */
#include <cuda_runtime.h>

#include <algorithm>
#include <vector>

#include "bbt.h"
#include "classify.cuh"
#include "ctx.hpp"
#include "score_value.cuh"
#include "seqeval_chunk.cuh"
#include "twopass.cuh"
#include "window.cuh"

namespace bbt {
namespace {

constexpr int kScanBlock = 1024;

__device__ __forceinline__ uint64_t read_len(const ClassifyArgs &a, uint64_t r)
{
	const uint32_t mate = r >= a.n ? 1u : 0u;
	const uint64_t i = r - (mate ? a.n : 0);
	return a.off[mate][i + 1] - a.off[mate][i];
}

__device__ __forceinline__ uint64_t padded_frames(uint64_t len, unsigned k)
{
	return len < k ? 0 : ((len - k + 1 + 31) & ~31ull);
}

/* Per-block exclusive scan of the padded frame counts of reads
 * [r0, r0 + cnt); block b's total goes to sums[b]. */
__global__ void __launch_bounds__(kScanBlock) scan_frames_kernel(ClassifyArgs a, uint64_t r0,
		uint64_t cnt, unsigned k, uint64_t *local, unsigned long long *sums)
{
	__shared__ unsigned long long warp_tot[kScanBlock / 32];
	const uint64_t t = (uint64_t)blockIdx.x * kScanBlock + threadIdx.x;
	const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
	unsigned long long v = t < cnt ? padded_frames(read_len(a, r0 + t), k) : 0;
	unsigned long long x = v;
	for (int o = 1; o < 32; o <<= 1) {
		unsigned long long y = __shfl_up_sync(kFull, x, o);
		if (lane >= o)
			x += y;
	}
	if (lane == 31)
		warp_tot[warp] = x;
	__syncthreads();
	if (warp == 0) {
		unsigned long long w = warp_tot[lane];
		for (int o = 1; o < 32; o <<= 1) {
			unsigned long long y = __shfl_up_sync(kFull, w, o);
			if (lane >= o)
				w += y;
		}
		warp_tot[lane] = w; /* inclusive */
	}
	__syncthreads();
	const unsigned long long before = warp == 0 ? 0 : warp_tot[warp - 1];
	if (t < cnt)
		local[t] = before + x - v;
	if (threadIdx.x == kScanBlock - 1)
		sums[blockIdx.x] = before + x;
}

/* Exclusive scan of the block totals in place; sums[nb] = grand total. */
__global__ void __launch_bounds__(kScanBlock) scan_sums_kernel(unsigned long long *sums,
		uint64_t nb)
{
	__shared__ unsigned long long warp_tot[kScanBlock / 32];
	__shared__ unsigned long long carry;
	const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
	if (threadIdx.x == 0)
		carry = 0;
	__syncthreads();
	for (uint64_t base = 0; base < nb; base += kScanBlock) {
		const uint64_t t = base + threadIdx.x;
		unsigned long long v = t < nb ? sums[t] : 0;
		unsigned long long x = v;
		for (int o = 1; o < 32; o <<= 1) {
			unsigned long long y = __shfl_up_sync(kFull, x, o);
			if (lane >= o)
				x += y;
		}
		if (lane == 31)
			warp_tot[warp] = x;
		__syncthreads();
		if (warp == 0) {
			unsigned long long w = warp_tot[lane];
			for (int o = 1; o < 32; o <<= 1) {
				unsigned long long y = __shfl_up_sync(kFull, w, o);
				if (lane >= o)
					w += y;
			}
			warp_tot[lane] = w;
		}
		__syncthreads();
		const unsigned long long before = warp == 0 ? 0 : warp_tot[warp - 1];
		if (t < nb)
			sums[t] = carry + before + x - v;
		__syncthreads();
		if (threadIdx.x == 0)
			carry += warp_tot[kScanBlock / 32 - 1];
		__syncthreads();
	}
	if (threadIdx.x == 0)
		sums[nb] = carry;
}

/* First frame slot of read t (batch-relative index), relative to the
 * sub-batch whose first slot is s0. */
__device__ __forceinline__ uint64_t frame_base(const TwoPassArgs &p, uint64_t t)
{
	return p.local[t] + p.sums[t / kScanBlock] - p.s0;
}

/* Hash pass: reads [t0, t1) of the batch; one warp per read. */
template <int SEG, bool COUNT>
__global__ void __launch_bounds__(256) hash_pass_kernel(ClassifyArgs a, TwoPassArgs p)
{
	extern __shared__ __align__(16) unsigned char smem[];
	const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
	const Window<SEG> win = window_at<SEG>(smem + warp * window_stride<SEG>(a.kmax));
	constexpr int W = Window<SEG>::W;
	set_tables<SEG>(win, p.k, lane);
	unsigned long long frames_acc = 0;
	for (;;) {
		unsigned long long t = 0;
		if (lane == 0)
			t = atomicAdd(p.work, 1ull);
		t = __shfl_sync(kFull, t, 0) + p.t0;
		if (t >= p.t1)
			break;
		const uint64_t r = p.r_first + t;
		const uint32_t mate = r >= a.n ? 1u : 0u;
		const uint64_t i = r - (mate ? a.n : 0);
		const uint64_t len = a.off[mate][i + 1] - a.off[mate][i];
		if (len < p.k)
			continue;
		const Bases s = read_bases(a, mate, a.off[mate][i] - a.off_base[mate]);
		const uint64_t frames = len - p.k + 1;
		const uint64_t base = frame_base(p, t);
		for (uint64_t w0 = 0; w0 < frames; w0 += W) {
			const int wn = (int)min((uint64_t)W, frames - w0);
			hash_window<SEG>(s, w0, wn, p.k, win, lane);
			for (int q = lane; q < wn; q += 32)
				p.h0[base + w0 + q] = win.h0[q];
			const int nw = (wn + 31) >> 5;
			if (lane < nw)
				p.vmask[(base + w0) / 32 + lane] = win.vmask[lane];
			__syncwarp();
			if (COUNT && lane == 0)
				frames_acc += wn;
		}
	}
	if (COUNT && lane == 0 && a.frames && frames_acc)
		atomicAdd(a.frames, frames_acc);
}

/* Per-item metadata of the filter pass: read length and first frame slot. */
struct ItemMeta {
	uint64_t len;
	uint64_t base;
	uint64_t i;
	uint64_t start;   /* the read's first base in its mate array (DUST mask index) */
	uint32_t mate;
};

__device__ __forceinline__ ItemMeta item_meta(const ClassifyArgs &a, const TwoPassArgs &p,
		uint64_t t)
{
	ItemMeta m;
	const uint64_t r = p.r_first + t;
	m.mate = r >= a.n ? 1u : 0u;
	m.i = r - (m.mate ? a.n : 0);
	const uint64_t o = a.off[m.mate][m.i];
	m.len = a.off[m.mate][m.i + 1] - o;
	m.start = o - a.off_base[m.mate];
	m.base = frame_base(p, t);
	return m;
}

/* Filter pass: (filter, read) items of reads [t0, t1) in filter-major order.
 * The next chunk's hashes and validity word, and the next item's metadata,
 * are loaded while the current ones are in use, to overlap their latency
 * with the probes.  MODE is the scoring method: SIMPLE and BINOMIAL run the
 * chunk machine of simple_chunk (BINOMIAL with integer hits), LENGTH
 * length_chunk, HARMONIC the sequential walk seq_chunk.  With DUST masking a
 * frame whose first base is masked is a miss that is not probed. */
template <bool COUNT, int MODE>
__global__ void __launch_bounds__(256, 6) filter_pass_kernel(ClassifyArgs a, TwoPassArgs p)
{
	constexpr bool LENGTH_MODE = MODE == BBT_SCORE_LENGTH;
	constexpr bool SEQ_MODE = MODE == BBT_SCORE_HARMONIC;
	const int lane = threadIdx.x & 31;
	const uint64_t nreads = p.t1 - p.t0;
	const uint64_t items = nreads * a.nf;
	const uint64_t pol = evict_first_policy();
	unsigned long long probe_acc = 0, alg_acc = 0;
	for (;;) {
		unsigned long long b = 0;
		if (lane == 0)
			b = atomicAdd(p.work, 32ull);
		b = __shfl_sync(kFull, b, 0);
		if (b >= items)
			break;
		uint32_t f = (uint32_t)(b / nreads);
		uint64_t t = p.t0 + (b - (uint64_t)f * nreads);
		const uint64_t e = b + 32 < items ? b + 32 : items;
		FilterDev F = a.filters[f];
		ItemMeta cur = item_meta(a, p, t);
		for (uint64_t it = b; it < e; ++it) {
			/* next item (same read range, maybe next filter) */
			uint64_t tn = t + 1 == p.t1 ? p.t0 : t + 1;
			ItemMeta nxt = cur;
			if (it + 1 < e)
				nxt = item_meta(a, p, tn);
			if (cur.len >= F.k) {
				const uint64_t frames = cur.len - F.k + 1;
				const uint32_t *vm = p.vmask + cur.base / 32;
				const uint64_t *hs = p.h0 + cur.base;
				SimpleState st;
				LengthState ls;
				SeqState qs;
				if (LENGTH_MODE)
					length_init(ls, a.min_len, cur.len, (int)F.k);
				else if (SEQ_MODE)
					harmonic_init(qs, a.score, a.one_minus, frames);
				else if (MODE == BBT_SCORE_BINOMIAL)
					binomial_simple_init(st, a.bthres[f * a.bthres_rows + frames], frames);
				else
					simple_init(st, a.score, a.one_minus, frames);
				const uint32_t *dm = a.dust[cur.mate];
				int decided = EVAL_OPEN;
				unsigned reads = 0;
				/* two chunks (64 frames) per step; the second one's probes are
				 * speculative whenever the first one decides or opens a skip
				 * window into it */
				uint32_t Vn0 = ld_stream_u32(vm, pol);
				uint32_t Vn1 = frames > 32 ? ld_stream_u32(vm + 1, pol) : 0u;
				uint64_t hn0 = ((Vn0 >> lane) & 1u) ? ld_stream_u64(hs + lane, pol) : 0;
				uint64_t hn1 = ((Vn1 >> lane) & 1u) ? ld_stream_u64(hs + 32 + lane, pol) : 0;
				for (uint64_t c = 0; c < frames; c += 64) {
					const uint32_t V0 = Vn0, V1 = Vn1;
					const uint64_t h0v = hn0, h1v = hn1;
					if (c + 64 < frames) {
						Vn0 = ld_stream_u32(vm + (c >> 5) + 2, pol);
						Vn1 = c + 96 < frames ? ld_stream_u32(vm + (c >> 5) + 3, pol) : 0u;
						hn0 = ((Vn0 >> lane) & 1u) ? ld_stream_u64(hs + c + 64 + lane, pol) : 0;
						hn1 = ((Vn1 >> lane) & 1u) ? ld_stream_u64(hs + c + 96 + lane, pol) : 0;
					}
					const int32_t pf = (int32_t)c + lane;
					const int32_t from = LENGTH_MODE ? 0 : SEQ_MODE ? (int32_t)seq_probe_from(qs)
					                                                 : st.skip_until;
					const bool p0 = ((V0 >> lane) & 1u) && pf >= from &&
							!dust_low(dm, cur.start + (uint64_t)pf);
					const bool p1 = ((V1 >> lane) & 1u) && pf + 32 >= from &&
							!dust_low(dm, cur.start + (uint64_t)pf + 32);
					bool hit0, hit1;
					unsigned r0 = 0, r1 = 0;
					contains2(F, h0v, p0, h1v, p1, hit0, hit1, r0, r1);
					const uint32_t H0 = __ballot_sync(kFull, hit0);
					const uint32_t H1 = __ballot_sync(kFull, hit1);
					if (COUNT)
						reads += r0 + r1;
					uint32_t alg = 0;
					const int nf0 = (int)min((uint64_t)32, frames - c);
					decided = LENGTH_MODE
							? length_chunk(ls, V0, H0, (int64_t)c, nf0, COUNT ? &alg : nullptr)
							: SEQ_MODE
							? seq_chunk(qs, V0, H0, (int64_t)c, nf0, (int)F.k, a.streak_thr,
									COUNT ? &alg : nullptr)
							: simple_chunk(st, V0, H0, (int32_t)c, nf0, (int)F.k, (int)a.streak_thr,
									COUNT ? &alg : nullptr);
					if (COUNT && ((alg >> lane) & 1u))
						alg_acc += r0;
					if (decided || c + 32 >= frames)
						break;
					alg = 0;
					const int nf1 = (int)min((uint64_t)32, frames - c - 32);
					decided = LENGTH_MODE
							? length_chunk(ls, V1, H1, (int64_t)c + 32, nf1, COUNT ? &alg : nullptr)
							: SEQ_MODE
							? seq_chunk(qs, V1, H1, (int64_t)c + 32, nf1, (int)F.k, a.streak_thr,
									COUNT ? &alg : nullptr)
							: simple_chunk(st, V1, H1, (int32_t)c + 32, nf1, (int)F.k,
									(int)a.streak_thr, COUNT ? &alg : nullptr);
					if (COUNT && ((alg >> lane) & 1u))
						alg_acc += r1;
					if (decided)
						break;
				}
				if (COUNT)
					probe_acc += reads;
				if (decided == EVAL_ACCEPT && lane == (int)(f >> 6))
					atomicOr((unsigned long long *)&a.hits[cur.mate][cur.i * a.words + lane],
							1ull << (f & 63));
			}
			t = tn;
			if (t == p.t0) {
				++f;
				if (f < a.nf)
					F = a.filters[f];
			}
			cur = nxt;
		}
	}
	if (COUNT) {
		for (int o = 16; o; o >>= 1) {
			probe_acc += __shfl_xor_sync(kFull, probe_acc, o);
			alg_acc += __shfl_xor_sync(kFull, alg_acc, o);
		}
		if (lane == 0) {
			if (a.probes)
				atomicAdd(a.probes, probe_acc);
			if (a.alg_probes)
				atomicAdd(a.alg_probes, alg_acc);
		}
	}
}

/* Score pass: SeqEval::evalScore of (filter, read) items in filter-major
 * order (BESTHIT / SCORES), the exhaustive walk of score_chunk over the
 * stored hashes; lane 0 writes the item's score to sa.scores[mate]. */
template <int MODE>
__global__ void __launch_bounds__(256, 6) score_pass_kernel(ClassifyArgs a, TwoPassArgs p,
		ScoreArgs sa)
{
	const int lane = threadIdx.x & 31;
	const uint64_t nreads = p.t1 - p.t0;
	const uint64_t items = nreads * a.nf;
	const uint64_t pol = evict_first_policy();
	for (;;) {
		unsigned long long b = 0;
		if (lane == 0)
			b = atomicAdd(p.work, 32ull);
		b = __shfl_sync(kFull, b, 0);
		if (b >= items)
			break;
		uint32_t f = (uint32_t)(b / nreads);
		uint64_t t = p.t0 + (b - (uint64_t)f * nreads);
		const uint64_t e = b + 32 < items ? b + 32 : items;
		FilterDev F = a.filters[f];
		ItemMeta cur = item_meta(a, p, t);
		for (uint64_t it = b; it < e; ++it) {
			uint64_t tn = t + 1 == p.t1 ? p.t0 : t + 1;
			ItemMeta nxt = cur;
			if (it + 1 < e)
				nxt = item_meta(a, p, tn);
			ScoreState st;
			score_init(st);
			if (cur.len >= F.k) {
				const uint64_t frames = cur.len - F.k + 1;
				const uint32_t *vm = p.vmask + cur.base / 32;
				const uint64_t *hs = p.h0 + cur.base;
				const uint32_t *dm = a.dust[cur.mate];
				unsigned reads = 0;
				uint32_t Vn = ld_stream_u32(vm, pol);
				uint64_t hn = ((Vn >> lane) & 1u) ? ld_stream_u64(hs + lane, pol) : 0;
				for (uint64_t c = 0; c < frames; c += 32) {
					const uint32_t V = Vn;
					const uint64_t hv = hn;
					if (c + 32 < frames) {
						Vn = ld_stream_u32(vm + (c >> 5) + 1, pol);
						hn = ((Vn >> lane) & 1u) ? ld_stream_u64(hs + c + 32 + lane, pol) : 0;
					}
					const int64_t pf = (int64_t)c + lane;
					const bool probe = ((V >> lane) & 1u) &&
							(MODE == SCORE_LENGTH || pf >= st.skip_end) &&
							!dust_low(dm, cur.start + (uint64_t)pf);
					const bool hit = probe && contains(F, hv, reads);
					const uint32_t H = __ballot_sync(kFull, hit);
					const int nfc = (int)min((uint64_t)32, frames - c);
					score_chunk(st, V, H, (int64_t)c, nfc, (int)F.k, a.streak_thr, MODE);
				}
			}
			const double val = score_value<MODE>(st, cur.len, F.k,
					MODE == SCORE_BINOMIAL ? sa.fpr[f] : 0.0, lane);
			if (lane == 0)
				sa.scores[cur.mate][cur.i * a.nf + f] = val;
			t = tn;
			if (t == p.t0) {
				++f;
				if (f < a.nf)
					F = a.filters[f];
			}
			cur = nxt;
		}
	}
}

template <typename K>
unsigned persistent_blocks(K kern, int threads, size_t smem, int num_sms, uint64_t warps_needed)
{
	int per_sm = 0;
	if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, threads, smem) != cudaSuccess ||
			per_sm < 1)
		per_sm = 1;
	const uint64_t need = (warps_needed + threads / 32 - 1) / (threads / 32);
	const uint64_t full = (uint64_t)per_sm * num_sms;
	return (unsigned)std::max<uint64_t>(1, std::min(need, full));
}

} // namespace

cudaError_t two_pass_scan(const ClassifyArgs &a, unsigned k, uint64_t *local,
		unsigned long long *sums, cudaStream_t s)
{
	const uint64_t total = a.n * a.mates;
	const uint64_t nb = (total + kScanBlock - 1) / kScanBlock;
	scan_frames_kernel<<<(unsigned)nb, kScanBlock, 0, s>>>(a, 0, total, k, local, sums);
	cudaError_t e = cudaGetLastError();
	if (e != cudaSuccess)
		return e;
	scan_sums_kernel<<<1, kScanBlock, 0, s>>>(sums, nb);
	return cudaGetLastError();
}

uint64_t two_pass_block_reads()
{
	return kScanBlock;
}

cudaError_t two_pass_sub_batch(const ClassifyArgs &a, const TwoPassArgs &p, const LaunchConfig &lc,
		cudaStream_t s, const ScoreArgs *sa, bool classify)
{
	const uint64_t nreads = p.t1 - p.t0;
	if (nreads == 0)
		return cudaSuccess;
	cudaError_t e = cudaMemsetAsync(p.work, 0, sizeof(unsigned long long), s);
	if (e != cudaSuccess)
		return e;
	const int threads = 256;
	const bool C = lc.count != 0;
	{
		const size_t smem = (lc.seg == 8 ? window_stride<8>(a.kmax) : window_stride<4>(a.kmax)) *
				(threads / 32);
		auto kern = lc.seg == 8 ? (C ? hash_pass_kernel<8, true> : hash_pass_kernel<8, false>)
		                        : (C ? hash_pass_kernel<4, true> : hash_pass_kernel<4, false>);
		if ((e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
				(int)smem)) != cudaSuccess)
			return e;
		kern<<<persistent_blocks(kern, threads, smem, lc.num_sms, nreads), threads, smem, s>>>(a, p);
		if ((e = cudaGetLastError()) != cudaSuccess)
			return e;
	}
	if (classify) {
		if ((e = cudaMemsetAsync(p.work, 0, sizeof(unsigned long long), s)) != cudaSuccess)
			return e;
		auto kern = a.scoring == BBT_SCORE_LENGTH
				? (C ? filter_pass_kernel<true, BBT_SCORE_LENGTH>
				     : filter_pass_kernel<false, BBT_SCORE_LENGTH>)
				: a.scoring == BBT_SCORE_HARMONIC
				? (C ? filter_pass_kernel<true, BBT_SCORE_HARMONIC>
				     : filter_pass_kernel<false, BBT_SCORE_HARMONIC>)
				: a.scoring == BBT_SCORE_BINOMIAL
				? (C ? filter_pass_kernel<true, BBT_SCORE_BINOMIAL>
				     : filter_pass_kernel<false, BBT_SCORE_BINOMIAL>)
				: (C ? filter_pass_kernel<true, BBT_SCORE_SIMPLE>
				     : filter_pass_kernel<false, BBT_SCORE_SIMPLE>);
		kern<<<persistent_blocks(kern, threads, 0, lc.num_sms, (nreads * a.nf + 31) / 32), threads,
				0, s>>>(a, p);
		if ((e = cudaGetLastError()) != cudaSuccess)
			return e;
	}
	if (sa) {
		if ((e = cudaMemsetAsync(p.work, 0, sizeof(unsigned long long), s)) != cudaSuccess)
			return e;
		auto kern = a.scoring == BBT_SCORE_LENGTH ? score_pass_kernel<SCORE_LENGTH>
		          : a.scoring == BBT_SCORE_HARMONIC ? score_pass_kernel<SCORE_HARMONIC>
		          : a.scoring == BBT_SCORE_BINOMIAL ? score_pass_kernel<SCORE_BINOMIAL>
		                                            : score_pass_kernel<SCORE_SIMPLE>;
		kern<<<persistent_blocks(kern, threads, 0, lc.num_sms, (nreads * a.nf + 31) / 32), threads,
				0, s>>>(a, p, *sa);
		if ((e = cudaGetLastError()) != cudaSuccess)
			return e;
	}
	return cudaSuccess;
}

} // namespace bbt
