/*
 * score.cu -- the exhaustive scoring kernel behind the BESTHIT (-b) and
 * SCORES (-w) modes: SeqEval::evalScore (Common/SeqEval.h:534-560) of every
 * read against every filter, as BioBloomClassifier::evaluateReadBestHit and
 * evaluateReadScore (BioBloomClassifier.cpp:1194-1237) call it.
 *
 * One warp scores one read (or mate) against all filters.  The hash window is
 * staged once per k (window.cuh); each 32-frame step probes the frames that
 * are not inside an open skip window, one per lane, and the warp-uniform walk
 * (score_chunk, seqeval_chunk.cuh) adds them up exactly as the sequential
 * loop does.  Nothing stops early: the whole read is walked for every filter.
 *
 * BESTHIT keeps, as the read's hit bits, the filters whose score equals the
 * largest one (maxScore < score replaces, == adds), and none when the largest
 * is not above 0 (evaluateReadBestHit).  SCORES writes every filter's score;
 * its hit bits come from the classification kernel.
 */
#include "classify.cuh"
#include "score_value.cuh"
#include "seqeval_chunk.cuh"
#include "window.cuh"

#include "bbt.h"

namespace bbt {

namespace {

template <int SEG, int MODE>
__device__ void score_read(const ClassifyArgs &a, const ScoreArgs &sa, uint64_t r,
		const Window<SEG> &win, int lane)
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
	double best = 0.0;
	uint64_t myword = 0;
	for (uint32_t f = 0; f < a.nf; ++f) {
		const FilterDev F = a.filters[f];
		const unsigned k = F.k;
		ScoreState st;
		score_init(st);
		if (len >= k) {
			const uint64_t frames = len - k + 1;
			for (uint64_t w0 = 0; w0 < frames; w0 += W) {
				const int wn = (int)min((uint64_t)W, frames - w0);
				if (cached_k != k || cached_w0 != (int64_t)w0) {
					if (cached_k != k)
						set_tables<SEG>(win, k, lane);
					hash_window<SEG>(s, w0, wn, k, win, lane);
					cached_k = k;
					cached_w0 = (int64_t)w0;
				}
				for (int c = 0; c < wn; c += 32) {
					const int nfc = min(32, wn - c);
					const int q = c + lane;
					const int64_t p = (int64_t)w0 + q;
					uint32_t V = win.vmask[c >> 5];
					if (nfc < 32)
						V &= (1u << nfc) - 1u;
					const bool v = (V >> lane) & 1u;
					const bool probe = v && (MODE == SCORE_LENGTH || p >= st.skip_end) &&
							!dust_low(a.dust[mate], start + (uint64_t)p);
					const bool hit = probe && contains(F, win.h0[q], reads);
					const uint32_t H = __ballot_sync(kFull, hit);
					score_chunk(st, V, H, (int64_t)w0 + c, nfc, (int)k, a.streak_thr, MODE);
				}
			}
		}
		const double val = score_value<MODE>(st, len, k, MODE == SCORE_BINOMIAL ? sa.fpr[f] : 0.0,
				lane);
		if (sa.scores[mate] && lane == 0)
			sa.scores[mate][i * a.nf + f] = val;
		if (sa.besthit) {
			const uint64_t bit = (lane == (int)(f >> 6)) ? 1ull << (f & 63) : 0ull;
			if (best < val) {
				best = val;
				myword = bit;
			} else if (best == val) {
				myword |= bit;
			}
		}
	}
	if (sa.besthit) {
		if (!(best > 0.0))
			myword = 0;
		if (lane < (int)a.words)
			a.hits[mate][i * a.words + lane] = myword;
	}
}

template <int SEG, int MODE>
__global__ void __launch_bounds__(256, 4) score_kernel(ClassifyArgs a, ScoreArgs sa)
{
	extern __shared__ __align__(16) unsigned char smem[];
	const int lane = threadIdx.x & 31;
	const int warp = threadIdx.x >> 5;
	const Window<SEG> win = window_at<SEG>(smem + warp * window_stride<SEG>(a.kmax));
	const uint64_t r = (uint64_t)blockIdx.x * (blockDim.x >> 5) + warp;
	if (r < a.n * a.mates)
		score_read<SEG, MODE>(a, sa, r, win, lane);
}

template <int SEG>
cudaError_t launch_score_seg(const ClassifyArgs &a, const ScoreArgs &sa, const LaunchConfig &lc,
		cudaStream_t s)
{
	const int threads = lc.warps_per_block * 32;
	const size_t smem = classify_smem_bytes(lc, a.kmax);
	auto kern = a.scoring == BBT_SCORE_LENGTH ? score_kernel<SEG, SCORE_LENGTH>
	          : a.scoring == BBT_SCORE_HARMONIC ? score_kernel<SEG, SCORE_HARMONIC>
	          : a.scoring == BBT_SCORE_BINOMIAL ? score_kernel<SEG, SCORE_BINOMIAL>
	                                            : score_kernel<SEG, SCORE_SIMPLE>;
	cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
			(int)smem);
	if (e != cudaSuccess)
		return e;
	const uint64_t total = a.n * a.mates;
	const uint64_t blocks = (total + lc.warps_per_block - 1) / lc.warps_per_block;
	if (blocks == 0)
		return cudaSuccess;
	kern<<<(unsigned)blocks, threads, smem, s>>>(a, sa);
	return cudaGetLastError();
}

/* evaluateReadBestHit over stored scores: one thread per read (mate). */
__global__ void best_hits_kernel(ClassifyArgs a, const double *s0, const double *s1)
{
	const uint64_t total = a.n * a.mates;
	for (uint64_t r = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; r < total;
			r += (uint64_t)gridDim.x * blockDim.x) {
		const uint32_t mate = r >= a.n ? 1u : 0u;
		const uint64_t i = r - (mate ? a.n : 0);
		const double *sc = (mate ? s1 : s0) + i * a.nf;
		uint64_t *h = a.hits[mate] + i * a.words;
		double best = 0.0;
		for (uint32_t f = 0; f < a.nf; ++f) {
			const double v = sc[f];
			if (best < v)
				best = v;
		}
		/* the filters whose score equals the largest, when it is above 0 */
		for (uint32_t w = 0; w < a.words; ++w) {
			uint64_t word = 0;
			if (best > 0.0)
				for (uint32_t b = 0; b < 64 && w * 64 + b < a.nf; ++b)
					word |= (uint64_t)(sc[w * 64 + b] == best) << b;
			h[w] = word;
		}
	}
}

} // namespace

cudaError_t launch_best_hits(const ClassifyArgs &a, double *const *scores, int num_sms,
		cudaStream_t s)
{
	const uint64_t total = a.n * a.mates;
	if (total == 0)
		return cudaSuccess;
	const uint64_t need = (total + 255) / 256;
	const uint64_t cap = (uint64_t)num_sms * 8;
	best_hits_kernel<<<(unsigned)(need < cap ? need : cap), 256, 0, s>>>(a, scores[0],
			a.mates == 2 ? scores[1] : nullptr);
	return cudaGetLastError();
}

cudaError_t launch_scores(const ClassifyArgs &a, const ScoreArgs &sa, const LaunchConfig &lc,
		cudaStream_t s)
{
	return lc.seg == 8 ? launch_score_seg<8>(a, sa, lc, s) : launch_score_seg<4>(a, sa, lc, s);
}

} // namespace bbt
