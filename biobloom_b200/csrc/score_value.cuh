/*
 * score_value.cuh -- the last step of SeqEval::evalScore (Common/SeqEval.h:
 * 534-560) for one (read, filter): from the exhaustive walk's state
 * (score_chunk, seqeval_chunk.cuh) to the value the reference returns.
 * Device code shared by the read-major scoring kernel (score.cu) and the
 * filter-major score pass (twopass.cu).  Every lane of the warp calls these
 * together (the binomial tail is summed by the warp).
 */
#ifndef BBT_SCORE_VALUE_CUH
#define BBT_SCORE_VALUE_CUH

#include <stdint.h>

#include "seqeval_chunk.cuh"
#include "window.cuh"

namespace bbt {

/* Sum over the warp in a fixed order, the same value in every lane (a
 * butterfly would give lanes differently rounded sums). */
__device__ __forceinline__ double warp_sum_uniform(double v)
{
	for (int o = 16; o; o >>= 1)
		v += __shfl_down_sync(kFull, v, o);
	return __shfl_sync(kFull, v, 0);
}

/*
 * P(X > c) for X ~ Binomial(n, p): SeqEval::calcProbMatches
 * (Common/SeqEval.h:209-216), boost's cdf(complement(binomial(n, p), c)).
 * The probability masses C(n,i) p^i (1-p)^(n-i) are evaluated in log space
 * (lgamma, log, log1p, exp), 32 terms per step, from i = c + 1 upwards; past
 * the mode (n+1)p the terms only shrink, and the sum stops once a step adds
 * less than 2^-60 of it.  Within a few units in the last place of boost's
 * value (the terms are positive, so the sum has no cancellation).
 */
__device__ __forceinline__ double binom_sf_warp(uint32_t n, double p, uint32_t c, int lane)
{
	if (c >= n)
		return 0.0;
	if (p <= 0.0)
		return 0.0;
	if (p >= 1.0)
		return 1.0;
	const double dn = (double)n;
	const double lp = log(p), lq = log1p(-p), lgn = lgamma(dn + 1.0);
	const double mode = floor((dn + 1.0) * p);
	double sum = 0.0;
	for (uint32_t i0 = c + 1; i0 <= n; i0 += 32) {
		const uint32_t i = i0 + (uint32_t)lane;
		double t = 0.0;
		if (i <= n && i >= i0) {
			const double di = (double)i;
			t = exp(lgn - lgamma(di + 1.0) - lgamma(dn - di + 1.0) + di * lp + (dn - di) * lq);
		}
		const double step = warp_sum_uniform(t);
		sum += step;
		if ((double)i0 > mode && step <= sum * 0x1p-60)
			break;
		if (i0 > n - 32u)
			break;
	}
	return sum;
}

/* log10(calcProbMatches(...)) * -10, as evalScore returns it for BINOMIAL
 * (Common/SeqEval.h:545-555); a read shorter than k scores log10(1.0) * -10. */
__device__ __forceinline__ double binomial_score(uint64_t len, unsigned k, uint32_t count, double fpr, int lane)
{
	if (len < k)
		return log10(1.0) * -10.0;
	const uint32_t frame_len = (uint32_t)(len - k + 1);
	return log10(binom_sf_warp(frame_len, fpr, count, lane)) * -10.0;
}

/* The score of one (read, filter) walk: SIMPLE / HARMONIC sum over
 * len - k + 1, LENGTH's final run, BINOMIAL's -10 log10 P(X > hits). */
template <int MODE>
__device__ __forceinline__ double score_value(const ScoreState &st, uint64_t len, unsigned k,
		double fpr, int lane)
{
	if (MODE == SCORE_LENGTH)
		return (double)st.run;
	if (MODE == SCORE_BINOMIAL)
		return binomial_score(len, k, (uint32_t)st.score, fpr, lane);
	return score_normalize(st.score, len, k);
}

} // namespace bbt

#endif
