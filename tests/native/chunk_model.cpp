/*
 * chunk_model.cpp -- host build of the product's chunked SeqEval state
 * machine (biobloom_b200/csrc/seqeval_chunk.cuh), fed with per-frame hit bits
 * from the CPU oracle.  Used by tests/test_chunk_model.py to check the
 * chunked decision, and the count of probes the sequential algorithm makes,
 * against the oracle's evalSimple / evalMinMatchLen on random reads, without a
 * GPU.
 */
#include "seqeval_chunk.cuh"
#include "bbt_oracle.h"
#include <vector>

static int model_eval_steps(const char *seq, uint64_t len, const oracle_bf *bf,
		double threshold, unsigned streak_thr, int scoring, uint64_t *alg_probes, int tight,
		int count);

extern "C" int model_eval(const char *seq, uint64_t len, const oracle_bf *bf,
		double threshold, unsigned streak_thr, int scoring, uint64_t *alg_probes)
{
	/* both step policies of the kernel must give the oracle's decision and
	 * algorithmic probe count, and the kernels' path without probe
	 * accounting (alg == nullptr) the same decision */
	uint64_t a1 = 0, a2 = 0, a3 = 0;
	const int d1 = model_eval_steps(seq, len, bf, threshold, streak_thr, scoring, &a1, 1, 1);
	const int d2 = model_eval_steps(seq, len, bf, threshold, streak_thr, scoring, &a2, 0, 1);
	const int d3 = model_eval_steps(seq, len, bf, threshold, streak_thr, scoring, &a3, 0, 0);
	if (d1 != d2 || a1 != a2 || d3 != d1)
		return -1;
	*alg_probes += a1;
	return d1;
}

static int model_eval_steps(const char *seq, uint64_t len, const oracle_bf *bf,
		double threshold, unsigned streak_thr, int scoring, uint64_t *alg_probes, int tight,
		int count)
{
	const unsigned k = bf->k;
	if (len < k)
		return 0;
	const uint64_t frames = len - k + 1;
	std::vector<uint8_t> valid(frames), hit(frames);
	std::vector<uint32_t> cost(frames);
	/* validity, hit bit and bit-test count of every frame, from the oracle */
	oracle_ntitr it;
	for (oracle_ntitr_init(&it, seq, len, bf->h, k); !oracle_ntitr_end(&it);
			oracle_ntitr_next(&it)) {
		uint64_t c = 0;
		valid[it.pos] = 1;
		hit[it.pos] = (uint8_t)oracle_bf_contains(bf, it.hv, &c);
		cost[it.pos] = (uint32_t)c;
	}
	if (scoring == ORACLE_HARMONIC) {
		/* the kernel's 32-frame steps over the sequential walk */
		bbt::SeqState qs;
		bbt::harmonic_init(qs, threshold, 1.0 - threshold, frames);
		for (uint64_t base = 0; base < frames; base += 32) {
			const int nf = frames - base >= 32 ? 32 : (int)(frames - base);
			const int64_t from = bbt::seq_probe_from(qs);
			uint32_t V = 0, H = 0;
			for (int j = 0; j < nf; ++j) {
				const uint64_t p = base + j;
				if (!valid[p])
					continue;
				V |= 1u << j;
				if ((int64_t)p >= from && hit[p])
					H |= 1u << j;
			}
			uint32_t alg = 0;
			const int d = bbt::seq_chunk(qs, V, H, (int64_t)base, nf, (int)k, streak_thr,
					count ? &alg : nullptr);
			for (int j = 0; j < nf; ++j)
				if ((alg >> j) & 1u)
					*alg_probes += cost[base + j];
			if (d)
				return d == bbt::EVAL_ACCEPT;
		}
		return 0;
	}
	bbt::SimpleState ss;
	bbt::LengthState ls;
	if (scoring == ORACLE_LENGTH)
		bbt::length_init(ls, (unsigned)(threshold + 0.5), len, (int)k);
	else if (scoring == ORACLE_BINOMIAL) /* evalSimple's machine with integer hits */
		bbt::binomial_simple_init(ss, oracle_calc_min_count((unsigned)frames,
				oracle_bf_fpr(bf), threshold), frames);
	else
		bbt::simple_init(ss, threshold, 1.0 - threshold, frames);
	for (uint64_t base = 0; base < frames;) {
		/* step sizes as the kernel takes them (classify.cu) */
		const int step = (scoring == ORACLE_LENGTH || !tight) ? 32 : bbt::simple_step_frames(ss);
		int nf = frames - base >= (uint64_t)step ? step : (int)(frames - base);
		uint32_t V = 0, H = 0;
		for (int j = 0; j < nf; ++j) {
			uint64_t p = base + j;
			if (!valid[p])
				continue;
			V |= 1u << j;
			bool probe = scoring == ORACLE_LENGTH || (int64_t)p >= ss.skip_until;
			if (probe && hit[p])
				H |= 1u << j;
		}
		uint32_t alg = 0;
		uint32_t *ap = count ? &alg : nullptr;
		int d = scoring == ORACLE_LENGTH
				? bbt::length_chunk(ls, V, H, (int64_t)base, nf, ap)
				: bbt::simple_chunk(ss, V, H, (int32_t)base, nf, (int)k, (int)streak_thr, ap);
		for (int j = 0; j < nf; ++j)
			if ((alg >> j) & 1u)
				*alg_probes += cost[base + j];
		if (d)
			return d == bbt::EVAL_ACCEPT;
		base += nf;
	}
	return 0;
}

/* SeqEval::evalScore as the scoring kernels compute it: 32-frame chunks,
 * frames probed from the skip window's end (every valid frame for LENGTH),
 * score_chunk over the ballots, then the final value (the BINOMIAL tail from
 * the oracle's own sum, which the tests compare against). */
extern "C" double model_score(const char *seq, uint64_t len, const oracle_bf *bf, int scoring,
		unsigned streak_thr, double fpr)
{
	const unsigned k = bf->k;
	bbt::ScoreState st;
	bbt::score_init(st);
	const int mode = scoring; /* ORACLE_* and SCORE_* share values */
	if (len >= k) {
		const uint64_t frames = len - k + 1;
		std::vector<uint8_t> valid(frames), hit(frames);
		oracle_ntitr it;
		for (oracle_ntitr_init(&it, seq, len, bf->h, k); !oracle_ntitr_end(&it);
				oracle_ntitr_next(&it)) {
			valid[it.pos] = 1;
			hit[it.pos] = (uint8_t)oracle_bf_contains(bf, it.hv, nullptr);
		}
		for (uint64_t base = 0; base < frames; base += 32) {
			const int nf = frames - base >= 32 ? 32 : (int)(frames - base);
			const int64_t from = st.skip_end;
			uint32_t V = 0, H = 0;
			for (int j = 0; j < nf; ++j) {
				const uint64_t p = base + j;
				if (!valid[p])
					continue;
				V |= 1u << j;
				if ((mode == bbt::SCORE_LENGTH || (int64_t)p >= from) && hit[p])
					H |= 1u << j;
			}
			bbt::score_chunk(st, V, H, (int64_t)base, nf, (int)k, streak_thr, mode);
		}
	}
	if (mode == bbt::SCORE_LENGTH)
		return (double)st.run;
	if (mode == bbt::SCORE_BINOMIAL) {
		if (len < k)
			return log10(1.0) * -10;
		return log10(oracle_binom_sf((unsigned)(len - k + 1), fpr, (unsigned)st.score)) * -10;
	}
	return bbt::score_normalize(st.score, len, k);
}
