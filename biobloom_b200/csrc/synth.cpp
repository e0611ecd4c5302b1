/*
 * synth.cpp -- seeded synthetic genomes and reads for the benchmark and test
 * workloads (the reference measures on dwgsim-simulated reads,
 * Tests/SystemTests/systemTest.pl:36-39; no dataset is available here, so
 * these generators stand in with the shapes, sizes and error rates of the
 * workloads).
 *
 * Every random draw comes from a counter-based generator (splitmix64 of
 * seed, stream, index), so output is identical for any thread count.
 * Host-only code; it needs no GPU.
 */
#include "bbt.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <omp.h>
#include <vector>

namespace {

inline uint64_t mix64(uint64_t z)
{
	z += 0x9e3779b97f4a7c15ULL;
	z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
	z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
	return z ^ (z >> 31);
}

/* Small sequential generator seeded from (seed, stream, index). */
struct Rng {
	uint64_t s;
	Rng(uint64_t seed, uint64_t stream, uint64_t index)
		: s(mix64(seed ^ mix64(stream * 0x632be59bd9b4e019ULL ^ mix64(index)))) {}
	uint64_t next() { s += 0x9e3779b97f4a7c15ULL; return mix64(s); }
	double uniform() { return double(next() >> 11) * (1.0 / 9007199254740992.0); }
	uint64_t below(uint64_t n) { return n ? next() % n : 0; }
};

const char kBases[4] = {'A', 'C', 'G', 'T'};

inline char random_base(Rng &r, double gc)
{
	double u = r.uniform();
	if (u < gc)
		return u < gc * 0.5 ? 'C' : 'G';
	return (u - gc) < (1.0 - gc) * 0.5 ? 'A' : 'T';
}

inline char substitute(Rng &r, char b)
{
	int idx = b == 'A' ? 0 : b == 'C' ? 1 : b == 'G' ? 2 : 3;
	return kBases[(idx + 1 + (int)r.below(3)) & 3];
}

inline char complement(char b)
{
	switch (b) {
	case 'A': return 'T';
	case 'C': return 'G';
	case 'G': return 'C';
	case 'T': return 'A';
	default: return 'N';
	}
}

inline uint32_t log_uniform(Rng &r, double lo, double hi)
{
	double v = std::exp(std::log(lo) + r.uniform() * (std::log(hi) - std::log(lo)));
	uint32_t x = (uint32_t)std::floor(v);
	return x < (uint32_t)lo ? (uint32_t)lo : x;
}

} // namespace

extern "C" int bbt_synth_genome(uint64_t seed, uint64_t len, double gc,
		double repeat_frac, uint32_t rep_min, uint32_t rep_max,
		double div_min, double div_max, char *out)
{
	if (!out || gc < 0 || gc > 1 || repeat_frac < 0 || repeat_frac >= 1)
		return BBT_ERR_ARG;
	const uint64_t chunk = 1 << 16;
	const uint64_t nchunks = (len + chunk - 1) / chunk;
#pragma omp parallel for schedule(static)
	for (int64_t c = 0; c < (int64_t)nchunks; ++c) {
		Rng r(seed, 1, (uint64_t)c);
		uint64_t b = (uint64_t)c * chunk, e = std::min(len, b + chunk);
		for (uint64_t i = b; i < e; ++i)
			out[i] = random_base(r, gc);
	}
	if (repeat_frac <= 0 || rep_min == 0 || rep_max < rep_min || len < 2ull * rep_max)
		return BBT_OK;
	/* Repeat families: random templates of log-uniform length in
	 * [rep_min, rep_max]; copies with per-copy divergence in [div_min,
	 * div_max] are placed in fixed-size blocks (one copy per block, at a
	 * random offset), with the copy probability per block chosen so the
	 * expected repeated fraction is repeat_frac. */
	const uint32_t nfam = 64;
	std::vector<std::vector<char> > fam(nfam);
	double mean_len = 0;
	for (uint32_t f = 0; f < nfam; ++f) {
		Rng r(seed, 2, f);
		uint32_t L = rep_min == rep_max ? rep_min : log_uniform(r, rep_min, rep_max);
		fam[f].resize(L);
		for (uint32_t i = 0; i < L; ++i)
			fam[f][i] = random_base(r, gc);
		mean_len += L;
	}
	mean_len /= nfam;
	const uint64_t block = std::max<uint64_t>(2ull * rep_max, (uint64_t)std::ceil(mean_len / repeat_frac));
	const double p_copy = std::min(1.0, repeat_frac * (double)block / mean_len);
	const uint64_t nblocks = len / block;
#pragma omp parallel for schedule(static)
	for (int64_t bk = 0; bk < (int64_t)nblocks; ++bk) {
		Rng r(seed, 3, (uint64_t)bk);
		if (r.uniform() >= p_copy)
			continue;
		const std::vector<char> &t = fam[r.below(nfam)];
		uint64_t start = (uint64_t)bk * block + r.below(block - t.size() + 1);
		double d = div_min + (div_max - div_min) * r.uniform();
		for (size_t i = 0; i < t.size(); ++i)
			out[start + i] = (d > 0 && r.uniform() < d) ? substitute(r, t[i]) : t[i];
	}
	return BBT_OK;
}

namespace {

struct ReadSpec {
	const char *refs;
	const uint64_t *ref_off;
	uint32_t n_refs;
	const double *ref_frac; /* cumulative over references; rest random */
	const bbt_synth_read_params *p;
};

inline uint32_t draw_length(Rng &r, const bbt_synth_read_params *p)
{
	if (p->len_min == p->len_max && p->long_frac <= 0)
		return p->len_min;
	if (p->long_frac > 0 && r.uniform() < p->long_frac)
		return log_uniform(r, p->long_min, p->long_max);
	return log_uniform(r, p->len_min, p->len_max);
}

/* Source of read i: reference index, or n_refs for random. */
inline uint32_t draw_source(Rng &r, const ReadSpec &s)
{
	double u = r.uniform();
	for (uint32_t j = 0; j < s.n_refs; ++j)
		if (u < s.ref_frac[j])
			return j;
	return s.n_refs;
}

/* Fill one read (or mate) of length L. */
void make_read(Rng &r, const ReadSpec &s, uint32_t src, uint64_t frag_start,
		bool minus, uint32_t L, char *dst)
{
	const bbt_synth_read_params *p = s.p;
	if (src >= s.n_refs) {
		for (uint32_t i = 0; i < L; ++i)
			dst[i] = kBases[r.below(4)];
	} else {
		const char *ref = s.refs + s.ref_off[src];
		for (uint32_t i = 0; i < L; ++i)
			dst[i] = minus ? complement(ref[frag_start + L - 1 - i]) : ref[frag_start + i];
	}
	for (uint32_t i = 0; i < L; ++i) {
		if (p->sub_rate > 0 && r.uniform() < p->sub_rate)
			dst[i] = substitute(r, dst[i] == 'N' ? 'A' : dst[i]);
		if (p->n_rate > 0 && r.uniform() < p->n_rate)
			dst[i] = 'N';
	}
}

} // namespace

extern "C" int bbt_synth_read_lengths(uint64_t seed,
		const bbt_synth_read_params *p, uint64_t n_reads, uint64_t *out_off)
{
	if (!p || !out_off || p->len_min == 0 || p->len_max < p->len_min)
		return BBT_ERR_ARG;
	out_off[0] = 0;
#pragma omp parallel for schedule(static)
	for (int64_t i = 0; i < (int64_t)n_reads; ++i) {
		Rng r(seed, 10, (uint64_t)i);
		out_off[i + 1] = draw_length(r, p);
	}
	for (uint64_t i = 0; i < n_reads; ++i)
		out_off[i + 1] += out_off[i];
	return BBT_OK;
}

extern "C" int bbt_synth_reads(uint64_t seed, const char *refs,
		const uint64_t *ref_off, uint32_t n_refs, const double *ref_frac,
		const bbt_synth_read_params *p, uint64_t n_reads,
		const uint64_t *off, char *out1, char *out2, uint32_t *out_src)
{
	if (!p || !off || !out1 || (n_refs && (!refs || !ref_off || !ref_frac)))
		return BBT_ERR_ARG;
	std::vector<double> cum(n_refs);
	double acc = 0;
	for (uint32_t j = 0; j < n_refs; ++j) {
		acc += ref_frac[j];
		cum[j] = acc;
	}
	ReadSpec s = {refs, ref_off, n_refs, cum.data(), p};
	int bad = 0;
#pragma omp parallel for schedule(static) reduction(| : bad)
	for (int64_t i = 0; i < (int64_t)n_reads; ++i) {
		uint32_t L = (uint32_t)(off[i + 1] - off[i]);
		Rng r(seed, 11, (uint64_t)i);
		uint32_t src = draw_source(r, s);
		bool minus = (r.next() & 1) != 0;
		uint64_t frag = 0;
		uint32_t flen = L;
		if (out2 && p->frag_max > 0)
			flen = std::max<uint32_t>(L, p->frag_min + (uint32_t)r.below(p->frag_max - p->frag_min + 1));
		if (src < n_refs) {
			uint64_t rl = ref_off[src + 1] - ref_off[src];
			if (rl < flen) {
				bad |= 1;
				continue;
			}
			frag = r.below(rl - flen + 1);
		}
		if (out_src)
			out_src[i] = src;
		if (!out2) {
			make_read(r, s, src, frag, minus, L, out1 + off[i]);
		} else {
			/* mate 1 reads the fragment's first L bases on its strand,
			 * mate 2 the last L bases on the other strand */
			uint64_t a = frag, b = frag + flen - L;
			make_read(r, s, src, minus ? b : a, minus, L, out1 + off[i]);
			make_read(r, s, src, minus ? a : b, !minus, L, out2 + off[i]);
		}
	}
	return bad ? BBT_ERR_ARG : BBT_OK;
}
