/*
 * synth_oracle.c -- TEST INFRASTRUCTURE ONLY.
 *
 * The seeded workload generator and a multi-threaded Bloom filter build for
 * the CPU arm of the benchmark, which must run the reference's classifier on
 * the same inputs as the GPU arm without loading the product library.
 *
 * The generator restates the product's bbt_synth_genome /
 * bbt_synth_read_lengths / bbt_synth_reads (a counter-based generator:
 * splitmix64 of (seed, stream, index), so the output does not depend on the
 * thread count); tests/test_synth_oracle.py checks that both produce the
 * same bytes.  The reference measures on dwgsim-simulated reads
 * (Tests/SystemTests/systemTest.pl:36-39); no dataset is available here.
 *
 * oracle_make_filter_par builds the bit array of
 * BloomFilterGenerator::generate (BioBloomMaker/BloomFilterGenerator.cpp:54-73)
 * with OpenMP threads setting bits by atomic OR.  The bit array does not depend
 * on insertion order, so it equals the sequential build's (tested against
 * oracle_make_filter); the count of k-mers found already present does depend
 * on the order, as it does in the reference's own threaded loaders.
 */
#include "bbt_oracle.h"
#include "synth_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

static uint64_t mix64(uint64_t z)
{
	z += 0x9e3779b97f4a7c15ULL;
	z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
	z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
	return z ^ (z >> 31);
}

typedef struct {
	uint64_t s;
} rng_t;

static void rng_init(rng_t *r, uint64_t seed, uint64_t stream, uint64_t index)
{
	r->s = mix64(seed ^ mix64(stream * 0x632be59bd9b4e019ULL ^ mix64(index)));
}

static uint64_t rng_next(rng_t *r)
{
	r->s += 0x9e3779b97f4a7c15ULL;
	return mix64(r->s);
}

static double rng_uniform(rng_t *r)
{
	return (double)(rng_next(r) >> 11) * (1.0 / 9007199254740992.0);
}

static uint64_t rng_below(rng_t *r, uint64_t n)
{
	return n ? rng_next(r) % n : 0;
}

static const char kBases[4] = {'A', 'C', 'G', 'T'};

static char random_base(rng_t *r, double gc)
{
	double u = rng_uniform(r);
	if (u < gc)
		return u < gc * 0.5 ? 'C' : 'G';
	return (u - gc) < (1.0 - gc) * 0.5 ? 'A' : 'T';
}

static char substitute(rng_t *r, char b)
{
	int idx = b == 'A' ? 0 : b == 'C' ? 1 : b == 'G' ? 2 : 3;
	return kBases[(idx + 1 + (int)rng_below(r, 3)) & 3];
}

static char complement(char b)
{
	switch (b) {
	case 'A': return 'T';
	case 'C': return 'G';
	case 'G': return 'C';
	case 'T': return 'A';
	default: return 'N';
	}
}

static uint32_t log_uniform(rng_t *r, double lo, double hi)
{
	double v = exp(log(lo) + rng_uniform(r) * (log(hi) - log(lo)));
	uint32_t x = (uint32_t)floor(v);
	return x < (uint32_t)lo ? (uint32_t)lo : x;
}

int oracle_synth_genome(uint64_t seed, uint64_t len, double gc, double repeat_frac,
		uint32_t rep_min, uint32_t rep_max, double div_min, double div_max, char *out)
{
	if (!out || gc < 0 || gc > 1 || repeat_frac < 0 || repeat_frac >= 1)
		return -1;
	const uint64_t chunk = 1 << 16;
	const int64_t nchunks = (int64_t)((len + chunk - 1) / chunk);
#pragma omp parallel for schedule(static)
	for (int64_t c = 0; c < nchunks; ++c) {
		rng_t r;
		rng_init(&r, seed, 1, (uint64_t)c);
		uint64_t b = (uint64_t)c * chunk, e = b + chunk < len ? b + chunk : len;
		for (uint64_t i = b; i < e; ++i)
			out[i] = random_base(&r, gc);
	}
	if (repeat_frac <= 0 || rep_min == 0 || rep_max < rep_min || len < 2ull * rep_max)
		return 0;
	/* repeat families: 64 random templates, copies placed one per block */
	enum { NFAM = 64 };
	char *fam[NFAM];
	uint32_t flen[NFAM];
	double mean_len = 0;
	for (uint32_t f = 0; f < NFAM; ++f) {
		rng_t r;
		rng_init(&r, seed, 2, f);
		uint32_t L = rep_min == rep_max ? rep_min : log_uniform(&r, rep_min, rep_max);
		fam[f] = (char *)malloc(L ? L : 1);
		if (!fam[f]) {
			for (uint32_t g = 0; g < f; ++g)
				free(fam[g]);
			return -1;
		}
		flen[f] = L;
		for (uint32_t i = 0; i < L; ++i)
			fam[f][i] = random_base(&r, gc);
		mean_len += L;
	}
	mean_len /= NFAM;
	uint64_t block = (uint64_t)ceil(mean_len / repeat_frac);
	if (block < 2ull * rep_max)
		block = 2ull * rep_max;
	double p_copy = repeat_frac * (double)block / mean_len;
	if (p_copy > 1.0)
		p_copy = 1.0;
	const int64_t nblocks = (int64_t)(len / block);
#pragma omp parallel for schedule(static)
	for (int64_t bk = 0; bk < nblocks; ++bk) {
		rng_t r;
		rng_init(&r, seed, 3, (uint64_t)bk);
		if (rng_uniform(&r) >= p_copy)
			continue;
		const uint64_t f = rng_below(&r, NFAM);
		const char *t = fam[f];
		const uint64_t tl = flen[f];
		uint64_t start = (uint64_t)bk * block + rng_below(&r, block - tl + 1);
		double d = div_min + (div_max - div_min) * rng_uniform(&r);
		for (uint64_t i = 0; i < tl; ++i)
			out[start + i] = (d > 0 && rng_uniform(&r) < d) ? substitute(&r, t[i]) : t[i];
	}
	for (uint32_t f = 0; f < NFAM; ++f)
		free(fam[f]);
	return 0;
}

static uint32_t draw_length(rng_t *r, const oracle_read_params *p)
{
	if (p->len_min == p->len_max && p->long_frac <= 0)
		return p->len_min;
	if (p->long_frac > 0 && rng_uniform(r) < p->long_frac)
		return log_uniform(r, p->long_min, p->long_max);
	return log_uniform(r, p->len_min, p->len_max);
}

int oracle_synth_read_lengths(uint64_t seed, const oracle_read_params *p, uint64_t n_reads,
		uint64_t *out_off)
{
	if (!p || !out_off || p->len_min == 0 || p->len_max < p->len_min)
		return -1;
	out_off[0] = 0;
#pragma omp parallel for schedule(static)
	for (int64_t i = 0; i < (int64_t)n_reads; ++i) {
		rng_t r;
		rng_init(&r, seed, 10, (uint64_t)i);
		out_off[i + 1] = draw_length(&r, p);
	}
	for (uint64_t i = 0; i < n_reads; ++i)
		out_off[i + 1] += out_off[i];
	return 0;
}

static void make_read(rng_t *r, const char *refs, const uint64_t *ref_off, uint32_t n_refs,
		const oracle_read_params *p, uint32_t src, uint64_t frag_start, int minus, uint32_t L,
		char *dst)
{
	if (src >= n_refs) {
		for (uint32_t i = 0; i < L; ++i)
			dst[i] = kBases[rng_below(r, 4)];
	} else {
		const char *ref = refs + ref_off[src];
		for (uint32_t i = 0; i < L; ++i)
			dst[i] = minus ? complement(ref[frag_start + L - 1 - i]) : ref[frag_start + i];
	}
	for (uint32_t i = 0; i < L; ++i) {
		if (p->sub_rate > 0 && rng_uniform(r) < p->sub_rate)
			dst[i] = substitute(r, dst[i] == 'N' ? 'A' : dst[i]);
		if (p->n_rate > 0 && rng_uniform(r) < p->n_rate)
			dst[i] = 'N';
	}
}

int oracle_synth_reads(uint64_t seed, const char *refs, const uint64_t *ref_off,
		uint32_t n_refs, const double *ref_frac, const oracle_read_params *p,
		uint64_t n_reads, const uint64_t *off, char *out1, char *out2, uint32_t *out_src)
{
	if (!p || !off || !out1 || (n_refs && (!refs || !ref_off || !ref_frac)))
		return -1;
	double *cum = (double *)malloc((n_refs ? n_refs : 1) * sizeof(double));
	if (!cum)
		return -1;
	double acc = 0;
	for (uint32_t j = 0; j < n_refs; ++j) {
		acc += ref_frac[j];
		cum[j] = acc;
	}
	int bad = 0;
#pragma omp parallel for schedule(static) reduction(| : bad)
	for (int64_t i = 0; i < (int64_t)n_reads; ++i) {
		uint32_t L = (uint32_t)(off[i + 1] - off[i]);
		rng_t r;
		rng_init(&r, seed, 11, (uint64_t)i);
		double u = rng_uniform(&r);
		uint32_t src = n_refs;
		for (uint32_t j = 0; j < n_refs; ++j)
			if (u < cum[j]) {
				src = j;
				break;
			}
		int minus = (rng_next(&r) & 1) != 0;
		uint64_t frag = 0;
		uint32_t flen = L;
		if (out2 && p->frag_max > 0) {
			uint32_t fl = p->frag_min + (uint32_t)rng_below(&r, p->frag_max - p->frag_min + 1);
			flen = fl > L ? fl : L;
		}
		if (src < n_refs) {
			uint64_t rl = ref_off[src + 1] - ref_off[src];
			if (rl < flen) {
				bad |= 1;
				continue;
			}
			frag = rng_below(&r, rl - flen + 1);
		}
		if (out_src)
			out_src[i] = src;
		if (!out2) {
			make_read(&r, refs, ref_off, n_refs, p, src, frag, minus, L, out1 + off[i]);
		} else {
			uint64_t a = frag, b = frag + flen - L;
			make_read(&r, refs, ref_off, n_refs, p, src, minus ? b : a, minus, L, out1 + off[i]);
			make_read(&r, refs, ref_off, n_refs, p, src, minus ? a : b, !minus, L, out2 + off[i]);
		}
	}
	free(cum);
	return bad ? -1 : 0;
}

/* The k-mers [q0, q1) of seq (a window of one sequence), inserted with atomic
 * OR.  Their words are prefetched kDepth k-mers ahead, so that a core has
 * several cache misses in flight instead of one locked miss at a time.
 * *fresh receives the count of k-mers that set at least one new bit; the
 * return value counts those whose bits were all set already. */
enum { kDepth = 16, kMaxH = 64 };

static uint64_t insert_range(oracle_bf *bf, const char *seq, uint64_t len, uint64_t q0,
		uint64_t q1, uint64_t *fresh)
{
	const unsigned k = bf->k, h = bf->h;
	uint64_t red = 0, tot = 0;
	uint64_t *words = (uint64_t *)bf->bits;
	uint64_t ring[kDepth][kMaxH];
	unsigned head = 0, used = 0;
	oracle_ntitr it;
	uint64_t e = q1 + k - 1 < len ? q1 + k - 1 : len;
	oracle_ntitr_init(&it, seq + q0, (size_t)(e - q0), h, k);
	for (;;) {
		const int more = !oracle_ntitr_end(&it);
		if (more) {
			uint64_t *slot = ring[(head + used) % kDepth];
			for (unsigned i = 0; i < h; ++i) {
				slot[i] = it.hv[i] % bf->m;
				__builtin_prefetch(words + (slot[i] >> 6), 1, 0);
			}
			++used;
			oracle_ntitr_next(&it);
		}
		if (used == 0)
			break;
		if (used < kDepth && more)
			continue;
		const uint64_t *b = ring[head];
		int found = 1;
		for (unsigned i = 0; i < h; ++i) {
			uint64_t bit = 1ull << (b[i] & 63);
			uint64_t old = __atomic_fetch_or(words + (b[i] >> 6), bit, __ATOMIC_RELAXED);
			if (!(old & bit))
				found = 0;
		}
		red += (uint64_t)found;
		tot += (uint64_t)!found;
		head = (head + 1) % kDepth;
		--used;
	}
	*fresh = tot;
	return red;
}

int oracle_make_filter_par(oracle_bf *bf, const char *const *seqs, const uint64_t *lens,
		size_t n, unsigned k, double fpr, unsigned h, uint64_t *expected_entries,
		uint64_t *redundant)
{
	uint64_t expected = 0;
	for (size_t i = 0; i < n; ++i)
		expected += lens[i] - k + 1; /* size_t arithmetic, as upstream */
	if (h == 0)
		h = oracle_calc_optimal_hash_num(fpr);
	uint64_t m = oracle_calc_optimal_size(expected, fpr, h);
	if (h > kMaxH || oracle_bf_create(bf, m, h, k))
		return -1;
	bf->dfpr = fpr;
	uint64_t red = 0, tot = 0;
	const uint64_t piece = 1 << 20; /* k-mers per task */
	for (size_t s = 0; s < n; ++s) {
		if (lens[s] < k)
			continue;
		const uint64_t frames = lens[s] - k + 1;
		const int64_t np = (int64_t)((frames + piece - 1) / piece);
#pragma omp parallel for schedule(dynamic, 4) reduction(+ : red, tot)
		for (int64_t p = 0; p < np; ++p) {
			uint64_t q0 = (uint64_t)p * piece;
			uint64_t q1 = q0 + piece < frames ? q0 + piece : frames;
			uint64_t fresh = 0;
			red += insert_range(bf, seqs[s], lens[s], q0, q1, &fresh);
			tot += fresh;
		}
	}
	bf->n_entry = tot;
	bf->t_entry = tot + red;
	if (expected_entries)
		*expected_entries = expected;
	if (redundant)
		*redundant = red;
	return 0;
}
