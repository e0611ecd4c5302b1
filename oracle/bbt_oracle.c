/*
 * bbt_oracle.c -- CPU oracle (test infrastructure only; see bbt_oracle.h).
 *
 * Plain sequential C.  Every function follows one reference function; the
 * comment above each names it.  Nothing here is optimised: it is the oracle
 * the GPU results are compared with.
 */
#include "bbt_oracle.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------------ */
/* ntHash (Mohamadi et al. 2016).  Each base has a 64-bit random seed; the    */
/* forward hash of s[0..k) is XOR_i rol(seed(s_i), k-1-i), the reverse-      */
/* complement hash is XOR_i rol(seed(comp(s_i)), i), the canonical hash is   */
/* the smaller of the two, and extra hashes are derived from the canonical   */
/* one by a multiply / shift-xor step.  Seeds are those of the published     */
/* method.                                                                    */
/* ------------------------------------------------------------------------ */

#define NT_SEED_A 0x3c8bfbb395c60474ULL
#define NT_SEED_C 0x3193c18562a02b4cULL
#define NT_SEED_G 0x20323ed082572324ULL
#define NT_SEED_T 0x295549f54be24456ULL
#define NT_MULTI_SEED 0x90b45d39fb6da1faULL
#define NT_MULTI_SHIFT 27

static inline uint64_t rol64(uint64_t v, unsigned s)
{
	s &= 63u;
	return s ? (v << s) | (v >> (64u - s)) : v;
}

static inline uint64_t ror64(uint64_t v, unsigned s)
{
	s &= 63u;
	return s ? (v >> s) | (v << (64u - s)) : v;
}

uint64_t oracle_nt_seed(unsigned char c)
{
	switch (c) {
	case 'A': case 'a': return NT_SEED_A;
	case 'C': case 'c': return NT_SEED_C;
	case 'G': case 'g': return NT_SEED_G;
	case 'T': case 't': return NT_SEED_T;
	default: return 0;
	}
}

uint64_t oracle_nt_seed_rc(unsigned char c)
{
	switch (c) {
	case 'A': case 'a': return NT_SEED_T;
	case 'C': case 'c': return NT_SEED_G;
	case 'G': case 'g': return NT_SEED_C;
	case 'T': case 't': return NT_SEED_A;
	default: return 0;
	}
}

int oracle_nt_valid(unsigned char c)
{
	return oracle_nt_seed(c) != 0;
}

uint64_t oracle_nt_forward(const char *s, unsigned k)
{
	uint64_t h = 0;
	for (unsigned i = 0; i < k; ++i)
		h ^= rol64(oracle_nt_seed((unsigned char)s[i]), k - 1 - i);
	return h;
}

uint64_t oracle_nt_reverse(const char *s, unsigned k)
{
	uint64_t h = 0;
	for (unsigned i = 0; i < k; ++i)
		h ^= rol64(oracle_nt_seed_rc((unsigned char)s[i]), i);
	return h;
}

uint64_t oracle_nt_extra(uint64_t canon, unsigned k, unsigned i)
{
	uint64_t t = canon * ((uint64_t)i ^ ((uint64_t)k * NT_MULTI_SEED));
	t ^= t >> NT_MULTI_SHIFT;
	return t;
}

static void ntitr_fill(oracle_ntitr *it)
{
	uint64_t c = it->fh < it->rh ? it->fh : it->rh;
	unsigned n = it->h < 64 ? it->h : 64;
	if (n == 0)
		return;
	it->hv[0] = c;
	for (unsigned i = 1; i < n; ++i)
		it->hv[i] = oracle_nt_extra(c, it->k, i);
}

/* Find the first k-mer at or after it->pos with no invalid base. */
static void ntitr_seek(oracle_ntitr *it)
{
	size_t p = it->pos;
	for (;;) {
		if (it->len < it->k || p > it->len - it->k) {
			it->pos = (size_t)-1;
			return;
		}
		size_t bad = (size_t)-1;
		for (size_t j = 0; j < it->k; ++j)
			if (!oracle_nt_valid((unsigned char)it->seq[p + j]))
				bad = p + j; /* keep the last invalid base */
		if (bad == (size_t)-1)
			break;
		p = bad + 1;
	}
	it->pos = p;
	it->fh = oracle_nt_forward(it->seq + p, it->k);
	it->rh = oracle_nt_reverse(it->seq + p, it->k);
	ntitr_fill(it);
}

/* ntHashIterator(seq, h, k) construction. */
void oracle_ntitr_init(oracle_ntitr *it, const char *seq, size_t len,
		unsigned h, unsigned k)
{
	memset(it, 0, sizeof(*it));
	it->seq = seq;
	it->len = len;
	it->k = k;
	it->h = h;
	it->pos = 0;
	if (k == 0) {
		it->pos = (size_t)-1;
		return;
	}
	ntitr_seek(it);
}

/* ntHashIterator::operator++: roll by one base, or re-seek past an invalid
 * incoming base. */
void oracle_ntitr_next(oracle_ntitr *it)
{
	if (it->pos == (size_t)-1)
		return;
	size_t p = it->pos + 1;
	if (p > it->len - it->k) {
		it->pos = (size_t)-1;
		return;
	}
	unsigned char in = (unsigned char)it->seq[p + it->k - 1];
	if (!oracle_nt_valid(in)) {
		it->pos = p + it->k; /* first start past the invalid base */
		ntitr_seek(it);
		return;
	}
	unsigned char out = (unsigned char)it->seq[p - 1];
	it->fh = rol64(it->fh, 1) ^ rol64(oracle_nt_seed(out), it->k)
			^ oracle_nt_seed(in);
	it->rh = ror64(it->rh, 1) ^ ror64(oracle_nt_seed_rc(out), 1)
			^ rol64(oracle_nt_seed_rc(in), it->k - 1);
	it->pos = p;
	ntitr_fill(it);
}

/* ------------------------------------------------------------------------ */
/* Bloom filter.  Bit j lives in byte j/8 at bit position j%8 (LSB first);   */
/* hash value v maps to bit v mod m; m is padded up to a multiple of 64 bits. */
/* ------------------------------------------------------------------------ */

int oracle_bf_create(oracle_bf *bf, uint64_t m, unsigned h, unsigned k)
{
	memset(bf, 0, sizeof(*bf));
	if (m % 64)
		m += 64 - m % 64;
	bf->m = m;
	bf->h = h;
	bf->k = k;
	bf->bits = (uint8_t *)calloc((size_t)(m / 8), 1);
	return bf->bits ? 0 : -1;
}

void oracle_bf_free(oracle_bf *bf)
{
	free(bf->bits);
	bf->bits = NULL;
}

int oracle_bf_contains(const oracle_bf *bf, const uint64_t *hv, uint64_t *probes)
{
	for (unsigned i = 0; i < bf->h; ++i) {
		uint64_t b = hv[i] % bf->m;
		if (probes)
			++*probes;
		if (!((bf->bits[b >> 3] >> (b & 7)) & 1))
			return 0;
	}
	return 1;
}

void oracle_bf_insert(oracle_bf *bf, const uint64_t *hv)
{
	for (unsigned i = 0; i < bf->h; ++i) {
		uint64_t b = hv[i] % bf->m;
		bf->bits[b >> 3] |= (uint8_t)(1u << (b & 7));
	}
}

int oracle_bf_insert_check(oracle_bf *bf, const uint64_t *hv)
{
	int found = 1;
	for (unsigned i = 0; i < bf->h; ++i) {
		uint64_t b = hv[i] % bf->m;
		uint8_t mask = (uint8_t)(1u << (b & 7));
		if (!(bf->bits[b >> 3] & mask)) {
			found = 0;
			bf->bits[b >> 3] |= mask;
		}
	}
	return found;
}

/*
 * .bf layout: a text header of "key = value" lines between "[BTLBloomFilter]"
 * and "[HeaderEnd]" (each line ends in '\n'), then the m/8 filter bytes.
 */
int oracle_bf_store(const oracle_bf *bf, const char *path)
{
	FILE *f = fopen(path, "wb");
	if (!f)
		return -1;
	fprintf(f, "[BTLBloomFilter]\nFormat = 1\nBloomFilterSize = %llu\n"
			"HashNum = %u\nKmerSize = %u\ndFPR = %.17g\nnEntry = %llu\n"
			"tEntry = %llu\n[HeaderEnd]\n",
			(unsigned long long)bf->m, bf->h, bf->k, bf->dfpr,
			(unsigned long long)bf->n_entry,
			(unsigned long long)bf->t_entry);
	size_t nb = (size_t)(bf->m / 8);
	int rc = fwrite(bf->bits, 1, nb, f) == nb ? 0 : -1;
	if (fclose(f))
		rc = -1;
	return rc;
}

int oracle_bf_load(oracle_bf *bf, const char *path)
{
	memset(bf, 0, sizeof(*bf));
	FILE *f = fopen(path, "rb");
	if (!f)
		return -1;
	char line[512];
	int in_header = 0, done = 0;
	unsigned long long m = 0, ne = 0, te = 0;
	unsigned h = 0, k = 0;
	double dfpr = 0;
	while (fgets(line, sizeof line, f)) {
		if (!in_header) {
			if (strcmp(line, "[BTLBloomFilter]\n"))
				break;
			in_header = 1;
			continue;
		}
		if (!strcmp(line, "[HeaderEnd]\n")) {
			done = 1;
			break;
		}
		sscanf(line, "BloomFilterSize = %llu", &m);
		sscanf(line, "HashNum = %u", &h);
		sscanf(line, "KmerSize = %u", &k);
		sscanf(line, "dFPR = %lf", &dfpr);
		sscanf(line, "nEntry = %llu", &ne);
		sscanf(line, "tEntry = %llu", &te);
	}
	if (!done || m == 0 || m % 64 || h == 0 || k == 0) {
		fclose(f);
		return -2;
	}
	bf->m = m;
	bf->h = h;
	bf->k = k;
	bf->dfpr = dfpr;
	bf->n_entry = ne;
	bf->t_entry = te;
	bf->bits = (uint8_t *)malloc((size_t)(m / 8));
	if (!bf->bits) {
		fclose(f);
		return -1;
	}
	size_t nb = (size_t)(m / 8);
	size_t got = fread(bf->bits, 1, nb, f);
	fclose(f);
	if (got != nb) {
		oracle_bf_free(bf);
		return -3;
	}
	return 0;
}

/* BloomFilterInfo::calcOptimalSize (Common/BloomFilterInfo.h:57-65). */
uint64_t oracle_calc_optimal_size(uint64_t entries, double fpr, unsigned h)
{
	uint64_t v = (uint64_t)(-(double)entries * (double)h
			/ log(1.0 - pow(fpr, (double)(1 / ((double)h)))));
	return v + (64 - v % 64);
}

/* BloomFilterInfo::calcOptimalHashNum (Common/BloomFilterInfo.h:73-76). */
unsigned oracle_calc_optimal_hash_num(double fpr)
{
	return (unsigned)(-log(fpr) / log(2));
}

/* BloomFilterGenerator::calcExpectedEntries + generate + loadFilter
 * (BioBloomMaker/BloomFilterGenerator.h:108-188, .cpp:54-73). */
int oracle_make_filter(oracle_bf *bf, const char *const *seqs,
		const uint64_t *lens, size_t n, unsigned k, double fpr, unsigned h,
		uint64_t *expected_entries, uint64_t *redundant)
{
	uint64_t expected = 0;
	for (size_t i = 0; i < n; ++i)
		expected += lens[i] - k + 1; /* size_t arithmetic, as upstream */
	if (h == 0)
		h = oracle_calc_optimal_hash_num(fpr);
	uint64_t m = oracle_calc_optimal_size(expected, fpr, h);
	if (oracle_bf_create(bf, m, h, k))
		return -1;
	bf->dfpr = fpr;
	uint64_t red = 0, tot = 0;
	for (size_t i = 0; i < n; ++i) {
		oracle_ntitr it;
		for (oracle_ntitr_init(&it, seqs[i], (size_t)lens[i], h, k);
				!oracle_ntitr_end(&it); oracle_ntitr_next(&it)) {
			int found = oracle_bf_insert_check(bf, it.hv);
			red += (uint64_t)found;
			tot += (uint64_t)!found;
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

/* BloomFilterInfo::printInfoFile layout (Common/BloomFilterInfo.cpp:81-116).
 * Doubles use the default ostream format, which is printf %g. */
int oracle_write_info(const char *path, const char *filter_id, unsigned k,
		double fpr, unsigned h, uint64_t expected, const char *sources,
		uint64_t size, uint64_t num_entries, double approx_fpr,
		uint64_t redundant, double redundant_fpr)
{
	FILE *f = fopen(path, "w");
	if (!f)
		return -1;
	fprintf(f, "[user_input_options]\nfilter_id=%s\nkmer_size=%u\n"
			"desired_false_positve_rate=%g\nnumber_of_hash_functions=%u\n"
			"expected_num_entries=%llu\nsequence_sources=%s \n\n"
			"[runtime_options]\nsize=%llu\nnum_entries=%llu\n"
			"approximate_false_positive_rate=%g\nredundant_sequences=%llu\n"
			"redundant_fpr=%g\n",
			filter_id, k, fpr, h, (unsigned long long)expected, sources,
			(unsigned long long)size, (unsigned long long)num_entries,
			approx_fpr, (unsigned long long)redundant, redundant_fpr);
	return fclose(f) ? -1 : 0;
}

/* ------------------------------------------------------------------------ */
/* SeqEval                                                                   */
/* ------------------------------------------------------------------------ */

/* ------------------------------------------------------------------------ */
/* SDUST low-complexity masking (-D)                                         */
/* ------------------------------------------------------------------------ */

/*
 * The symmetric DUST algorithm (Morgulis et al., "A fast and symmetric DUST
 * implementation to mask low-complexity DNA sequences", J Comput Biol 2006)
 * as the reference runs it: Common/sdust.c (sdust_core, shift_window,
 * find_perfect, save_masked_regions), called once per evaluated read by
 * Common/SDust.hpp with T = opt::dustT (20) and W = opt::dustWindow (64).
 *
 * Words are the triplets of consecutive A/C/G/T bases (any case).  The
 * window holds the last W - 2 triplets; for a set of triplets the score is
 * sum over triplet kinds of c(c-1)/2.  cw / rw count the whole window; cv /
 * rv count its longest suffix of L triplets in which no triplet kind occurs
 * more than 2T/10 times.  When 10 rw > L T the window may hold "perfect
 * intervals": suffixes whose score r over length l has 10 r > T l and is at
 * least that of every perfect interval starting inside them; those are kept,
 * by descending start, in `perf`.  A perfect interval whose start falls out of
 * the window is saved as masked, merged with the previous masked interval if
 * they touch.  A non-ACGT base (and the end of the read) flushes all pending
 * perfect intervals, but does not empty the window.
 */
typedef struct {
	int start, finish, r, l;
} dust_perfect;

typedef struct {
	int T, W;
	int *ring;             /* window triplets, oldest first */
	size_t head, size, cap;
	int cw[64], cv[64];
	int rw, rv, L;
	dust_perfect *perf;    /* by descending start, then ascending finish */
	size_t np, pcap;
	uint64_t *res;         /* masked intervals: start << 32 | finish (exclusive) */
	size_t nres, rcap;
	size_t max_np;         /* largest perf size seen (capacity studies) */
} dust_state;

static int dust_code(unsigned char c)
{
	switch (c) {
	case 'A': case 'a': return 0;
	case 'C': case 'c': return 1;
	case 'G': case 'g': return 2;
	case 'T': case 't': return 3;
	default: return 4;
	}
}

static int dust_at(const dust_state *d, size_t i)
{
	return d->ring[(d->head + i) % d->cap];
}

static void dust_save(dust_state *d, int start)
{
	if (d->np == 0 || d->perf[d->np - 1].start >= start)
		return;
	const dust_perfect *p = &d->perf[d->np - 1];
	int merged = 0;
	if (d->nres) {
		const int s = (int)(d->res[d->nres - 1] >> 32);
		const int f = (int)(uint32_t)d->res[d->nres - 1];
		if (p->start <= f) {
			merged = 1;
			d->res[d->nres - 1] = (uint64_t)s << 32 | (uint64_t)(f > p->finish ? f : p->finish);
		}
	}
	if (!merged) {
		if (d->nres == d->rcap) {
			d->rcap = d->rcap ? 2 * d->rcap : 16;
			d->res = (uint64_t *)realloc(d->res, d->rcap * sizeof(uint64_t));
		}
		d->res[d->nres++] = (uint64_t)p->start << 32 | (uint64_t)p->finish;
	}
	long i = (long)d->np - 1;
	while (i >= 0 && d->perf[i].start < start)
		--i;
	d->np = (size_t)(i + 1);
}

static void dust_shift(dust_state *d, int t)
{
	if ((int)d->size >= d->W - 2) {
		const int s = d->ring[d->head];
		d->head = (d->head + 1) % d->cap;
		--d->size;
		d->rw -= --d->cw[s];
		if (d->L > (int)d->size) {
			--d->L;
			d->rv -= --d->cv[s];
		}
	}
	d->ring[(d->head + d->size) % d->cap] = t;
	++d->size;
	++d->L;
	d->rw += d->cw[t]++;
	d->rv += d->cv[t]++;
	if (d->cv[t] * 10 > d->T * 2) {
		int s;
		do {
			s = dust_at(d, d->size - (size_t)d->L);
			d->rv -= --d->cv[s];
			--d->L;
		} while (s != t);
	}
}

static void dust_find_perfect(dust_state *d, int start)
{
	int c[64];
	memcpy(c, d->cv, sizeof c);
	int r = d->rv, max_r = 0, max_l = 0;
	for (long i = (long)d->size - d->L - 1; i >= 0; --i) {
		const int t = dust_at(d, (size_t)i);
		r += c[t]++;
		const int new_r = r, new_l = (int)((long)d->size - i - 1);
		if (new_r * 10 <= d->T * new_l)
			continue;
		size_t j = 0;
		for (; j < d->np && d->perf[j].start >= (int)i + start; ++j) {
			const dust_perfect *p = &d->perf[j];
			if (max_r == 0 || p->r * max_l > max_r * p->l) {
				max_r = p->r;
				max_l = p->l;
			}
		}
		if (max_r == 0 || new_r * max_l >= max_r * new_l) {
			max_r = new_r;
			max_l = new_l;
			if (d->np == d->pcap) {
				d->pcap = d->pcap ? 2 * d->pcap : 16;
				d->perf = (dust_perfect *)realloc(d->perf, d->pcap * sizeof(dust_perfect));
			}
			memmove(d->perf + j + 1, d->perf + j, (d->np - j) * sizeof(dust_perfect));
			++d->np;
			d->perf[j].start = (int)i + start;
			d->perf[j].finish = (int)d->size + 2 + start;
			d->perf[j].r = new_r;
			d->perf[j].l = new_l;
			if (d->np > d->max_np)
				d->max_np = d->np;
		}
	}
}

static void dust_run(dust_state *d, const char *seq, int len)
{
	int l = 0;
	unsigned t = 0;
	for (int i = 0; i <= len; ++i) {
		const int b = i < len ? dust_code((unsigned char)seq[i]) : 4;
		if (b < 4) {
			++l;
			t = (t << 2 | (unsigned)b) & 63u;
			if (l >= 3) {
				const int start = (l - d->W > 0 ? l - d->W : 0) + (i + 1 - l);
				dust_save(d, start);
				dust_shift(d, (int)t);
				if (d->rw * 10 > d->L * d->T)
					dust_find_perfect(d, start);
			}
		} else {
			int start = (l - d->W + 1 > 0 ? l - d->W + 1 : 0) + (i + 1 - l);
			while (d->np)
				dust_save(d, start++);
			l = 0;
			t = 0;
		}
	}
}

static void dust_free(dust_state *d)
{
	free(d->ring);
	free(d->perf);
	free(d->res);
}

int oracle_sdust(const char *seq, size_t len, int T, int W, uint64_t *out, int cap,
		int *max_perfect)
{
	dust_state d;
	memset(&d, 0, sizeof d);
	d.T = T;
	d.W = W;
	d.cap = W > 3 ? (size_t)W : 4;
	d.ring = (int *)malloc(d.cap * sizeof(int));
	dust_run(&d, seq, (int)len);
	int n = (int)d.nres;
	for (int i = 0; i < n && i < cap; ++i)
		out[i] = d.res[i];
	if (max_perfect)
		*max_perfect = (int)d.max_np;
	dust_free(&d);
	return n;
}

/* -D: SeqEval's evaluation functions treat a frame whose start lies in a
 * masked interval as a miss without probing the filter (the
 * sduster->isLowComp(itr.pos()) test, Common/SeqEval.h:53,78,...). */
static int g_dust = 0, g_dust_T = 20, g_dust_W = 64;

void oracle_set_dust(int on, int T, int W)
{
	g_dust = on != 0;
	g_dust_T = T;
	g_dust_W = W;
}

/* SDust (Common/SDust.hpp): the masked intervals of one read and a cursor
 * that only moves forward, as isLowComp assumes increasing positions. */
typedef struct {
	uint64_t *iv;
	int n, cur;
} dust_mask;

static void dust_mask_init(dust_mask *m, const char *seq, size_t len)
{
	m->iv = NULL;
	m->n = 0;
	m->cur = 0;
	if (!g_dust)
		return;
	dust_state d;
	memset(&d, 0, sizeof d);
	d.T = g_dust_T;
	d.W = g_dust_W;
	d.cap = g_dust_W > 3 ? (size_t)g_dust_W : 4;
	d.ring = (int *)malloc(d.cap * sizeof(int));
	dust_run(&d, seq, (int)len);
	m->iv = d.res;
	m->n = (int)d.nres;
	d.res = NULL;
	dust_free(&d);
}

static int dust_low(dust_mask *m, size_t pos)
{
	const unsigned p = (unsigned)pos;
	while (m->cur < m->n && p >= (unsigned)m->iv[m->cur])
		++m->cur;
	return m->cur < m->n && p >= (unsigned)(m->iv[m->cur] >> 32) &&
			p < (unsigned)m->iv[m->cur];
}

/* A frame's hit: not masked, and in the filter. */
static int frame_hit(const oracle_bf *bf, const oracle_ntitr *it, dust_mask *m, uint64_t *probes)
{
	if (m->n && dust_low(m, it->pos))
		return 0;
	return oracle_bf_contains(bf, it->hv, probes);
}

/* SeqEval::evalSimple (Common/SeqEval.h:37-114), without dust/subtract. */
static int oracle_eval_simple_impl(dust_mask *dm, const char *seq, size_t len, const oracle_bf *bf,
		double threshold, unsigned streak_threshold, uint64_t *probes)
{
	const size_t frames = len - bf->k + 1; /* size_t arithmetic, as upstream */
	const double thres = threshold * (double)frames;
	const double anti_thres = floor((1.0 - threshold) * (double)frames);
	double score = 0;
	unsigned anti = 0, streak = 0, prev = 0;
	oracle_ntitr it;
	oracle_ntitr_init(&it, seq, len, bf->k, bf->k);
	if (!oracle_ntitr_end(&it)) {
		if (frame_hit(bf, &it, dm, probes)) {
			score += 0.5;
			if (thres <= score)
				return 1;
			++streak;
		} else {
			if (anti_thres <= ++anti)
				return 0;
		}
		prev = (unsigned)it.pos;
		oracle_ntitr_next(&it);
	}
	while (!oracle_ntitr_end(&it)) {
		if (it.pos != (size_t)prev + 1) {
			anti += (unsigned)(it.pos - prev - 1);
			if (anti_thres <= anti)
				return 0;
			streak = 0;
		}
		if (frame_hit(bf, &it, dm, probes)) {
			if (streak == 0)
				score += 0.5;
			else
				score += 1.0;
			if (thres <= score)
				return 1;
			prev = (unsigned)it.pos;
			oracle_ntitr_next(&it);
			++streak;
		} else {
			if (streak < streak_threshold) {
				if (anti_thres <= ++anti)
					return 0;
				prev = (unsigned)it.pos;
				oracle_ntitr_next(&it);
			} else {
				unsigned skip_end = (unsigned)it.pos + bf->k;
				/* the end state has pos SIZE_MAX, which ends the window */
				while (it.pos < skip_end) {
					if (anti_thres <= ++anti)
						return 0;
					prev = (unsigned)it.pos;
					oracle_ntitr_next(&it);
				}
			}
			streak = 0;
		}
	}
	return 0;
}

int oracle_eval_simple(const char *seq, size_t len, const oracle_bf *bf,
		double threshold, unsigned streak_threshold, uint64_t *probes)
{
	dust_mask dm;
	dust_mask_init(&dm, seq, len);
	int v = oracle_eval_simple_impl(&dm, seq, len, bf, threshold, streak_threshold, probes);
	free(dm.iv);
	return v;
}

/* SeqEval::evalHarmonic (Common/SeqEval.h:116-193), without dust/subtract:
 * evalSimple's walk, with a hit in a streak of s earlier hits adding
 * 1 - 1/(1 + s) instead of 1. */
static int oracle_eval_harmonic_impl(dust_mask *dm, const char *seq, size_t len, const oracle_bf *bf,
		double threshold, unsigned streak_threshold, uint64_t *probes)
{
	const size_t frames = len - bf->k + 1; /* size_t arithmetic, as upstream */
	const double thres = threshold * (double)frames;
	const double anti_thres = floor((1.0 - threshold) * (double)frames);
	double score = 0;
	unsigned anti = 0, streak = 0, prev = 0;
	oracle_ntitr it;
	oracle_ntitr_init(&it, seq, len, bf->k, bf->k);
	if (!oracle_ntitr_end(&it)) {
		if (frame_hit(bf, &it, dm, probes)) {
			score += 0.5;
			if (thres <= score)
				return 1;
			++streak;
		} else {
			if (anti_thres <= ++anti)
				return 0;
		}
		prev = (unsigned)it.pos;
		oracle_ntitr_next(&it);
	}
	while (!oracle_ntitr_end(&it)) {
		if (it.pos != (size_t)prev + 1) {
			anti += (unsigned)(it.pos - prev - 1);
			if (anti_thres <= anti)
				return 0;
			streak = 0;
		}
		if (frame_hit(bf, &it, dm, probes)) {
			if (streak == 0)
				score += 0.5;
			else
				score += 1.0 - 1.0 / (1.0 + (double)streak);
			if (thres <= score)
				return 1;
			prev = (unsigned)it.pos;
			oracle_ntitr_next(&it);
			++streak;
		} else {
			if (streak < streak_threshold) {
				if (anti_thres <= ++anti)
					return 0;
				prev = (unsigned)it.pos;
				oracle_ntitr_next(&it);
			} else {
				unsigned skip_end = (unsigned)it.pos + bf->k;
				while (it.pos < skip_end) {
					if (anti_thres <= ++anti)
						return 0;
					prev = (unsigned)it.pos;
					oracle_ntitr_next(&it);
				}
			}
			streak = 0;
		}
	}
	return 0;
}

int oracle_eval_harmonic(const char *seq, size_t len, const oracle_bf *bf,
		double threshold, unsigned streak_threshold, uint64_t *probes)
{
	dust_mask dm;
	dust_mask_init(&dm, seq, len);
	int v = oracle_eval_harmonic_impl(&dm, seq, len, bf, threshold, streak_threshold, probes);
	free(dm.iv);
	return v;
}

/* BloomFilter::getFPRPrecompute as restated: (set bits / m) ^ h. */
double oracle_bf_fpr(const oracle_bf *bf)
{
	uint64_t pop = 0;
	for (uint64_t i = 0; i < bf->m / 8; ++i)
		pop += (uint64_t)__builtin_popcount(bf->bits[i]);
	return pow((double)pop / (double)bf->m, (double)bf->h);
}

/* P(X > x) summed from the top of the tail down, and the smallest x with
 * P(X > x) <= q. */
static double binom_pmf(double n, double p, double i)
{
	if (p <= 0.0)
		return i == 0 ? 1.0 : 0.0;
	if (p >= 1.0)
		return i == n ? 1.0 : 0.0;
	return exp(lgamma(n + 1) - lgamma(i + 1) - lgamma(n - i + 1) + i * log(p) +
			(n - i) * log1p(-p));
}

unsigned oracle_binom_upper_quantile(unsigned n, double p, double q)
{
	double x = n, tail = 0.0;
	while (x > 0) {
		double t = tail + binom_pmf(n, p, x);
		if (t > q)
			break;
		tail = t;
		x -= 1.0;
	}
	return (unsigned)x;
}

/* SeqEval::calcMinCount (Common/SeqEval.h:199-207). */
unsigned oracle_calc_min_count(unsigned frame_len, double bf_fpr, double min_fpr)
{
	unsigned i = oracle_binom_upper_quantile(frame_len, bf_fpr, min_fpr);
	return i > 1 ? i : 1;
}

/* SeqEval::evalBinomial (Common/SeqEval.h:218-290), without dust/subtract:
 * every hit adds 1; accept at calcMinCount hits, reject at frameLen minus that
 * many misses.  fpr = the filter's getFPRPrecompute(). */
static int oracle_eval_binomial_impl(dust_mask *dm, const char *seq, size_t len, const oracle_bf *bf,
		double threshold, double fpr, unsigned streak_threshold, uint64_t *probes)
{
	if (len < bf->k)
		return 0;
	const unsigned frame_len = (unsigned)(len - bf->k + 1);
	const unsigned thres = oracle_calc_min_count(frame_len, fpr, threshold);
	const unsigned anti_thres = frame_len - thres;
	unsigned score = 0, anti = 0, streak = 0, prev = 0;
	oracle_ntitr it;
	oracle_ntitr_init(&it, seq, len, bf->k, bf->k);
	if (!oracle_ntitr_end(&it)) {
		if (frame_hit(bf, &it, dm, probes)) {
			score++;
			if (thres <= score)
				return 1;
			++streak;
		} else {
			if (anti_thres <= ++anti)
				return 0;
		}
		prev = (unsigned)it.pos;
		oracle_ntitr_next(&it);
	}
	while (!oracle_ntitr_end(&it)) {
		if (it.pos != (size_t)prev + 1) {
			anti += (unsigned)(it.pos - prev - 1);
			if (anti_thres <= anti)
				return 0;
			streak = 0;
		}
		if (frame_hit(bf, &it, dm, probes)) {
			++score;
			if (thres <= score)
				return 1;
			prev = (unsigned)it.pos;
			oracle_ntitr_next(&it);
			++streak;
		} else {
			if (streak < streak_threshold) {
				if (anti_thres <= ++anti)
					return 0;
				prev = (unsigned)it.pos;
				oracle_ntitr_next(&it);
			} else {
				unsigned skip_end = (unsigned)it.pos + bf->k;
				while (it.pos < skip_end) {
					if (anti_thres <= ++anti)
						return 0;
					prev = (unsigned)it.pos;
					oracle_ntitr_next(&it);
				}
			}
			streak = 0;
		}
	}
	return 0;
}

int oracle_eval_binomial(const char *seq, size_t len, const oracle_bf *bf,
		double threshold, double fpr, unsigned streak_threshold, uint64_t *probes)
{
	dust_mask dm;
	dust_mask_init(&dm, seq, len);
	int v = oracle_eval_binomial_impl(&dm, seq, len, bf, threshold, fpr, streak_threshold, probes);
	free(dm.iv);
	return v;
}

/* SeqEval::evalMinMatchLen (Common/SeqEval.h:295-332), without
 * dust/subtract.  The iterator is built with getHashNum() hashes. */
static int oracle_eval_min_match_len_impl(dust_mask *dm, const char *seq, size_t len,
		const oracle_bf *bf, unsigned min_match_len, uint64_t *probes)
{
	unsigned match = 0, prev = 0;
	oracle_ntitr it;
	for (oracle_ntitr_init(&it, seq, len, bf->h, bf->k);
			!oracle_ntitr_end(&it); oracle_ntitr_next(&it)) {
		if (len - it.pos + match < min_match_len)
			return 0;
		if (it.pos != (size_t)prev + 1)
			match = 0;
		if (frame_hit(bf, &it, dm, probes)) {
			if (match == 0)
				match = bf->k;
			else
				++match;
		} else {
			match = 0;
		}
		if (match >= min_match_len)
			return 1;
		prev = (unsigned)it.pos;
	}
	return 0;
}

int oracle_eval_min_match_len(const char *seq, size_t len,
		const oracle_bf *bf, unsigned min_match_len, uint64_t *probes)
{
	dust_mask dm;
	dust_mask_init(&dm, seq, len);
	int v = oracle_eval_min_match_len_impl(&dm, seq, len, bf, min_match_len, probes);
	free(dm.iv);
	return v;
}

/* ------------------------------------------------------------------------ */
/* Batch driver and summary                                                  */
/* ------------------------------------------------------------------------ */

/* BioBloomClassifier::evaluateReadStd (BioBloomClassifier.cpp:1182-1189). */
/* boost's cdf(complement(binomial(n, p), x)) = P(X > x), summed from the top
 * of the tail down (SeqEval::calcProbMatches, Common/SeqEval.h:209-216). */
double oracle_binom_sf(unsigned n, double p, unsigned x)
{
	double tail = 0.0;
	for (double i = n; i > (double)x; i -= 1.0)
		tail += binom_pmf(n, p, i);
	return tail;
}

/* SeqEval::evalScore (Common/SeqEval.h:534-560), without dust/subtract:
 * evalSimpleScore (:334-376), evalHarmonicScore (:378-419),
 * evalMinMatchLenScore (:421-448) and evalBinomialScore (:450-491) followed by
 * log10(...) * -10.  fpr is the filter's getFPRPrecompute (BINOMIAL only). */
static double oracle_eval_score_impl(dust_mask *dm, const char *seq, size_t len, const oracle_bf *bf, int scoring,
		unsigned streak_threshold, double fpr)
{
	oracle_ntitr it;
	if (scoring == ORACLE_LENGTH) {
		unsigned match_len = 0, prev = 0;
		oracle_ntitr_init(&it, seq, len, bf->h, bf->k);
		while (!oracle_ntitr_end(&it)) {
			if (it.pos != (size_t)prev + 1)
				match_len = 0;
			if (frame_hit(bf, &it, dm, NULL))
				match_len = match_len == 0 ? bf->k : match_len + 1;
			else
				match_len = 0;
			prev = (unsigned)it.pos;
			oracle_ntitr_next(&it);
		}
		return (double)match_len;
	}
	if (scoring == ORACLE_BINOMIAL && len < bf->k)
		return log10(1.0) * -10;
	double score = 0;
	unsigned streak = 0, prev = 0;
	oracle_ntitr_init(&it, seq, len, bf->k, bf->k);
	while (!oracle_ntitr_end(&it)) {
		if (it.pos != (size_t)prev + 1)
			streak = 0;
		if (frame_hit(bf, &it, dm, NULL)) {
			if (scoring == ORACLE_BINOMIAL)
				score += 1;
			else if (streak == 0)
				score += 0.5;
			else if (scoring == ORACLE_HARMONIC)
				score += 1.0 - 1.0 / (1.0 + (double)streak);
			else
				score += 1;
			prev = (unsigned)it.pos;
			oracle_ntitr_next(&it);
			++streak;
		} else {
			if (streak < streak_threshold) {
				prev = (unsigned)it.pos;
				oracle_ntitr_next(&it);
			} else {
				unsigned skip_end = (unsigned)it.pos + bf->k;
				while (it.pos < skip_end) {
					prev = (unsigned)it.pos;
					oracle_ntitr_next(&it);
				}
			}
			streak = 0;
		}
	}
	if (scoring == ORACLE_BINOMIAL) {
		const unsigned frame_len = (unsigned)(len - bf->k + 1);
		return log10(oracle_binom_sf(frame_len, fpr, (unsigned)score)) * -10;
	}
	/* normalizeScore (:33-35): the divisor in size_t arithmetic */
	return score / (double)(len - bf->k + 1);
}

double oracle_eval_score(const char *seq, size_t len, const oracle_bf *bf, int scoring,
		unsigned streak_threshold, double fpr)
{
	dust_mask dm;
	dust_mask_init(&dm, seq, len);
	double v = oracle_eval_score_impl(&dm, seq, len, bf, scoring, streak_threshold, fpr);
	free(dm.iv);
	return v;
}

void oracle_classify_scores(const char *seq, const uint64_t *off, size_t n,
		const oracle_bf *const *filters, unsigned nf, int scoring,
		unsigned streak_threshold, double *scores)
{
	double fpr[1024];
	for (unsigned f = 0; f < nf && f < 1024; ++f)
		fpr[f] = scoring == ORACLE_BINOMIAL ? oracle_bf_fpr(filters[f]) : 0.0;
	for (size_t r = 0; r < n; ++r) {
		const char *s = seq + off[r];
		size_t len = (size_t)(off[r + 1] - off[r]);
		for (unsigned f = 0; f < nf && f < 1024; ++f)
			scores[r * nf + f] = oracle_eval_score(s, len, filters[f], scoring,
					streak_threshold, fpr[f]);
	}
}

/* BioBloomClassifier::evaluateReadBestHit (BioBloomClassifier.cpp:1194-1218)
 * over one read's scores: the filters of the largest score (a larger score
 * replaces the list, an equal one joins it), kept only when that score is
 * above 0.  Returns the largest score (0 when none is above 0). */
double oracle_best_hit(const double *scores, unsigned nf, uint64_t *hits)
{
	unsigned words = (nf + 63) / 64;
	double max_score = 0;
	memset(hits, 0, words * sizeof(uint64_t));
	for (unsigned f = 0; f < nf; ++f) {
		double sc = scores[f];
		if (max_score < sc) {
			max_score = sc;
			memset(hits, 0, words * sizeof(uint64_t));
			hits[f >> 6] |= 1ULL << (f & 63);
		} else if (max_score == sc) {
			hits[f >> 6] |= 1ULL << (f & 63);
		}
	}
	if (!(max_score > 0))
		memset(hits, 0, words * sizeof(uint64_t));
	return max_score;
}

/* evaluateReadOrdered / evaluateReadOrderedPair (BioBloomClassifier.cpp:
 * 1145-1180) from the STD hit words: the first filter the read passes (pairs:
 * that both mates pass, or either with inclusive) is the only hit, of both
 * mates.  hits2 may be NULL (single end). */
void oracle_ordered(uint64_t *hits1, uint64_t *hits2, unsigned nf, int inclusive)
{
	unsigned words = (nf + 63) / 64, f = nf;
	for (unsigned i = 0; i < nf; ++i) {
		int a = (int)((hits1[i >> 6] >> (i & 63)) & 1);
		int pass = a;
		if (hits2) {
			int b = (int)((hits2[i >> 6] >> (i & 63)) & 1);
			pass = inclusive ? (a || b) : (a && b);
		}
		if (pass) {
			f = i;
			break;
		}
	}
	memset(hits1, 0, words * sizeof(uint64_t));
	if (hits2)
		memset(hits2, 0, words * sizeof(uint64_t));
	if (f < nf) {
		hits1[f >> 6] |= 1ULL << (f & 63);
		if (hits2)
			hits2[f >> 6] |= 1ULL << (f & 63);
	}
}

void oracle_classify(const char *seq, const uint64_t *off, size_t n,
		const oracle_bf *const *filters, unsigned nf, double threshold,
		unsigned streak_threshold, int scoring, uint64_t *hits,
		uint64_t *probes)
{
	unsigned words = (nf + 63) / 64;
	double fpr[1024];
	if (scoring == ORACLE_BINOMIAL)
		for (unsigned f = 0; f < nf && f < 1024; ++f)
			fpr[f] = oracle_bf_fpr(filters[f]);
	for (size_t r = 0; r < n; ++r) {
		const char *s = seq + off[r];
		size_t len = (size_t)(off[r + 1] - off[r]);
		uint64_t *hr = hits + r * words;
		memset(hr, 0, words * sizeof(uint64_t));
		for (unsigned f = 0; f < nf; ++f) {
			int hit;
			if (scoring == ORACLE_LENGTH)
				hit = oracle_eval_min_match_len(s, len, filters[f],
						(unsigned)round(threshold), probes);
			else if (scoring == ORACLE_HARMONIC)
				hit = oracle_eval_harmonic(s, len, filters[f], threshold,
						streak_threshold, probes);
			else if (scoring == ORACLE_BINOMIAL)
				hit = oracle_eval_binomial(s, len, filters[f], threshold, fpr[f],
						streak_threshold, probes);
			else
				hit = oracle_eval_simple(s, len, filters[f], threshold,
						streak_threshold, probes);
			if (hit)
				hr[f >> 6] |= 1ULL << (f & 63);
		}
	}
}

/* counts layout: above[nf+2] | unique[nf+2] | multi | noMatch */
static unsigned summary_finish(uint64_t *counts, unsigned nf, unsigned idx)
{
	uint64_t *unique = counts + (nf + 2);
	if (idx == nf)
		++counts[2 * (nf + 2) + 1];
	else if (idx == nf + 1)
		++counts[2 * (nf + 2)];
	else
		++unique[idx];
	return idx;
}

/* ResultsManager::updateSummaryData(hits) (ResultsManager.hpp:66-89). */
unsigned oracle_update_summary(uint64_t *counts, unsigned nf,
		const uint64_t *hits)
{
	unsigned idx = nf;
	for (unsigned f = 0; f < nf; ++f) {
		if (!((hits[f >> 6] >> (f & 63)) & 1))
			continue;
		++counts[f];
		idx = idx == nf ? f : nf + 1;
	}
	return summary_finish(counts, nf, idx);
}

/* ResultsManager::updateSummaryData(hits1, hits2) (ResultsManager.hpp:91-189):
 * inclusive counts the union of the two ascending hit lists, the default
 * counts their intersection. */
unsigned oracle_update_summary_pair(uint64_t *counts, unsigned nf,
		const uint64_t *hits1, const uint64_t *hits2, int inclusive)
{
	unsigned idx = nf;
	for (unsigned f = 0; f < nf; ++f) {
		int a = (int)((hits1[f >> 6] >> (f & 63)) & 1);
		int b = (int)((hits2[f >> 6] >> (f & 63)) & 1);
		if (inclusive ? (a || b) : (a && b)) {
			++counts[f];
			idx = idx == nf ? f : nf + 1;
		}
	}
	return summary_finish(counts, nf, idx);
}

/* ResultsManager::getResultsSummary (ResultsManager.hpp:191-237). */
size_t oracle_summary_tsv(const uint64_t *counts, unsigned nf,
		const char *const *ids, uint64_t read_count, char *out, size_t cap)
{
	const uint64_t *above = counts;
	const uint64_t *unique = counts + (nf + 2);
	uint64_t multi = counts[2 * (nf + 2)];
	uint64_t nomatch = counts[2 * (nf + 2) + 1];
	double rc = (double)read_count;
	size_t len = 0;
	char line[1024];
#define EMIT(...) do { \
		int w = snprintf(line, sizeof line, __VA_ARGS__); \
		if (out && len + (size_t)w < cap) memcpy(out + len, line, (size_t)w + 1); \
		len += (size_t)w; \
	} while (0)
	EMIT("filter_id\thits\tmisses\tshared\trate_hit\trate_miss\trate_shared\n");
	for (unsigned i = 0; i < nf; ++i) {
		uint64_t a = above[i], u = unique[i];
		EMIT("%s\t%llu\t%llu\t%llu\t%g\t%g\t%g\n", ids[i],
				(unsigned long long)a, (unsigned long long)(read_count - a),
				(unsigned long long)(a - u), (double)a / rc,
				(double)(read_count - a) / rc, (double)(a - u) / rc);
	}
	EMIT("multiMatch\t%llu\t%llu\t0\t%g\t%g\t0\n", (unsigned long long)multi,
			(unsigned long long)(read_count - multi), (double)multi / rc,
			(double)(read_count - multi) / rc);
	EMIT("noMatch\t%llu\t%llu\t0\t%g\t%g\t0\n", (unsigned long long)nomatch,
			(unsigned long long)(read_count - nomatch), (double)nomatch / rc,
			(double)(read_count - nomatch) / rc);
#undef EMIT
	return len;
}
