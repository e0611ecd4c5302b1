/*
 * mibf_oracle.c -- CPU oracle for the miBF path (test infrastructure only;
 * the restated semantics are spelled out in mibf_oracle.h).
 */
#include "mibf_oracle.h"
#include "bbt_oracle.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

static inline uint64_t rol64(uint64_t v, unsigned s)
{
	s &= 63u;
	return s ? (v << s) | (v >> (64u - s)) : v;
}

static inline uint64_t mix64(uint64_t z)
{
	z += 0x9e3779b97f4a7c15ULL;
	z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
	z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
	return z ^ (z >> 31);
}

uint64_t oracle_st_hash(const char *seed, unsigned k, const char *x)
{
	uint64_t f = 0, r = 0;
	for (unsigned j = 0; j < k; ++j) {
		if (seed[j] != '1')
			continue;
		f ^= rol64(oracle_nt_seed((unsigned char)x[j]), k - 1 - j);
		r ^= rol64(oracle_nt_seed_rc((unsigned char)x[j]), j);
	}
	return f < r ? f : r;
}

int oracle_mibf_frame_ok(const oracle_mibf *f, const char *x)
{
	for (unsigned j = 0; j < f->k; ++j)
		if (!oracle_nt_valid((unsigned char)x[j]))
			return 0;
	return 1;
}

void oracle_mibf_values(const oracle_mibf *f, const char *x, uint64_t *out)
{
	if (f->nseeds) {
		for (unsigned i = 0; i < f->nseeds; ++i)
			out[i] = oracle_st_hash(f->seeds[i], f->k, x);
		return;
	}
	uint64_t fw = oracle_nt_forward(x, f->k), rv = oracle_nt_reverse(x, f->k);
	uint64_t c = fw < rv ? fw : rv;
	out[0] = c;
	for (unsigned i = 1; i < f->h; ++i)
		out[i] = oracle_nt_extra(c, f->k, i);
}

static inline int bit_set(const oracle_mibf *f, uint64_t p)
{
	return (int)((f->bv[p >> 6] >> (p & 63)) & 1u);
}

uint64_t oracle_mibf_rank(const oracle_mibf *f, uint64_t p)
{
	uint64_t w = f->bv[p >> 6] & ((p & 63) ? ((1ull << (p & 63)) - 1) : 0);
	return f->rank_word[p >> 6] + (uint64_t)__builtin_popcountll(w);
}

static void build_rank(oracle_mibf *f)
{
	uint64_t words = f->m / 64, acc = 0;
	f->rank_word = (uint64_t *)malloc((words + 1) * sizeof(uint64_t));
	for (uint64_t w = 0; w < words; ++w) {
		f->rank_word[w] = acc;
		acc += (uint64_t)__builtin_popcountll(f->bv[w]);
	}
	f->rank_word[words] = acc;
	f->pop = acc;
}

static uint16_t priority(uint64_t slot, unsigned id)
{
	return (uint16_t)(mix64(slot ^ ((uint64_t)id * 0x9e3779b97f4a7c15ULL)) >> 48);
}

/* MIBFGen::generate / generateBV (BioBloomMaker/MIBFGen.hpp:131-415),
 * restated as three order-free passes. */
int oracle_mibf_build(oracle_mibf *f, const char *const *seqs, const uint64_t *lens,
		const uint16_t *seq_id, size_t n, const char *const *seeds, unsigned nseeds,
		unsigned k, unsigned h, double occupancy)
{
	memset(f, 0, sizeof(*f));
	if (nseeds > ORACLE_MIBF_MAX_SEEDS || k == 0 || k > 255)
		return -1;
	f->k = k;
	f->nseeds = nseeds;
	f->h = nseeds ? nseeds : h;
	for (unsigned i = 0; i < nseeds; ++i) {
		if (strlen(seeds[i]) != k)
			return -1;
		strcpy(f->seeds[i], seeds[i]);
	}
	uint64_t expected = 0;
	for (size_t i = 0; i < n; ++i)
		expected += lens[i] - k + 1; /* size_t arithmetic, as upstream */
	double mb = ceil((double)expected * f->h / -log(1.0 - occupancy));
	uint64_t m = (uint64_t)mb;
	m += (64 - m % 64) % 64;
	if (m == 0)
		m = 64;
	f->m = m;
	f->bv = (uint64_t *)calloc(m / 64, sizeof(uint64_t));
	if (!f->bv)
		return -2;
	uint64_t vals[ORACLE_MIBF_MAX_SEEDS > 64 ? ORACLE_MIBF_MAX_SEEDS : 64];
	/* pass 1: bit vector */
	for (size_t i = 0; i < n; ++i) {
		if (lens[i] < k)
			continue;
		for (uint64_t q = 0; q + k <= lens[i]; ++q) {
			if (!oracle_mibf_frame_ok(f, seqs[i] + q))
				continue;
			oracle_mibf_values(f, seqs[i] + q, vals);
			for (unsigned v = 0; v < f->h; ++v) {
				uint64_t p = vals[v] % m;
				f->bv[p >> 6] |= 1ull << (p & 63);
			}
		}
	}
	build_rank(f);
	/* pass 2: slot owners */
	uint32_t *best = (uint32_t *)calloc(f->pop ? f->pop : 1, sizeof(uint32_t));
	f->ids = (uint16_t *)calloc(f->pop ? f->pop : 1, sizeof(uint16_t));
	if (!best || !f->ids)
		return -2;
	for (size_t i = 0; i < n; ++i) {
		if (lens[i] < k)
			continue;
		for (uint64_t q = 0; q + k <= lens[i]; ++q) {
			if (!oracle_mibf_frame_ok(f, seqs[i] + q))
				continue;
			oracle_mibf_values(f, seqs[i] + q, vals);
			for (unsigned v = 0; v < f->h; ++v) {
				uint64_t slot = oracle_mibf_rank(f, vals[v] % m);
				uint32_t cand = ((uint32_t)priority(slot, seq_id[i]) << 16) | seq_id[i];
				if (cand > best[slot])
					best[slot] = cand;
			}
		}
	}
	for (uint64_t s = 0; s < f->pop; ++s)
		f->ids[s] = (uint16_t)(best[s] & 0xFFFF);
	free(best);
	/* pass 3: saturation */
	for (size_t i = 0; i < n; ++i) {
		if (lens[i] < k)
			continue;
		for (uint64_t q = 0; q + k <= lens[i]; ++q) {
			if (!oracle_mibf_frame_ok(f, seqs[i] + q))
				continue;
			oracle_mibf_values(f, seqs[i] + q, vals);
			uint64_t slots[64];
			int owned = 0;
			for (unsigned v = 0; v < f->h; ++v) {
				slots[v] = oracle_mibf_rank(f, vals[v] % m);
				if ((f->ids[slots[v]] & 0x7FFF) == seq_id[i])
					owned = 1;
			}
			if (!owned)
				for (unsigned v = 0; v < f->h; ++v)
					f->ids[slots[v]] |= ORACLE_MIBF_SAT;
		}
	}
	return 0;
}

void oracle_mibf_free(oracle_mibf *f)
{
	free(f->bv);
	free(f->rank_word);
	free(f->ids);
	f->bv = NULL;
	f->rank_word = NULL;
	f->ids = NULL;
}

int oracle_mibf_store(const oracle_mibf *f, const char *prefix)
{
	char path[4096];
	snprintf(path, sizeof path, "%s.bf", prefix);
	FILE *o = fopen(path, "wb");
	if (!o)
		return -1;
	fprintf(o, "[BTLMIBloomFilter]\nFormat = 1\nBitVectorSize = %llu\nHashNum = %u\n"
			"KmerSize = %u\nIDWidth = 16\nSeeds =", (unsigned long long)f->m, f->h, f->k);
	for (unsigned i = 0; i < f->nseeds; ++i)
		fprintf(o, " %s", f->seeds[i]);
	fprintf(o, "\nPopCount = %llu\n[HeaderEnd]\n", (unsigned long long)f->pop);
	size_t ok = fwrite(f->ids, sizeof(uint16_t), (size_t)f->pop, o);
	if (fclose(o) || ok != (size_t)f->pop)
		return -1;
	snprintf(path, sizeof path, "%s.sdsl", prefix);
	o = fopen(path, "wb");
	if (!o)
		return -1;
	ok = fwrite(f->bv, sizeof(uint64_t), (size_t)(f->m / 64), o);
	if (fclose(o) || ok != (size_t)(f->m / 64))
		return -1;
	return 0;
}

int oracle_mibf_load(oracle_mibf *f, const char *bf_path)
{
	memset(f, 0, sizeof(*f));
	FILE *in = fopen(bf_path, "rb");
	if (!in)
		return -1;
	char line[8192];
	int started = 0, done = 0;
	unsigned long long m = 0, pop = 0;
	while (fgets(line, sizeof line, in)) {
		if (!started) {
			if (strcmp(line, "[BTLMIBloomFilter]\n"))
				break;
			started = 1;
			continue;
		}
		if (!strcmp(line, "[HeaderEnd]\n")) {
			done = 1;
			break;
		}
		sscanf(line, "BitVectorSize = %llu", &m);
		sscanf(line, "HashNum = %u", &f->h);
		sscanf(line, "KmerSize = %u", &f->k);
		sscanf(line, "PopCount = %llu", &pop);
		if (!strncmp(line, "Seeds =", 7)) {
			char *p = line + 7;
			char tok[256];
			int used;
			while (f->nseeds < ORACLE_MIBF_MAX_SEEDS && sscanf(p, "%255s%n", tok, &used) == 1) {
				strcpy(f->seeds[f->nseeds++], tok);
				p += used;
			}
		}
	}
	if (!done || m == 0 || m % 64 || f->h == 0 || f->k == 0) {
		fclose(in);
		return -2;
	}
	f->m = m;
	f->ids = (uint16_t *)malloc((size_t)(pop ? pop : 1) * sizeof(uint16_t));
	size_t got = fread(f->ids, sizeof(uint16_t), (size_t)pop, in);
	fclose(in);
	if (got != (size_t)pop)
		return -3;
	size_t L = strlen(bf_path);
	if (L < 3)
		return -1;
	char path[4096];
	snprintf(path, sizeof path, "%.*s.sdsl", (int)(L - 3), bf_path);
	in = fopen(path, "rb");
	if (!in)
		return -1;
	f->bv = (uint64_t *)malloc((size_t)(m / 64) * sizeof(uint64_t));
	got = fread(f->bv, sizeof(uint64_t), (size_t)(m / 64), in);
	fclose(in);
	if (got != (size_t)(m / 64))
		return -3;
	build_rank(f);
	return f->pop == pop ? 0 : -4;
}

double oracle_mibf_frame_probs(const oracle_mibf *f, double *probs, unsigned nids,
		unsigned allowed_miss)
{
	uint64_t *owned = (uint64_t *)calloc(nids ? nids : 1, sizeof(uint64_t));
	uint64_t sat = 0;
	for (uint64_t s = 0; s < f->pop; ++s) {
		unsigned id = f->ids[s] & 0x7FFF;
		if (id < nids)
			++owned[id];
		sat += (f->ids[s] & ORACLE_MIBF_SAT) != 0;
	}
	unsigned need = allowed_miss >= f->h ? 0 : f->h - allowed_miss;
	for (unsigned id = 0; id < nids; ++id) {
		double p = (double)owned[id] / (double)f->m;
		double acc = 0;
		for (unsigned j = need; j <= f->h; ++j) {
			double c = 1;
			for (unsigned t = 0; t < j; ++t)
				c = c * (double)(f->h - t) / (double)(t + 1);
			acc += c * pow(p, (double)j) * pow(1.0 - p, (double)(f->h - j));
		}
		probs[id] = acc;
	}
	free(owned);
	return f->pop ? (double)sat / (double)f->pop : 0.0;
}

typedef struct {
	uint32_t count, nonsat, solid, total, total_nonsat, nonsat_frame;
} tally;

static int cmp_ids(const void *a, const void *b, void *ctx)
{
	const tally *t = (const tally *)ctx;
	unsigned x = *(const unsigned *)a, y = *(const unsigned *)b;
	if (t[x].count != t[y].count)
		return t[x].count > t[y].count ? -1 : 1;
	if (t[x].nonsat != t[y].nonsat)
		return t[x].nonsat > t[y].nonsat ? -1 : 1;
	if (t[x].total != t[y].total)
		return t[x].total > t[y].total ? -1 : 1;
	return x < y ? -1 : (x > y);
}

static void sort_ids(unsigned *v, unsigned n, const tally *t)
{
	for (unsigned i = 1; i < n; ++i) { /* insertion sort: small candidate lists */
		unsigned x = v[i], j = i;
		while (j > 0 && cmp_ids(&x, &v[j - 1], (void *)t) < 0) {
			v[j] = v[j - 1];
			--j;
		}
		v[j] = x;
	}
}

static void query_mate(const oracle_mibf *f, const char *seq, size_t len, unsigned nids,
		unsigned need, tally *t, uint32_t *sat_count, uint64_t *lookups)
{
	uint64_t vals[64];
	uint16_t fid[64];
	uint8_t fsat[64];
	if (len < f->k)
		return;
	for (size_t q = 0; q + f->k <= len; ++q) {
		if (!oracle_mibf_frame_ok(f, seq + q))
			continue;
		oracle_mibf_values(f, seq + q, vals);
		int any_sat = 0;
		for (unsigned v = 0; v < f->h; ++v) {
			uint64_t p = vals[v] % f->m;
			fid[v] = 0;
			fsat[v] = 0;
			if (lookups)
				++*lookups;
			if (!bit_set(f, p))
				continue;
			if (lookups)
				++*lookups;
			uint16_t e = f->ids[oracle_mibf_rank(f, p)];
			fid[v] = e & 0x7FFF;
			fsat[v] = (e & ORACLE_MIBF_SAT) != 0;
			any_sat |= fsat[v];
		}
		if (any_sat)
			++*sat_count;
		for (unsigned v = 0; v < f->h; ++v) {
			unsigned id = fid[v];
			if (id == 0 || id >= nids)
				continue;
			int first = 1;
			for (unsigned u = 0; u < v; ++u)
				if (fid[u] == id)
					first = 0;
			if (!first)
				continue;
			unsigned hits = 0, ns = 0;
			for (unsigned u = v; u < f->h; ++u)
				if (fid[u] == id) {
					++hits;
					ns += !fsat[u];
				}
			t[id].total += hits;
			t[id].total_nonsat += ns;
			if (hits >= need) {
				++t[id].count;
				if (!any_sat)
					++t[id].nonsat_frame;
			}
			if (ns >= need)
				++t[id].nonsat;
			if (hits == f->h)
				++t[id].solid;
		}
	}
}

unsigned oracle_mibf_query(const oracle_mibf *f, const char *seq, size_t len,
		const char *seq2, size_t len2, const uint32_t *min_count, unsigned nids,
		double multi_thresh, unsigned allowed_miss, unsigned min_nonsat, int best_agree,
		oracle_qres *out, unsigned max_out, uint32_t *sat_count, uint64_t *lookups)
{
	tally *t = (tally *)calloc(nids ? nids : 1, sizeof(tally));
	unsigned need = allowed_miss >= f->h ? 0 : f->h - allowed_miss;
	uint32_t sc = 0;
	query_mate(f, seq, len, nids, need, t, &sc, lookups);
	if (seq2)
		query_mate(f, seq2, len2, nids, need, t, &sc, lookups);
	if (sat_count)
		*sat_count = sc;
	unsigned *cand = (unsigned *)malloc((nids ? nids : 1) * sizeof(unsigned));
	unsigned nc = 0;
	for (unsigned id = 1; id < nids; ++id)
		if (t[id].count > 0 && t[id].count >= min_count[id] &&
				(min_nonsat == 0 || t[id].nonsat >= min_nonsat))
			cand[nc++] = id;
	unsigned nout = 0;
	if (nc) {
		sort_ids(cand, nc, t);
		int keep = 1;
		if (best_agree) {
			unsigned bn = cand[0];
			for (unsigned i = 1; i < nc; ++i)
				if (t[cand[i]].nonsat > t[bn].nonsat)
					bn = cand[i];
			keep = bn == cand[0];
		}
		for (unsigned i = 0; keep && i < nc && nout < max_out; ++i) {
			unsigned id = cand[i];
			if (i > 0 && !((double)t[id].count > (double)t[cand[0]].count - multi_thresh))
				break;
			oracle_qres r;
			r.id = (uint16_t)id;
			r.nonSatFrameCount = t[id].nonsat_frame;
			r.solidCount = t[id].solid;
			r.count = t[id].count;
			r.nonSatCount = t[id].nonsat;
			r.totalNonSatCount = t[id].total_nonsat;
			r.totalCount = t[id].total;
			out[nout++] = r;
		}
	}
	free(cand);
	free(t);
	return nout;
}
