/*
 * synth_oracle.h -- TEST INFRASTRUCTURE ONLY: the seeded workload generator
 * and the threaded filter build used by the benchmark's CPU arm and by tests
 * (synth_oracle.c).  Never linked into the product library.
 */
#ifndef SYNTH_ORACLE_H
#define SYNTH_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#include "bbt_oracle.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Same field layout and meaning as the product's bbt_synth_read_params. */
typedef struct {
	uint32_t len_min, len_max;
	double long_frac;
	uint32_t long_min, long_max;
	double sub_rate;
	double n_rate;
	uint32_t frag_min, frag_max;
} oracle_read_params;

int oracle_synth_genome(uint64_t seed, uint64_t len, double gc, double repeat_frac,
		uint32_t rep_min, uint32_t rep_max, double div_min, double div_max, char *out);
int oracle_synth_read_lengths(uint64_t seed, const oracle_read_params *p, uint64_t n_reads,
		uint64_t *out_off);
int oracle_synth_reads(uint64_t seed, const char *refs, const uint64_t *ref_off,
		uint32_t n_refs, const double *ref_frac, const oracle_read_params *p,
		uint64_t n_reads, const uint64_t *off, char *out1, char *out2, uint32_t *out_src);

/* oracle_make_filter's bit array, built by OpenMP threads. */
int oracle_make_filter_par(oracle_bf *bf, const char *const *seqs, const uint64_t *lens,
		size_t n, unsigned k, double fpr, unsigned h, uint64_t *expected_entries,
		uint64_t *redundant);

#ifdef __cplusplus
}
#endif
#endif
