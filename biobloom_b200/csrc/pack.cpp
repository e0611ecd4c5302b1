/*
 * pack.cpp -- bbt_pack_bases: ASCII bases to the BBT_BASES_2BIT batch form
 * (2-bit codes, base g at bits 2 (g % 16) of word g / 16, and validity bits,
 * bit g % 32 of word g / 32).  A 2-bit batch moves a quarter of the bytes to
 * the device; the kernels read the same codes the k-mer iterator would derive
 * from the ASCII bases (A/a = 0, C/c = 1, G/g = 2, T/t = 3, anything else
 * invalid).  Host only.
 */
#include "bbt.h"

#include <omp.h>

namespace {

/* code of a base and whether it is one of ACGTacgt */
struct CodeTable {
	uint8_t code[256];
	uint8_t ok[256];
	CodeTable()
	{
		for (int c = 0; c < 256; ++c) {
			code[c] = 0;
			ok[c] = 0;
		}
		const char *up = "ACGT", *lo = "acgt";
		for (int i = 0; i < 4; ++i) {
			code[(uint8_t)up[i]] = code[(uint8_t)lo[i]] = (uint8_t)i;
			ok[(uint8_t)up[i]] = ok[(uint8_t)lo[i]] = 1;
		}
	}
};

const CodeTable kTab;

} // namespace

extern "C" int bbt_pack_bases(const char *ascii, uint64_t n, uint32_t *words, uint32_t *valid,
		uint64_t *n_invalid)
{
	if ((!ascii && n) || (!words && n))
		return BBT_ERR_ARG;
	const int64_t nv = (int64_t)((n + 31) / 32); /* one validity word = two code words */
	uint64_t bad = 0;
#pragma omp parallel for schedule(static, 4096) reduction(+ : bad)
	for (int64_t v = 0; v < nv; ++v) {
		const uint64_t g0 = (uint64_t)v * 32;
		const uint64_t g1 = g0 + 32 < n ? g0 + 32 : n;
		uint32_t w[2] = {0, 0}, ok = 0;
		for (uint64_t g = g0; g < g1; ++g) {
			const uint8_t c = (uint8_t)ascii[g];
			const uint32_t j = (uint32_t)(g - g0);
			w[j >> 4] |= (uint32_t)kTab.code[c] << (2 * (j & 15));
			ok |= (uint32_t)kTab.ok[c] << j;
		}
		const uint32_t want = g1 - g0 == 32 ? 0xffffffffu : ((1u << (g1 - g0)) - 1u);
		bad += (uint64_t)__builtin_popcount(want & ~ok);
		words[2 * v] = w[0];
		if (g0 + 16 < n)
			words[2 * v + 1] = w[1];
		if (valid)
			valid[v] = ok;
	}
	if (n_invalid)
		*n_invalid = bad;
	return BBT_OK;
}
