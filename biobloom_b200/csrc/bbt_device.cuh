/*
 * bbt_device.cuh -- device building blocks of the classification path:
 * ntHash over ASCII bases, the derived extra hashes, hash -> bit reduction and
 * the Bloom bit probe.
 *
 * ntHash follows the published method (Mohamadi et al., Bioinformatics 2016),
 * which the reference uses through the btl_bloomfilter submodule
 * (Common/SeqEval.h:50): each base has a 64-bit seed, the forward hash of
 * s[0..k) is XOR_i rol(seed(s_i), k-1-i), the reverse-complement hash is
 * XOR_i rol(seed(comp(s_i)), i), the canonical hash is the smaller of the two,
 * and extra hash i (i >= 1) is canon * (i ^ (k * M)) followed by x ^= x >> 27.
 * Both strand hashes are built here in Horner form (one rotate-by-one per base)
 * and then rolled one base at a time.
 *
 * Filter layout in device memory: bit j of a filter is bit (j % 32) of 32-bit
 * word j / 32 (little-endian, so byte j / 8 bit j % 8 of the .bf payload).
 * A hash value v maps to bit v mod m.
 */
#ifndef BBT_DEVICE_CUH
#define BBT_DEVICE_CUH

#include <stdint.h>

namespace bbt {

constexpr uint64_t kSeedA = 0x3c8bfbb395c60474ULL;
constexpr uint64_t kSeedC = 0x3193c18562a02b4cULL;
constexpr uint64_t kSeedG = 0x20323ed082572324ULL;
constexpr uint64_t kSeedT = 0x295549f54be24456ULL;
constexpr uint64_t kMultiSeed = 0x90b45d39fb6da1faULL;
constexpr unsigned kMultiShift = 27;

/* One filter as the kernels see it. */
struct FilterDev {
	const uint32_t *words; /* m / 32 words */
	uint64_t m;            /* bits (a multiple of 64) */
	uint64_t minv;         /* floor((2^64 - 1) / m), for the reduction */
	uint64_t kmul;         /* k * kMultiSeed, for the extra hashes */
	uint32_t h;            /* hash functions */
	uint32_t k;            /* k-mer size */
};

/* Descriptor of a filter whose bit array is at `words` (device memory). */
inline FilterDev make_filter_dev(const void *words, uint64_t m, unsigned h, unsigned k)
{
	FilterDev f;
	f.words = (const uint32_t *)words;
	f.m = m;
	f.minv = ~0ull / m;
	f.kmul = (uint64_t)k * kMultiSeed;
	f.h = h;
	f.k = k;
	return f;
}

#if defined(__CUDACC__)

__device__ __forceinline__ uint64_t rol1(uint64_t v)
{
	return (v << 1) | (v >> 63);
}

__device__ __forceinline__ uint64_t ror1(uint64_t v)
{
	return (v >> 1) | (v << 63);
}

__device__ __forceinline__ uint64_t rolk(uint64_t v, unsigned s)
{
	s &= 63u;
	return s ? (v << s) | (v >> (64u - s)) : v;
}

/* Forward seed of an ASCII base, 0 for a base that is not ACGT/acgt. */
__device__ __forceinline__ uint64_t seed_fw(uint8_t c)
{
	uint8_t u = c & 0xDF; /* upper case */
	return u == 'A' ? kSeedA : u == 'C' ? kSeedC : u == 'G' ? kSeedG
	     : u == 'T' ? kSeedT : 0ull;
}

/* Seed of the complementary base. */
__device__ __forceinline__ uint64_t seed_rc(uint8_t c)
{
	uint8_t u = c & 0xDF;
	return u == 'A' ? kSeedT : u == 'C' ? kSeedG : u == 'G' ? kSeedC
	     : u == 'T' ? kSeedA : 0ull;
}

__device__ __forceinline__ bool base_ok(uint8_t c)
{
	uint8_t u = c & 0xDF;
	return u == 'A' || u == 'C' || u == 'G' || u == 'T';
}

__device__ __forceinline__ uint64_t extra_hash(uint64_t canon, unsigned k, unsigned i)
{
	uint64_t t = canon * ((uint64_t)i ^ ((uint64_t)k * kMultiSeed));
	return t ^ (t >> kMultiShift);
}

/* v mod m by Barrett reduction with minv = floor((2^64-1)/m).  Since
 * v/m - 1 < v*minv/2^64 <= v/m, the quotient estimate is the true quotient or
 * one below it, so one correction suffices. */
__device__ __forceinline__ uint64_t reduce(uint64_t v, uint64_t m, uint64_t minv)
{
	const uint64_t q = __umul64hi(v, minv);
	const uint64_t r = v - q * m;
	return r >= m ? r - m : r;
}

/* One 4-byte read through the read-only path.  On this GPU an isolated
 * random read costs a 128-byte L2 line fill from DRAM whatever the load
 * flavour (L1 bypass and smaller L2 fetch limits measured no different). */
__device__ __forceinline__ bool test_bit(const uint32_t *__restrict__ words, uint64_t b)
{
	uint32_t w = __ldg(words + (b >> 5));
	return (w >> (b & 31u)) & 1u;
}

/* BloomFilter::contains: all h bits set, reading them in order and stopping at
 * the first clear one.  *reads counts the words read. */
__device__ __forceinline__ bool contains(const FilterDev &f, uint64_t canon, unsigned &reads)
{
	if (!test_bit(f.words, reduce(canon, f.m, f.minv))) {
		++reads;
		return false;
	}
	++reads;
	for (unsigned i = 1; i < f.h; ++i) {
		++reads;
		uint64_t t = canon * ((uint64_t)i ^ f.kmul); /* extra_hash(canon, k, i) */
		t ^= t >> kMultiShift;
		if (!test_bit(f.words, reduce(t, f.m, f.minv)))
			return false;
	}
	return true;
}

/* BloomFilter::contains with the reads after the first issued together: the
 * first bit is read alone (most frames of a read that is not in the filter
 * stop there); when it is set, the other h - 1 bits (h <= 4) are read at once,
 * two dependent DRAM round trips instead of h.  The result is contains()'s.
 * *reads counts the words read; *seq the words the sequential contains()
 * reads (up to and including the first clear bit). */
__device__ __forceinline__ bool contains_split(const FilterDev &f, uint64_t canon,
		unsigned &reads, unsigned &seq)
{
	const uint64_t b0 = reduce(canon, f.m, f.minv);
	++reads;
	++seq;
	if (!test_bit(f.words, b0))
		return false;
	if (f.h > 4) {
		for (unsigned i = 1; i < f.h; ++i) {
			++reads;
			++seq;
			uint64_t t = canon * ((uint64_t)i ^ f.kmul);
			t ^= t >> kMultiShift;
			if (!test_bit(f.words, reduce(t, f.m, f.minv)))
				return false;
		}
		return true;
	}
	uint32_t w[3] = {0u, 0u, 0u};
	uint64_t b[3] = {0ull, 0ull, 0ull};
#pragma unroll
	for (unsigned i = 0; i < 3; ++i) {
		if (i + 1 < f.h) {
			uint64_t t = canon * ((uint64_t)(i + 1) ^ f.kmul);
			t ^= t >> kMultiShift;
			b[i] = reduce(t, f.m, f.minv);
			w[i] = __ldg(f.words + (b[i] >> 5));
		}
	}
	bool all = true;
#pragma unroll
	for (unsigned i = 0; i < 3; ++i) {
		if (i + 1 < f.h) {
			++reads;
			seq += all ? 1u : 0u;
			all = all && ((w[i] >> (b[i] & 31u)) & 1u);
		}
	}
	return all;
}

/* BloomFilter::contains with all h bits (h <= 4) read at once: one DRAM round
 * trip, at the price of the words after a clear bit.  The result is
 * contains()'s; *reads counts the words read, *seq the words the sequential
 * contains() reads. */
__device__ __forceinline__ bool contains_all(const FilterDev &f, uint64_t canon,
		unsigned &reads, unsigned &seq)
{
	if (f.h > 4)
		return contains_split(f, canon, reads, seq);
	uint32_t w[4] = {0u, 0u, 0u, 0u};
	uint64_t b[4] = {0ull, 0ull, 0ull, 0ull};
#pragma unroll
	for (unsigned i = 0; i < 4; ++i) {
		if (i < f.h) {
			uint64_t t = canon;
			if (i) {
				t = canon * ((uint64_t)i ^ f.kmul);
				t ^= t >> kMultiShift;
			}
			b[i] = reduce(t, f.m, f.minv);
			w[i] = __ldg(f.words + (b[i] >> 5));
		}
	}
	bool all = true;
#pragma unroll
	for (unsigned i = 0; i < 4; ++i) {
		if (i < f.h) {
			++reads;
			seq += all ? 1u : 0u;
			all = all && ((w[i] >> (b[i] & 31u)) & 1u);
		}
	}
	return all;
}

/* Loads of data read once per pass (the two-pass path's stored hashes):
 * marked evict-first in L2 so that they do not push the filter being probed
 * out of L2, and not allocated in L1. */
__device__ __forceinline__ uint64_t evict_first_policy()
{
	uint64_t pol;
	asm("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(pol));
	return pol;
}

__device__ __forceinline__ uint64_t ld_stream_u64(const uint64_t *p, uint64_t pol)
{
	uint64_t v;
	asm("ld.global.nc.L1::no_allocate.L2::cache_hint.b64 %0, [%1], %2;"
			: "=l"(v) : "l"(p), "l"(pol));
	return v;
}

__device__ __forceinline__ uint32_t ld_stream_u32(const uint32_t *p, uint64_t pol)
{
	uint32_t v;
	asm("ld.global.nc.L1::no_allocate.L2::cache_hint.b32 %0, [%1], %2;"
			: "=r"(v) : "l"(p), "l"(pol));
	return v;
}

/* A probe's filter word.  With BBT_PROBE_EVICT_LAST the load carries an L2
 * evict-last hint, so that a filter that fits L2 keeps its lines against the
 * streamed data (a build setting, off by default). */
#ifndef BBT_PROBE_EVICT_LAST
#define BBT_PROBE_EVICT_LAST 0
#endif
__device__ __forceinline__ uint32_t ld_probe_u32(const uint32_t *p)
{
#if BBT_PROBE_EVICT_LAST
	uint64_t pol;
	asm("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(pol));
	uint32_t v;
	asm("ld.global.nc.L1::no_allocate.L2::cache_hint.b32 %0, [%1], %2;"
			: "=r"(v) : "l"(p), "l"(pol));
	return v;
#else
	return __ldg(p);
#endif
}

/* Two independent BloomFilter::contains chains per lane, their rounds
 * interleaved so that both probes of a round are in flight together.
 * pa / pb: whether frame a / b is probed at all.  Word reads are counted in
 * ra / rb exactly as contains() counts them. */
__device__ __forceinline__ void contains2(const FilterDev &f, uint64_t ca, bool pa, uint64_t cb,
		bool pb, bool &ha, bool &hb, unsigned &ra, unsigned &rb)
{
	bool la = pa, lb = pb;
	for (unsigned i = 0; i < f.h && (la || lb); ++i) {
		uint64_t va = ca, vb = cb;
		if (i) {
			const uint64_t mul = (uint64_t)i ^ f.kmul;
			va = ca * mul;
			va ^= va >> kMultiShift;
			vb = cb * mul;
			vb ^= vb >> kMultiShift;
		}
		uint32_t wa = 0, wb = 0;
		uint64_t ba = 0, bb = 0;
		if (la) {
			ba = reduce(va, f.m, f.minv);
			wa = ld_probe_u32(f.words + (ba >> 5));
		}
		if (lb) {
			bb = reduce(vb, f.m, f.minv);
			wb = ld_probe_u32(f.words + (bb >> 5));
		}
		ra += la;
		rb += lb;
		la = la && ((wa >> (ba & 31u)) & 1u);
		lb = lb && ((wb >> (bb & 31u)) & 1u);
	}
	ha = la;
	hb = lb;
}

#endif /* __CUDACC__ */

} // namespace bbt

#endif
