/*
 * window.cuh -- per-warp hash window of the classification kernels: a run of
 * up to 32*SEG frames of one read, with the canonical ntHash and validity of
 * each frame in shared memory.
 */
#ifndef BBT_WINDOW_CUH
#define BBT_WINDOW_CUH

#include <stdint.h>

#include "bbt_device.cuh"

namespace bbt {

constexpr unsigned kFull = 0xffffffffu;

/* Per-warp shared-memory window. */
template <int SEG>
struct Window {
	static constexpr int W = 32 * SEG;
	uint64_t *tab;    /* [kWinTabEntries]: seed_fw, seed_rc, rol(seed_fw, k), rol(seed_rc, k-1)
	                     of codes A,C,G,T (4 each), then 4 zeros for code 4 (not ACGT);
	                     then the base-pair tables (kPairF, kPairR) */
	uint64_t *h0;     /* [W] canonical hash of frame q (window-relative) */
	uint32_t *vmask;  /* [SEG] bit j of word c: frame 32c+j holds only ACGT */
	uint8_t *vld;     /* [W] 1 if frame q holds only ACGT */
	uint8_t *code;    /* [W + kmax] base codes 0..3, 4 = not ACGT */
};

/* Base-pair tables for a read's first k-mer, indexed by 5 * a + b for the
 * codes a, b (0..3, 4 = not ACGT, seed 0) of bases j and j + 1:
 *   kPairF: rol1(seed_fw(a)) ^ seed_fw(b)  -- two Horner steps of the forward
 *           hash at once: fh = rol2(fh) ^ entry;
 *   kPairR: seed_rc(a) ^ rol1(seed_rc(b))  -- the two bases' share of the
 *           reverse-complement hash, XOR over j of rol(seed_rc(base j), j),
 *           before its rotation by j. */
constexpr int kPairF = 20;
constexpr int kPairR = 45;
constexpr int kWinTabEntries = 70;

template <int SEG>
__host__ __device__ __forceinline__ size_t window_stride(uint32_t kmax)
{
	size_t b = kWinTabEntries * 8 + (size_t)Window<SEG>::W * 8 + SEG * 4 + Window<SEG>::W +
			Window<SEG>::W + kmax;
	return (b + 15) & ~(size_t)15;
}

template <int SEG>
__device__ __forceinline__ Window<SEG> window_at(unsigned char *base)
{
	Window<SEG> w;
	w.tab = reinterpret_cast<uint64_t *>(base);
	w.h0 = w.tab + kWinTabEntries;
	w.vmask = reinterpret_cast<uint32_t *>(w.h0 + Window<SEG>::W);
	w.vld = reinterpret_cast<uint8_t *>(w.vmask + SEG);
	w.code = w.vld + Window<SEG>::W;
	return w;
}

__device__ __forceinline__ uint64_t seed_fw_of_code(int c)
{
	return c == 0 ? kSeedA : c == 1 ? kSeedC : c == 2 ? kSeedG : c == 3 ? kSeedT : 0ull;
}

__device__ __forceinline__ uint64_t seed_rc_of_code(int c)
{
	return c == 0 ? kSeedT : c == 1 ? kSeedG : c == 2 ? kSeedC : c == 3 ? kSeedA : 0ull;
}

/* Seed tables of the current k (lanes 0-19 write one entry each) and the
 * base-pair tables (50 entries).  Entries 16-19 are 0: a base that is not
 * ACGT has seed 0, which is what keeps the rolling update exact across
 * invalid bases. */
template <int SEG>
__device__ __forceinline__ void set_tables(const Window<SEG> &win, unsigned k, int lane)
{
	if (lane < 20) {
		const int c = lane & 3, which = lane >> 2;
		const uint64_t fw = seed_fw_of_code(c), rc = seed_rc_of_code(c);
		const uint64_t v = which == 0 ? fw : which == 1 ? rc : which == 2 ? rolk(fw, k)
		                 : rolk(rc, k - 1);
		win.tab[lane] = which == 4 ? 0ull : v;
	}
	for (int e = lane; e < 50; e += 32) {
		const int x = e < 25 ? e : e - 25, a = x / 5, b = x % 5;
		win.tab[kPairF + e] = e < 25 ? rol1(seed_fw_of_code(a)) ^ seed_fw_of_code(b)
		                             : seed_rc_of_code(a) ^ rol1(seed_rc_of_code(b));
	}
	__syncwarp();
}

/* v rotated left by s (0..63): two funnel shifts of the 32-bit halves. */
__device__ __forceinline__ uint64_t rotl64(uint64_t v, unsigned s)
{
	uint32_t lo = (uint32_t)v, hi = (uint32_t)(v >> 32);
	if (s & 32u) {
		const uint32_t t = lo;
		lo = hi;
		hi = t;
	}
	const uint32_t nhi = __funnelshift_l(lo, hi, s);
	const uint32_t nlo = __funnelshift_l(hi, lo, s);
	return ((uint64_t)nhi << 32) | nlo;
}

__device__ __forceinline__ uint8_t base_code(uint8_t c)
{
	const uint8_t u = c & 0xDF;
	return u == 'A' ? 0 : u == 'C' ? 1 : u == 'G' ? 2 : u == 'T' ? 3 : 4;
}

/* table entry `which` (0 fw, 1 rc, 2 fw rolled by k, 3 rc rolled by k-1) of a
 * base code; code 4 reads one of the zero entries */
__device__ __forceinline__ uint64_t seed_of(const uint64_t *tab, int which, uint8_t code)
{
	return tab[code < 4 ? which * 4 + code : 16];
}

/* Where a read's bases are: base j of the read is element g0 + j of either an
 * ASCII byte array, or of 2-bit code words (base g at bits 2 (g % 16) of
 * words[g / 16]) with validity bits (bit g % 32 of valid[g / 32]; NULL = every
 * base is ACGT). */
struct Bases {
	const uint8_t *ascii;
	const uint32_t *words;
	const uint32_t *valid;
	uint64_t g0;
};

/* Code 0..3 of base j, 4 when it is not ACGT. */
__device__ __forceinline__ uint8_t base_code_at(const Bases &b, uint64_t j)
{
	const uint64_t g = b.g0 + j;
	if (b.ascii)
		return base_code(b.ascii[g]);
	if (b.valid && !((__ldg(b.valid + (g >> 5)) >> (g & 31u)) & 1u))
		return 4;
	return (uint8_t)((__ldg(b.words + (g >> 4)) >> (2u * (uint32_t)(g & 15u))) & 3u);
}

/* Hash frames [w0, w0 + wn) of the read whose bases src describes into the
 * window: base codes are staged with coalesced loads, then each lane hashes S
 * consecutive frames (its first k-mer two bases at a time from the base-pair
 * tables, rolling after), and the validity of the frames is balloted into one
 * mask word per 32 frames. */
template <int SEG>
__device__ void hash_window(const Bases &src, uint64_t w0, int wn, unsigned k,
		const Window<SEG> &win, int lane)
{
	const int nb = wn + (int)k - 1;
	for (int b = lane; b < nb; b += 32)
		win.code[b] = base_code_at(src, w0 + b);
	__syncwarp();
	const int S = (wn + 31) >> 5; /* frames per lane in this window */
	const int q0 = lane * S;
	const uint64_t *tab = win.tab;
	if (q0 < wn) {
		const uint8_t *cc = win.code + q0;
		/* fh = XOR_j rol(seed_fw(base j), k-1-j) by Horner's rule, rh = XOR_j
		 * rol(seed_rc(base j), j), over the k bases j of the first k-mer */
		uint64_t fh = 0, rh = 0;
		int lb = -1; /* last invalid base, window-relative */
		unsigned i = 0;
		if (k & 1u) {
			const uint8_t c = cc[0];
			fh = seed_of(tab, 0, c);
			rh = seed_of(tab, 1, c);
			if (c == 4)
				lb = q0;
			i = 1;
		}
		for (; i < k; i += 2) {
			const uint8_t c0 = cc[i], c1 = cc[i + 1];
			const int e = (int)c0 * 5 + (int)c1;
			fh = rolk(fh, 2) ^ tab[kPairF + e];
			rh ^= rotl64(tab[kPairR + e], i);
			if (c0 == 4)
				lb = q0 + (int)i;
			if (c1 == 4)
				lb = q0 + (int)i + 1;
		}
		win.h0[q0] = fh < rh ? fh : rh;
		win.vld[q0] = lb < q0;
		const int qe = min(q0 + S, wn);
		for (int q = q0 + 1; q < qe; ++q) {
			const uint8_t out = win.code[q - 1], in = win.code[q + k - 1];
			fh = rol1(fh) ^ seed_of(tab, 2, out) ^ seed_of(tab, 0, in);
			rh = ror1(rh) ^ ror1(seed_of(tab, 1, out)) ^ seed_of(tab, 3, in);
			if (in == 4)
				lb = q + (int)k - 1;
			win.h0[q] = fh < rh ? fh : rh;
			win.vld[q] = lb < q;
		}
	}
	__syncwarp();
	for (int c = 0; c < wn; c += 32) {
		const int q = c + lane;
		const uint32_t v = __ballot_sync(kFull, q < wn && win.vld[q]);
		if (lane == 0)
			win.vmask[c >> 5] = v;
	}
	__syncwarp();
}

} // namespace bbt

#endif
