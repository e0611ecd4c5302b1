/*
 * mibf.cu -- the miBF query path on the GPU: device layout of the filter, the
 * classification kernel, and the bbt_mibf_* entry points that drive it.
 *
 * Device layout.  The bit vector is cut into 32-byte blocks of 224 bits:
 * word 0 of a block is the number of set bits before the block counted from
 * the start of its superblock (2^20 blocks), words 1-7 hold bits
 * [224 b, 224 b + 224).  A probe of bit p reads one block (one DRAM sector) and
 * gets both the bit and its rank: superblock base (a small table that stays
 * in L1/L2) + block count + popcounts of the words before p in the block.  The
 * ID of a set bit is ids[rank] (a second, dependent read).  The reference's
 * MIBloomFilter keeps the same bits with sdsl rank support (a separate rank
 * structure); here rank and bits share the sector.
 *
 * Dense layout (the default when it fits in a fraction of free HBM): one
 * 16-bit entry per bit position, 0 for a clear bit, else the slot's ID with its
 * saturation bit, IDs outside 1 .. num_ids-1 stored as 0x7FFF (they count as
 * hits but tally nothing, as in the rank layout).  A probe is then a single
 * random 2-byte read instead of a block read followed by an ID read: twice the
 * bytes of the compact form for 40% fewer random DRAM accesses per read.
 *
 * Kernel.  One warp classifies one read (pair) at a time, taking reads from a
 * work counter four at a time.  Bases are staged 512 at a time as 2-bit codes
 * (one 64-bit word per 32 bases, built with three ballots over coalesced byte
 * loads) plus an invalid-base mask; each lane then takes one frame, computes
 * its h seed values from per-seed position tables in shared memory, issues
 * the h block reads, then the ID reads.  Per-frame, per-ID increments are
 * merged across the warp with __match_any_sync and added to a per-warp tally
 * table in shared memory (one slot per target ID), from which the warp picks
 * the significant IDs and writes the result list and the summary counters.
 */
#include <cuda_runtime.h>

#include <cub/device/device_scan.cuh>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <fstream>
#include <string>
#include <vector>

#include "bbt_device.cuh"
#include "bucketed.cuh"
#include "mibf_ctx.hpp"
#include "window.cuh"

namespace bbt {

constexpr int kBlockBits = 224;
constexpr int kSuperShift = 20;
constexpr int kStageBases = 512;
constexpr int kReadsPerGrab = 4;

struct MibfDev {
	const uint4 *blocks;
	const unsigned long long *super;
	const uint16_t *ids;
	const uint16_t *dense;
	uint64_t m, minv;
	uint32_t h, k, nse, nids;
	int kmer_mode;
};

struct MibfArgs {
	MibfDev f;
	const uint8_t *seq;         /* ASCII bases, or 2-bit code words when packed */
	const uint64_t *off;
	const uint8_t *seq2;
	const uint64_t *off2;
	int packed;                 /* bases are BBT_BASES_2BIT */
	const uint32_t *valid[2];   /* packed: validity bits per mate array (NULL = all ACGT) */
	uint64_t n_reads;
	const uint32_t *minc;
	uint32_t need, min_nonsat;
	int best_agree, skip_empty_summary;
	double multi;
	const unsigned long long *tables;
	bbt_mibf_hit *hits;
	uint32_t max_hits;
	uint32_t *n_hits, *sat;
	unsigned long long *counts; /* this batch's summary counters */
	unsigned long long *work;
	unsigned int *flags;
	unsigned long long *stat;   /* frames visited, values probed, probes that hit */
	uint32_t T;                 /* tally slots per warp, a multiple of 32 */
	unsigned long long *gtally; /* more than kMibfSmemIds IDs: per-warp tally tables in
	                               global memory (3 x T words each), zero between reads */
	/* bucketed query (PRE kernels): the entries of every frame resolved
	 * beforehand, frame order (h per frame), their validity bits, and the
	 * frame offsets of these reads (pre_fo[r] - pre_fo0 = first frame of
	 * read r) */
	const uint16_t *pre_e;
	const uint32_t *pre_valid;
	const uint64_t *pre_fo;
	uint64_t pre_fo0;
};

/* IDs a read may touch before a warp with global tally tables clears and scans
 * every slot instead of its list. */
constexpr uint32_t kTouchCap = 1024;

struct LaneCounts {
	unsigned long long frames = 0, probes = 0, hits = 0;
};

__host__ __device__ inline size_t mibf_warp_bytes(uint32_t T)
{
	return 17 * 8 + 18 * 4 + (size_t)3 * T * 8; /* codes, invalid words, tally */
}

/* With the tally in global memory: codes, invalid words, the touched count and
 * list; rounded up to 16 bytes so that every warp's code words stay 8-byte
 * aligned. */
__host__ __device__ inline size_t mibf_warp_bytes_big()
{
	return (17 * 8 + 18 * 4 + 4 + (size_t)kTouchCap * 4 + 15) & ~(size_t)15;
}
static_assert((17 * 8 + 18 * 4) % 8 == 0, "the tally words follow 8-byte aligned");

/* Seed tables: with BBT_MIBF_PAIR_TABLES (the default) one entry per pair of
 * positions and pair of base codes (16 x 16 per seed: a value costs 13 table
 * reads for k = 25), else one per position and base code (32 x 4). */
#ifndef BBT_MIBF_PAIR_TABLES
#define BBT_MIBF_PAIR_TABLES 1
#endif
constexpr int kTabEntries = BBT_MIBF_PAIR_TABLES ? 256 : 128; /* ulonglong2 per seed */
constexpr int kQueryThreads = BBT_MIBF_PAIR_TABLES ? 256 : 128;
#ifndef BBT_MIBF_MIN_BLOCKS
#define BBT_MIBF_MIN_BLOCKS (BBT_MIBF_PAIR_TABLES ? 2 : 4)
#endif
constexpr int kQueryMinBlocks = BBT_MIBF_MIN_BLOCKS;

__host__ inline size_t mibf_smem_bytes(uint32_t nse, uint32_t T, int warps, bool big)
{
	return (size_t)nse * kTabEntries * 16 +
			(size_t)warps * (big ? mibf_warp_bytes_big() : mibf_warp_bytes(T));
}

__device__ __forceinline__ uint64_t spread_bits(uint32_t v)
{
	uint64_t x = v;
	x = (x | (x << 16)) & 0x0000FFFF0000FFFFull;
	x = (x | (x << 8)) & 0x00FF00FF00FF00FFull;
	x = (x | (x << 4)) & 0x0F0F0F0F0F0F0F0Full;
	x = (x | (x << 2)) & 0x3333333333333333ull;
	x = (x | (x << 1)) & 0x5555555555555555ull;
	return x;
}

/* min(F, R) of one seed over the 2-bit codes w (base j at bits 2j, 2j+1),
 * from the pair tables: entry p * 16 + (codes of bases 2p, 2p+1). */
__device__ __forceinline__ uint64_t seed_value_pairs(const ulonglong2 *tab, uint64_t w, uint32_t k)
{
	uint64_t F = 0, R = 0;
#pragma unroll
	for (int p = 0; p < 16; ++p) {
		if (2 * p < (int)k) {
			const ulonglong2 e = tab[p * 16 + (int)((w >> (4 * p)) & 15u)];
			F ^= e.x;
			R ^= e.y;
		}
	}
	return F < R ? F : R;
}

/* min(F, R) of one seed over the 2-bit codes w (base j at bits 2j, 2j+1). */
#ifndef BBT_MIBF_SEED_UNROLL
#define BBT_MIBF_SEED_UNROLL 32
#endif
constexpr int kSeedUnroll = BBT_MIBF_SEED_UNROLL;
__device__ __forceinline__ uint64_t seed_value(const ulonglong2 *tab, uint64_t w, uint32_t k)
{
	uint64_t F = 0, R = 0;
#pragma unroll kSeedUnroll
	for (int j = 0; j < 32; ++j) {
		if (j < (int)k) {
			const ulonglong2 e = tab[j * 4 + (int)((w >> (2 * j)) & 3u)];
			F ^= e.x;
			R ^= e.y;
		}
	}
	return F < R ? F : R;
}

/* Tally word order: A = count | nonSatCount << 32, B = solidCount |
 * totalCount << 32, C = totalNonSatCount | nonSatFrameCount << 32. */
struct Cand {
	unsigned long long k1, k2; /* count << 32 | nonSat, total << 32 | ~id: larger is better */
};

/* k1 of a candidate from its A tally word (count low, nonSat high). */
__device__ __forceinline__ unsigned long long cand_k1(unsigned long long A)
{
	return (A << 32) | (A >> 32);
}

__device__ __forceinline__ bool cand_less(const Cand &a, const Cand &b)
{
	return a.k1 < b.k1 || (a.k1 == b.k1 && a.k2 < b.k2);
}

__device__ __forceinline__ Cand warp_best(Cand c)
{
#pragma unroll
	for (int o = 16; o; o >>= 1) {
		Cand x;
		x.k1 = __shfl_xor_sync(kFull, c.k1, o);
		x.k2 = __shfl_xor_sync(kFull, c.k2, o);
		if (cand_less(c, x))
			c = x;
	}
	return c;
}

/* The 2-bit codes (w) and validity of frame q of the staged bases. */
__device__ __forceinline__ bool frame_word(const uint64_t *cw, const uint32_t *iw, uint32_t q,
		uint32_t nfr, uint64_t kmask, uint64_t &w)
{
	w = 0;
	if (q >= nfr)
		return false;
	const uint32_t idx = q >> 5, sh = q & 31;
	const uint64_t lo = cw[idx], hi = cw[idx + 1];
	w = sh ? (lo >> (2 * sh)) | (hi << (64 - 2 * sh)) : lo;
	const uint64_t inv = ((uint64_t)iw[idx] | ((uint64_t)iw[idx + 1] << 32)) >> sh;
	return (inv & kmask) == 0;
}

/* The h values of a frame (seed hashes, or ntHash and its extra hashes). */
template <int H>
__device__ __forceinline__ void frame_values(const MibfDev &f, const ulonglong2 *tab, bool ok,
		uint64_t w, uint64_t *vals)
{
	const uint32_t k = f.k, h = f.h;
	if (f.kmer_mode) {
		const uint64_t c = ok ? (BBT_MIBF_PAIR_TABLES ? seed_value_pairs(tab, w, k)
		                                              : seed_value(tab, w, k)) : 0;
		vals[0] = c;
#pragma unroll
		for (int v = 1; v < H; ++v)
			vals[v] = extra_hash(c, k, v);
	} else {
#pragma unroll
		for (int v = 0; v < H; ++v)
			vals[v] = (ok && v < (int)h)
					? (BBT_MIBF_PAIR_TABLES ? seed_value_pairs(tab + v * kTabEntries, w, k)
					                        : seed_value(tab + v * kTabEntries, w, k))
					: 0;
	}
}

/* Dense layout: one 2-byte read per value; e = ID entry, 0 for a clear bit. */
template <int H>
__device__ __forceinline__ void probe_dense(const MibfArgs &a, bool ok, const uint64_t *vals,
		uint32_t *e)
{
#pragma unroll
	for (int v = 0; v < H; ++v) {
		e[v] = 0;
		if (ok && v < (int)a.f.h)
			e[v] = __ldg(a.f.dense + reduce(vals[v], a.f.m, a.f.minv));
	}
}

/* Rank layout: a block read per value, then an ID read per set bit. */
template <int H>
__device__ __forceinline__ void probe_rank(const MibfArgs &a, bool ok, const uint64_t *vals,
		uint32_t *e, bool *hit)
{
	uint4 q0v[H], q1v[H];
	uint32_t rr[H];
	uint64_t blk[H];
#pragma unroll
	for (int v = 0; v < H; ++v) {
		if (ok && v < (int)a.f.h) {
			const uint64_t p = reduce(vals[v], a.f.m, a.f.minv);
			blk[v] = p / kBlockBits;
			rr[v] = (uint32_t)(p - blk[v] * kBlockBits);
			q0v[v] = __ldg(a.f.blocks + 2 * blk[v]);
			q1v[v] = __ldg(a.f.blocks + 2 * blk[v] + 1);
		}
	}
#pragma unroll
	for (int v = 0; v < H; ++v) {
		hit[v] = false;
		e[v] = 0;
		if (ok && v < (int)a.f.h) {
			const uint32_t d[7] = {q0v[v].y, q0v[v].z, q0v[v].w, q1v[v].x, q1v[v].y, q1v[v].z,
					q1v[v].w};
			const uint32_t ws = rr[v] >> 5, bit = rr[v] & 31u;
			uint32_t acc = 0, word = 0;
#pragma unroll
			for (int i = 0; i < 7; ++i) {
				if ((uint32_t)i < ws)
					acc += __popc(d[i]);
				if ((uint32_t)i == ws)
					word = d[i];
			}
			if ((word >> bit) & 1u) {
				acc += __popc(word & ((1u << bit) - 1u));
				const uint64_t rank = a.f.super[blk[v] >> kSuperShift] + q0v[v].x + acc;
				hit[v] = true;
				e[v] = __ldg(a.f.ids + rank);
			}
		}
	}
}

/* A frame's per-ID increments, merged across the warp with __match_any_sync
 * and added to the warp's tally table. */
template <int H>
__device__ __forceinline__ void frame_tally(const MibfArgs &a, bool ok, const uint32_t *e,
		const bool *hit, unsigned long long *TA, unsigned long long *TB, unsigned long long *TC,
		uint32_t &satc, LaneCounts &lc, int lane, uint32_t *tlist)
{
	const uint32_t h = a.f.h, nids = a.f.nids, need = a.need;
	bool anysat = false;
#pragma unroll
	for (int v = 0; v < H; ++v) {
		anysat |= hit[v] && (e[v] & kMibfSat);
		lc.hits += hit[v] ? 1u : 0u;
	}
	lc.frames += ok ? 1u : 0u;
	lc.probes += ok ? h : 0u;
	satc += __popc(__ballot_sync(kFull, anysat));
#pragma unroll
	for (int r = 0; r < H; ++r) {
		uint32_t key = 0xFFFFFFFFu, id = 0, hits = 0, nsh = 0;
		if (hit[r]) {
			id = e[r] & 0x7FFFu;
			bool first = id != 0 && id < nids;
#pragma unroll
			for (int u = 0; u < r; ++u)
				if (hit[u] && (e[u] & 0x7FFFu) == id)
					first = false;
			if (first) {
#pragma unroll
				for (int u = 0; u < H; ++u)
					if (hit[u] && (e[u] & 0x7FFFu) == id) {
						++hits;
						nsh += (e[u] & kMibfSat) ? 0u : 1u;
					}
				key = id | (hits << 16) | (nsh << 21) | ((anysat ? 1u : 0u) << 26);
			}
		}
		const uint32_t grp = __match_any_sync(kFull, key);
		if (key != 0xFFFFFFFFu && lane == __ffs(grp) - 1) {
			const unsigned long long n = (unsigned long long)__popc(grp);
			const uint32_t cnt = hits >= need, ns = nsh >= need, sol = hits == h;
			const uint32_t nsf = cnt && !anysat;
			const unsigned long long ia = cnt | ((unsigned long long)ns << 32);
			const unsigned long long ib = sol | ((unsigned long long)hits << 32);
			const unsigned long long ic = nsh | ((unsigned long long)nsf << 32);
			if (ia)
				atomicAdd(TA + id, n * ia);
			/* ib is never 0 (hits >= 1): the old value says whether this read
			 * touched the ID before */
			const unsigned long long old = atomicAdd(TB + id, n * ib);
			if (tlist && old == 0) {
				const uint32_t at = atomicAdd(tlist, 1u);
				if (at < kTouchCap)
					tlist[1 + at] = id;
			}
			if (ic)
				atomicAdd(TC + id, n * ic);
		}
	}
}

/* The bases of mate array m from base g0 on (ASCII or 2-bit codes). */
__device__ __forceinline__ Bases mate_bases(const MibfArgs &a, uint32_t m, uint64_t g0)
{
	Bases b;
	const uint8_t *sq = m ? a.seq2 : a.seq;
	b.g0 = g0;
	b.ascii = a.packed ? nullptr : sq;
	b.words = a.packed ? reinterpret_cast<const uint32_t *>(sq) : nullptr;
	b.valid = a.packed ? a.valid[m] : nullptr;
	return b;
}

/* All frames of one mate: bases staged 512 at a time, then steps of 32 * FPL
 * frames, each lane holding FPL frames (FPL * h reads in flight per lane). */
template <int H, bool DENSE, int FPL>
__device__ __forceinline__ void mibf_scan_mate(const MibfArgs &a, const ulonglong2 *tab,
		uint64_t *cw, uint32_t *iw, unsigned long long *TA, unsigned long long *TB,
		unsigned long long *TC, const Bases &src, uint64_t len, uint32_t &satc,
		LaneCounts &lc, int lane, uint32_t *tlist)
{
	const uint32_t k = a.f.k;
	const uint64_t kmask = (k >= 64) ? ~0ull : ((1ull << k) - 1);
	if (len < k)
		return;
	for (uint64_t c0 = 0; c0 + k <= len; c0 += kStageBases - k + 1) {
		__syncwarp();
#pragma unroll 4
		for (int it = 0; it < kStageBases / 32; ++it) {
			const uint64_t pos = c0 + (uint64_t)it * 32 + lane;
			const uint8_t c = pos < len ? base_code_at(src, pos) : (uint8_t)4;
			const uint32_t lo = __ballot_sync(kFull, c & 1u);
			const uint32_t hi = __ballot_sync(kFull, (c >> 1) & 1u);
			const uint32_t inv = __ballot_sync(kFull, c >> 2);
			if (lane == it) {
				cw[it] = spread_bits(lo) | (spread_bits(hi) << 1);
				iw[it] = inv;
			}
		}
		if (lane == 16) {
			cw[16] = 0;
			iw[16] = ~0u;
		}
		__syncwarp();
		const uint64_t avail = len - c0 < (uint64_t)kStageBases ? len - c0 : kStageBases;
		const uint32_t nfr = (uint32_t)avail - k + 1;
		for (uint32_t q0 = 0; q0 < nfr; q0 += 32 * FPL) {
			bool ok[FPL];
			uint64_t vals[FPL][H];
			uint32_t e[FPL][H];
			bool hit[FPL][H];
#pragma unroll
			for (int f = 0; f < FPL; ++f) {
				uint64_t w;
				ok[f] = frame_word(cw, iw, q0 + 32 * f + lane, nfr, kmask, w);
				frame_values<H>(a.f, tab, ok[f], w, vals[f]);
			}
			if (DENSE) {
#pragma unroll
				for (int f = 0; f < FPL; ++f)
					probe_dense<H>(a, ok[f], vals[f], e[f]);
#pragma unroll
				for (int f = 0; f < FPL; ++f)
#pragma unroll
					for (int v = 0; v < H; ++v)
						hit[f][v] = e[f][v] != 0;
			} else {
#pragma unroll
				for (int f = 0; f < FPL; ++f)
					probe_rank<H>(a, ok[f], vals[f], e[f], hit[f]);
			}
#pragma unroll
			for (int f = 0; f < FPL; ++f)
				frame_tally<H>(a, ok[f], e[f], hit[f], TA, TB, TC, satc, lc, lane, tlist);
		}
	}
	__syncwarp();
}

/* The frames [x0, x0 + nfr) of one mate with their entries resolved
 * beforehand (a.pre_e, dense-layout values: 0 for a clear bit), one frame per
 * lane per step, tallied as mibf_scan_mate tallies them. */
template <int H>
__device__ __forceinline__ void mibf_scan_pre(const MibfArgs &a, uint64_t x0, uint32_t nfr,
		unsigned long long *TA, unsigned long long *TB, unsigned long long *TC, uint32_t &satc,
		LaneCounts &lc, int lane, uint32_t *tlist)
{
	const uint32_t h = a.f.h;
	for (uint32_t q0 = 0; q0 < nfr; q0 += 32) {
		const uint32_t q = q0 + lane;
		bool ok = false;
		uint32_t e[H];
		bool hit[H];
		const uint64_t x = x0 + q;
		if (q < nfr)
			ok = (__ldg(a.pre_valid + (x >> 5)) >> (x & 31u)) & 1u;
#pragma unroll
		for (int v = 0; v < H; ++v) {
			e[v] = (ok && v < (int)h) ? __ldg(a.pre_e + x * h + v) : 0u;
			hit[v] = e[v] != 0;
		}
		frame_tally<H>(a, ok, e, hit, TA, TB, TC, satc, lc, lane, tlist);
	}
}

/*
 * BIG (more than kMibfSmemIds IDs): each warp's tally table lives in global
 * memory (a.gtally, zero between reads) and the warp lists the IDs the read
 * touches (tlist in shared memory); candidates are looked for, and the table
 * is cleared, over that list (over every slot when the list overflowed).
 * PRE: the frames' entries come resolved (the bucketed query, dense layout).
 */
template <int H, bool DENSE, int FPL, bool BIG, bool PRE>
__global__ void __launch_bounds__(kQueryThreads, kQueryMinBlocks) mibf_query_kernel(MibfArgs a)
{
	extern __shared__ __align__(16) unsigned char smem[];
	const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
	const uint32_t nse = a.f.nse, T = a.T, nids = a.f.nids;
	unsigned long long *tabw = reinterpret_cast<unsigned long long *>(smem);
	for (uint32_t i = threadIdx.x; i < nse * kTabEntries * 2; i += blockDim.x)
		tabw[i] = a.tables[i];
	unsigned char *wb = smem + (size_t)nse * kTabEntries * 16 +
			(size_t)wib * (BIG ? mibf_warp_bytes_big() : mibf_warp_bytes(T));
	uint64_t *cw = reinterpret_cast<uint64_t *>(wb);
	uint32_t *iw = reinterpret_cast<uint32_t *>(wb + 17 * 8);
	unsigned long long *TA, *TB, *TC;
	uint32_t *tlist = nullptr;
	if (BIG) {
		const uint64_t gw = (uint64_t)blockIdx.x * (blockDim.x >> 5) + wib;
		TA = a.gtally + gw * 3ull * T;
		tlist = reinterpret_cast<uint32_t *>(wb + 17 * 8 + 18 * 4);
		if (lane == 0)
			tlist[0] = 0;
	} else {
		TA = reinterpret_cast<unsigned long long *>(wb + 17 * 8 + 18 * 4);
		for (uint32_t i = lane; i < 3 * T; i += 32)
			TA[i] = 0;
	}
	TB = TA + T;
	TC = TB + T;
	__syncthreads();
	const ulonglong2 *tab = reinterpret_cast<const ulonglong2 *>(smem);
	const uint32_t k = a.f.k;
	unsigned long long *above = a.counts, *unique = a.counts + (nids + 2);
	LaneCounts lc;
	for (;;) {
		unsigned long long r0 = 0;
		if (lane == 0)
			r0 = atomicAdd(a.work, (unsigned long long)kReadsPerGrab);
		r0 = __shfl_sync(kFull, r0, 0);
		if (r0 >= a.n_reads)
			break;
		const uint64_t r1 = r0 + kReadsPerGrab < a.n_reads ? r0 + kReadsPerGrab : a.n_reads;
		for (uint64_t r = r0; r < r1; ++r) {
			const uint64_t b1 = a.off[r], len1 = a.off[r + 1] - b1;
			uint64_t b2 = 0, len2 = 0;
			if (a.seq2) {
				b2 = a.off2[r];
				len2 = a.off2[r + 1] - b2;
			}
			/* frameCount (MIBFClassifier.hpp:774, 802-803) */
			const uint32_t fc = len1 >= k ? (uint32_t)(len1 - k + 1)
					: (len2 >= k ? (uint32_t)(len2 - k + 1) : 0u);
			uint32_t satc = 0;
			if (fc && PRE) {
				const uint64_t x = a.pre_fo[r] - a.pre_fo0;
				const uint32_t f1 = len1 >= k ? (uint32_t)(len1 - k + 1) : 0u;
				const uint32_t f2 = len2 >= k ? (uint32_t)(len2 - k + 1) : 0u;
				mibf_scan_pre<H>(a, x, f1, TA, TB, TC, satc, lc, lane, tlist);
				if (a.seq2)
					mibf_scan_pre<H>(a, x + f1, f2, TA, TB, TC, satc, lc, lane, tlist);
			} else if (fc) {
				mibf_scan_mate<H, DENSE, FPL>(a, tab, cw, iw, TA, TB, TC,
						mate_bases(a, 0, b1), len1, satc, lc, lane, tlist);
				if (a.seq2)
					mibf_scan_mate<H, DENSE, FPL>(a, tab, cw, iw, TA, TB, TC,
							mate_bases(a, 1, b2), len2, satc, lc, lane, tlist);
			}
			__syncwarp();
			/* the slots to look at: every slot, or the IDs the read touched */
			const uint32_t touched = BIG ? tlist[0] : 0u;
			const bool listed = BIG && touched <= kTouchCap;
			const uint32_t nslots = listed ? touched : T;
			auto slot_id = [&](uint32_t j) -> uint32_t { return listed ? tlist[1 + j] : j; };
			const uint32_t *mrow = a.minc + (size_t)fc * nids;
			auto significant = [&](uint32_t s) -> bool {
				const unsigned long long A = TA[s];
				const uint32_t cnt = (uint32_t)A, ns = (uint32_t)(A >> 32);
				return s >= 1 && s < nids && cnt > 0 && cnt >= __ldg(mrow + s) &&
						(a.min_nonsat == 0 || ns >= a.min_nonsat);
			};
			/* significant IDs */
			uint32_t cmask = 0, maxns = 0;
			Cand best = {0ull, 0ull};
			if (fc) {
				for (uint32_t j0 = 0; j0 < nslots; j0 += 32) {
					const uint32_t j = j0 + lane;
					if (j >= nslots)
						continue;
					const uint32_t s = slot_id(j);
					if (significant(s)) {
						if (!BIG)
							cmask |= 1u << (j0 >> 5);
						const unsigned long long A = TA[s];
						Cand c = {cand_k1(A), ((TB[s] >> 32) << 32) | (0xFFFFFFFFull - s)};
						if (cand_less(best, c))
							best = c;
						const uint32_t ns = (uint32_t)(A >> 32);
						maxns = ns > maxns ? ns : maxns;
					}
				}
			}
			best = warp_best(best);
			maxns = __reduce_max_sync(kFull, maxns);
			uint32_t n_out = 0;
			if (best.k1 && !(a.best_agree && maxns > (uint32_t)best.k1)) {
				const double thr = (double)(uint32_t)(best.k1 >> 32) - a.multi;
				Cand cur = best;
				for (;;) {
					const uint32_t id = 0xFFFFFFFFu - (uint32_t)cur.k2;
					if (lane == 0) {
						if (n_out < a.max_hits) {
							const unsigned long long A = TA[id], B = TB[id], C = TC[id];
							bbt_mibf_hit o;
							o.id = id;
							o.nonSatFrameCount = (uint32_t)(C >> 32);
							o.solidCount = (uint32_t)B;
							o.count = (uint32_t)A;
							o.nonSatCount = (uint32_t)(A >> 32);
							o.totalNonSatCount = (uint32_t)C;
							o.totalCount = (uint32_t)(B >> 32);
							a.hits[r * a.max_hits + n_out] = o;
						}
						atomicAdd(above + id, 1ull);
					}
					++n_out;
					/* next: the best candidate below cur that passes the threshold */
					Cand nx = {0ull, 0ull};
					for (uint32_t j0 = 0; j0 < nslots; j0 += 32) {
						if (!BIG && !((cmask >> (j0 >> 5)) & 1u))
							continue;
						const uint32_t j = j0 + lane;
						if (j >= nslots)
							continue;
						const uint32_t s = slot_id(j);
						if (BIG && !significant(s))
							continue;
						const unsigned long long A = TA[s];
						Cand c = {cand_k1(A), ((TB[s] >> 32) << 32) | (0xFFFFFFFFull - s)};
						if (cand_less(c, cur) && (double)(uint32_t)A > thr && cand_less(nx, c))
							nx = c;
					}
					nx = warp_best(nx);
					if (!nx.k1)
						break;
					cur = nx;
				}
			}
			if (lane == 0) {
				a.n_hits[r] = n_out;
				a.sat[r] = satc;
				if (n_out > a.max_hits)
					atomicOr(a.flags, 1u);
				if (n_out == 0) {
					if (!a.skip_empty_summary)
						atomicAdd(a.counts + 2 * (nids + 2) + 1, 1ull);
				} else if (n_out == 1) {
					atomicAdd(unique + (0xFFFFFFFFu - (uint32_t)best.k2), 1ull);
				} else {
					atomicAdd(a.counts + 2 * (nids + 2), 1ull);
				}
			}
			__syncwarp();
			for (uint32_t j = lane; j < nslots; j += 32) {
				const uint32_t s = slot_id(j);
				TA[s] = 0;
				TB[s] = 0;
				TC[s] = 0;
			}
			__syncwarp();
			if (BIG && lane == 0)
				tlist[0] = 0;
			__syncwarp();
		}
	}
#pragma unroll
	for (int o = 16; o; o >>= 1) {
		lc.frames += __shfl_xor_sync(kFull, lc.frames, o);
		lc.probes += __shfl_xor_sync(kFull, lc.probes, o);
		lc.hits += __shfl_xor_sync(kFull, lc.hits, o);
	}
	if (lane == 0 && (lc.frames || lc.probes)) {
		atomicAdd(a.stat, lc.frames);
		atomicAdd(a.stat + 1, lc.probes);
		atomicAdd(a.stat + 2, lc.hits);
	}
}

/* Add a batch's summary counters to the context's, unless a read of the
 * batch overflowed its result slots (the caller then runs the batch again). */
__global__ void mibf_commit_kernel(const unsigned long long *batch, unsigned long long *total,
		uint32_t n, const unsigned int *flags, uint64_t reads)
{
	if (flags[0])
		return;
	for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
		if (batch[i])
			atomicAdd(total + i, batch[i]); /* batches on other streams commit too */
	if (blockIdx.x == 0 && threadIdx.x == 0)
		atomicAdd(total + n, (unsigned long long)reads);
}

/* Largest frame count of a device batch and a bitmap of the frame counts
 * below 65536 that occur. */
__global__ void mibf_frame_counts_kernel(const uint64_t *off, const uint64_t *off2, uint64_t n,
		uint32_t k, unsigned int *out)
{
	for (uint64_t r = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; r < n;
			r += (uint64_t)gridDim.x * blockDim.x) {
		const uint64_t l1 = off[r + 1] - off[r];
		const uint64_t l2 = off2 ? off2[r + 1] - off2[r] : 0;
		const uint64_t f64 = l1 >= k ? l1 - k + 1 : (l2 >= k ? l2 - k + 1 : 0);
		const uint32_t fc = f64 > 0xFFFFFFFFull ? 0xFFFFFFFFu : (uint32_t)f64;
		atomicMax(out, fc);
		if (fc < 65536u)
			atomicOr(out + 1 + (fc >> 5), 1u << (fc & 31));
	}
}

/* Block popcounts of the raw bit vector (words of 32 bits). */
__global__ void mibf_block_pop_kernel(const uint32_t *raw, uint64_t nwords, uint64_t nblocks,
		unsigned long long *pop)
{
	for (uint64_t b = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; b < nblocks;
			b += (uint64_t)gridDim.x * blockDim.x) {
		unsigned c = 0;
		for (int i = 0; i < 7; ++i) {
			const uint64_t w = b * 7 + i;
			c += w < nwords ? __popc(raw[w]) : 0;
		}
		pop[b] = c;
	}
}

/* Blocks from the raw words and the exclusive scan of block popcounts. */
__global__ void mibf_block_build_kernel(const uint32_t *raw, uint64_t nwords, uint64_t nblocks,
		const unsigned long long *rank, unsigned long long *super, uint4 *blocks)
{
	for (uint64_t b = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; b < nblocks;
			b += (uint64_t)gridDim.x * blockDim.x) {
		uint32_t d[7];
		for (int i = 0; i < 7; ++i) {
			const uint64_t w = b * 7 + i;
			d[i] = w < nwords ? raw[w] : 0u;
		}
		const uint64_t sb = b >> kSuperShift;
		if ((b & ((1ull << kSuperShift) - 1)) == 0)
			super[sb] = rank[b];
		const unsigned long long base = rank[b & ~((1ull << kSuperShift) - 1)];
		blocks[2 * b] = make_uint4((uint32_t)(rank[b] - base), d[0], d[1], d[2]);
		blocks[2 * b + 1] = make_uint4(d[3], d[4], d[5], d[6]);
	}
}

/* Popcount of each 64-bit word of the bit vector. */
__global__ void mibf_word_pop_kernel(const uint64_t *raw, uint64_t n, unsigned long long *pop)
{
	for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
			i += (uint64_t)gridDim.x * blockDim.x)
		pop[i] = (unsigned long long)__popcll(raw[i]);
}

/* Dense ID map: two entries (bit positions 2t, 2t+1) per thread, so that the
 * 32-bit stores of a warp are contiguous. */
__global__ void mibf_dense_build_kernel(const uint64_t *raw, uint64_t m,
		const unsigned long long *rank, const uint16_t *ids, uint32_t nids, uint32_t *dense2)
{
	for (uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; t < m / 2;
			t += (uint64_t)gridDim.x * blockDim.x) {
		const uint64_t p = 2 * t, w = raw[p >> 6];
		const unsigned b = (unsigned)(p & 63);
		uint64_t r = rank[p >> 6] + (uint64_t)__popcll(b ? (w & ((1ull << b) - 1)) : 0ull);
		uint32_t out = 0;
		for (int j = 0; j < 2; ++j) {
			if ((w >> (b + j)) & 1ull) {
				const uint32_t e = ids[r++];
				const uint32_t id = e & 0x7FFFu;
				const uint32_t v = (e & kMibfSat) | ((id >= 1 && id < nids) ? id : 0x7FFFu);
				out |= v << (16 * j);
			}
		}
		dense2[t] = out;
	}
}

/* ---- bucketed query (dense layout) ----
 *
 * Every probe of the query is known once a read is hashed (MIBFQuerySupport
 * visits every frame), so the probes of a sub-batch of reads can be sorted by
 * address before any is made.  The dense ID map is cut into buckets of
 * 2^bshift entries that fit L2:
 *   hash     -- per window block of W frames (W * h <= kMbkRequests): every
 *               frame's h values, from the packed bases and the seed tables;
 *               its validity bit; its requests (entry offset in the bucket)
 *               staged in shared memory, counted per bucket, then written to
 *               the block's region of the pool in bucket order with their
 *               slot (frame * h + value) in the block;
 *   resolve  -- the (bucket, block) segments in bucket-major order, 32
 *               segments per warp: each request reads its entry out of the
 *               bucket held in L2 and writes it beside the request;
 *   unscatter-- per block, the entries go to their slots in shared memory and
 *               out to the sub-batch's entry array in frame order;
 * then the query kernel (PRE) tallies every read from those entries exactly
 * as it does from its own probes.
 */
constexpr uint32_t kMbkThreads = 256;
constexpr uint32_t kMbkRequests = 10752;
constexpr uint32_t kMbkMaxBuckets = 2048;

struct MbkArgs {
	MibfDev f;
	const unsigned long long *tables;
	PackedBases pk[2];
	const uint64_t *off, *off2;  /* the batch's base offsets (off2 NULL: single-end) */
	uint64_t r0, nr;             /* reads [r0, r0 + nr) */
	const uint64_t *fo;          /* frame offsets of the batch's reads (both mates) */
	uint64_t fo0, T;             /* fo[r0]; frames of the sub-batch */
	uint32_t W, nblk, nbkt, bshift;
	uint32_t *valid;             /* frame validity bits of the sub-batch */
	uint16_t *e;                 /* entries of the sub-batch, T * h */
	uint32_t *cnt, *loc, *btot;  /* per (bucket, block): requests, first slot; per block */
	uint64_t cap;                /* pool slots per block: W * h */
	uint32_t *req_off;           /* pool: entry offset inside the bucket */
	uint16_t *req_slot;          /*   frame * h + value inside the block */
	uint16_t *res;               /*   the entry read */
	unsigned long long *next;    /* resolve: next group of segments (zeroed before) */
};

__device__ __forceinline__ uint64_t mbk_find_read(const MbkArgs &b, uint64_t x)
{
	uint64_t lo = b.r0, hi = b.r0 + b.nr; /* fo[lo] - fo0 <= x < fo[hi] - fo0 */
	while (hi - lo > 1) {
		const uint64_t mid = lo + (hi - lo) / 2;
		if (b.fo[mid] - b.fo0 <= x)
			lo = mid;
		else
			hi = mid;
	}
	return lo;
}

/* In-place exclusive scan of v[0, n) in shared memory by the whole block
 * (blockDim.x == kMbkThreads); returns the total.  tmp: 33 words. */
__device__ uint32_t mbk_exscan(uint32_t *v, uint32_t n, uint32_t *tmp)
{
	const uint32_t t = threadIdx.x;
	const uint32_t per = (n + kMbkThreads - 1) / kMbkThreads;
	const uint32_t a0 = min(n, t * per), z = min(n, a0 + per);
	uint32_t sum = 0;
	for (uint32_t i = a0; i < z; ++i)
		sum += v[i];
	const uint32_t lane = t & 31u, wid = t >> 5;
	uint32_t inc = sum;
#pragma unroll
	for (uint32_t d = 1; d < 32; d <<= 1) {
		const uint32_t y = __shfl_up_sync(kFull, inc, d);
		if (lane >= d)
			inc += y;
	}
	if (lane == 31)
		tmp[wid] = inc;
	__syncthreads();
	if (wid == 0) {
		const uint32_t wv = lane < kMbkThreads / 32 ? tmp[lane] : 0u;
		uint32_t wi = wv;
#pragma unroll
		for (uint32_t d = 1; d < 32; d <<= 1) {
			const uint32_t y = __shfl_up_sync(kFull, wi, d);
			if (lane >= d)
				wi += y;
		}
		__syncwarp();
		tmp[lane] = wi - wv;
		if (lane == 31)
			tmp[32] = wi;
	}
	__syncthreads();
	uint32_t run = tmp[wid] + inc - sum;
	for (uint32_t i = a0; i < z; ++i) {
		const uint32_t x = v[i];
		v[i] = run;
		run += x;
	}
	const uint32_t total = tmp[32];
	__syncthreads();
	return total;
}

/* Shared memory of the hash kernel: seed tables, staged requests (offset,
 * bucket), their order by bucket, counts and first slots per bucket, validity
 * words. */
__host__ __device__ inline size_t mbk_hash_smem(uint32_t nse, uint32_t W, uint32_t h,
		uint32_t nbkt)
{
	const size_t req = (size_t)W * h;
	return (size_t)nse * kTabEntries * 16 + req * 4 + 2 * ((req * 2 + 15) & ~(size_t)15) +
			(size_t)nbkt * 8 + (size_t)(W / 32) * 4;
}

/* A thread's view of the packed bases of one mate array: the code and
 * validity words of the last frame fetched, reused while the next frame's
 * bases start in the same 16-base word.  frame() gives the 2-bit codes of 32
 * bases from base g (w, base j at bits 2j) and whether the k bases from g are
 * all ACGT. */
struct MbkCodes {
	uint64_t ci = ~0ull;
	uint32_t c0 = 0, c1 = 0, c2 = 0, v0 = 0, v1 = 0;

	__device__ __forceinline__ bool frame(const PackedBases &p, uint64_t g, unsigned k,
			uint64_t &w)
	{
		const uint64_t i = g >> 4;
		if (i != ci) {
			ci = i;
			c0 = i < p.nwords ? __ldg(p.words + i) : 0u;
			c1 = i + 1 < p.nwords ? __ldg(p.words + i + 1) : 0u;
			c2 = i + 2 < p.nwords ? __ldg(p.words + i + 2) : 0u;
			if (p.valid) {
				const uint64_t vi = g >> 5;
				v0 = vi < p.nvalid ? __ldg(p.valid + vi) : 0u;
				v1 = vi + 1 < p.nvalid ? __ldg(p.valid + vi + 1) : 0u;
			}
		}
		const uint32_t s = (uint32_t)(g & 15u) * 2u;
		const uint64_t lo = (uint64_t)c0 | ((uint64_t)c1 << 32);
		w = s ? (lo >> s) | ((uint64_t)c2 << (64u - s)) : lo;
		if (!p.valid)
			return true;
		/* validity bits g .. g + 31 (words g / 32 and g / 32 + 1, the same for
		 * every base of the 16-base word i) */
		const uint32_t v = __funnelshift_r(v0, v1, (uint32_t)(g & 31u));
		const uint32_t km = k >= 32 ? 0xffffffffu : ((1u << k) - 1u);
		return (~v & km) == 0;
	}
};

template <int H>
__global__ void __launch_bounds__(kMbkThreads) mbk_hash_kernel(MbkArgs b)
{
	extern __shared__ __align__(16) unsigned char smem[];
	const uint32_t nse = b.f.nse, h = b.f.h, W = b.W, k = b.f.k, t = threadIdx.x;
	const uint32_t blk = blockIdx.x, nreq = W * h;
	unsigned long long *tabw = reinterpret_cast<unsigned long long *>(smem);
	for (uint32_t i = t; i < nse * kTabEntries * 2; i += kMbkThreads)
		tabw[i] = b.tables[i];
	const ulonglong2 *tab = reinterpret_cast<const ulonglong2 *>(smem);
	uint32_t *st_off = reinterpret_cast<uint32_t *>(smem + (size_t)nse * kTabEntries * 16);
	uint16_t *st_bkt = reinterpret_cast<uint16_t *>(st_off + nreq);
	uint32_t *hist = reinterpret_cast<uint32_t *>(reinterpret_cast<unsigned char *>(st_bkt) +
			2 * (((size_t)nreq * 2 + 15) & ~(size_t)15));
	uint32_t *locs = hist + b.nbkt;
	uint32_t *vw = locs + b.nbkt;
	__shared__ uint32_t tmp[33];
	for (uint32_t q = t; q < b.nbkt; q += kMbkThreads)
		hist[q] = 0;
	for (uint32_t i = t; i < W / 32; i += kMbkThreads)
		vw[i] = 0;
	const uint64_t w0 = (uint64_t)blk * W;
	const uint64_t w1 = min(w0 + W, b.T);
	/* slots of frames past the sub-batch's end request nothing */
	for (uint32_t j = (uint32_t)(w1 - w0) * h + t; j < nreq; j += kMbkThreads)
		st_bkt[j] = 0xffffu;
	__syncthreads();
	const uint32_t R = W / kMbkThreads;
	const uint64_t x0 = w0 + (uint64_t)t * R;
	const unsigned sh = b.bshift;
	const uint64_t mask = (1ull << sh) - 1ull;
	if (x0 < w1) {
		const uint64_t x1 = min(x0 + R, w1);
		uint64_t r = mbk_find_read(b, x0);
		/* the read's frame range, base offsets and mate-1 frames, reloaded
		 * when the thread's frames move to the next read */
		uint64_t rs = b.fo[r] - b.fo0, re = b.fo[r + 1] - b.fo0;
		uint64_t o1 = b.off[r], o2 = b.off2 ? b.off2[r] : 0;
		uint64_t f1 = b.off[r + 1] - o1;
		f1 = f1 >= k ? f1 - k + 1 : 0;
		MbkCodes cc[2];
		for (uint64_t x = x0; x < x1; ++x) {
			while (re <= x) {
				++r;
				rs = re;
				re = b.fo[r + 1] - b.fo0;
				o1 = b.off[r];
				o2 = b.off2 ? b.off2[r] : 0;
				f1 = b.off[r + 1] - o1;
				f1 = f1 >= k ? f1 - k + 1 : 0;
			}
			const uint64_t q = x - rs;
			const uint32_t mate = q >= f1 ? 1u : 0u;
			const uint64_t g = mate ? o2 + (q - f1) : o1 + q;
			uint64_t w;
			const bool ok = cc[mate].frame(b.pk[mate], g, k, w);
			uint64_t vals[H];
			frame_values<H>(b.f, tab, ok, w, vals);
			const uint32_t fid = (uint32_t)(x - w0);
			if (ok)
				atomicOr(&vw[fid >> 5], 1u << (fid & 31u));
#pragma unroll
			for (int v = 0; v < H; ++v) {
				if (v < (int)h) {
					const uint32_t j = fid * h + v;
					if (ok) {
						const uint64_t pos = reduce(vals[v], b.f.m, b.f.minv);
						const uint32_t bk = (uint32_t)(pos >> sh);
						st_off[j] = (uint32_t)(pos & mask);
						st_bkt[j] = (uint16_t)bk;
						atomicAdd(&hist[bk], 1u);
					} else {
						st_bkt[j] = 0xffffu;
					}
				}
			}
		}
	}
	__syncthreads();
	const uint64_t vbase = w0 / 32, nv = (b.T + 31) / 32;
	for (uint32_t i = t; i < W / 32; i += kMbkThreads)
		if (vbase + i < nv)
			b.valid[vbase + i] = vw[i];
	for (uint32_t q = t; q < b.nbkt; q += kMbkThreads)
		locs[q] = hist[q];
	__syncthreads();
	const uint32_t total = mbk_exscan(locs, b.nbkt, tmp);
	if (t == 0)
		b.btot[blk] = total;
	for (uint32_t q = t; q < b.nbkt; q += kMbkThreads) {
		b.cnt[(uint64_t)q * b.nblk + blk] = hist[q];
		b.loc[(uint64_t)q * b.nblk + blk] = locs[q];
		hist[q] = 0;
	}
	__syncthreads();
	/* each request's place in bucket order (inv: place -> request), then the
	 * block's requests written out in that order, coalesced */
	uint16_t *inv = reinterpret_cast<uint16_t *>(reinterpret_cast<unsigned char *>(st_bkt) +
			(((size_t)nreq * 2 + 15) & ~(size_t)15));
	for (uint32_t j = t; j < nreq; j += kMbkThreads) {
		const uint32_t bk = st_bkt[j];
		if (bk != 0xffffu)
			inv[locs[bk] + atomicAdd(&hist[bk], 1u)] = (uint16_t)j;
	}
	__syncthreads();
	const uint64_t base = (uint64_t)blk * b.cap;
	for (uint32_t i = t; i < total; i += kMbkThreads) {
		const uint32_t j = inv[i];
		b.req_off[base + i] = st_off[j];
		b.req_slot[base + i] = (uint16_t)j;
	}
}

/* The (bucket, block) segments in bucket-major order, 32 consecutive segments
 * per warp taken from a work counter (every warp works at the front, so the
 * buckets in flight stay few), their requests 256 at a time, eight per lane in
 * flight; the bucket being read is held in L2, the pool streams through. */
__global__ void __launch_bounds__(256) mbk_resolve_kernel(MbkArgs b, const uint16_t *dense)
{
	__shared__ uint32_t spre[8][33];
	__shared__ unsigned long long sbase[8][32];
	__shared__ uint32_t sq[8][32];
	const uint32_t lane = threadIdx.x & 31u, wib = threadIdx.x >> 5;
	const uint64_t nseg = (uint64_t)b.nbkt * b.nblk;
	const uint64_t ngroups = (nseg + 31) / 32;
	const unsigned sh = b.bshift;
	for (;;) {
		unsigned long long g = 0;
		if (lane == 0)
			g = atomicAdd(b.next, 1ull);
		g = __shfl_sync(kFull, g, 0);
		if (g >= ngroups)
			break;
		const uint64_t sg = g * 32 + lane;
		uint32_t n = 0, lc = 0, q = 0, blk = 0;
		if (sg < nseg) {
			n = b.cnt[sg];
			lc = b.loc[sg];
			q = (uint32_t)(sg / b.nblk);
			blk = (uint32_t)(sg - (uint64_t)q * b.nblk);
		}
		uint32_t inc = n;
#pragma unroll
		for (uint32_t d = 1; d < 32; d <<= 1) {
			const uint32_t y = __shfl_up_sync(kFull, inc, d);
			if (lane >= d)
				inc += y;
		}
		const uint32_t total = __shfl_sync(kFull, inc, 31);
		spre[wib][lane] = inc - n;
		if (lane == 31)
			spre[wib][32] = inc;
		sbase[wib][lane] = (uint64_t)blk * b.cap + lc;
		sq[wib][lane] = q;
		__syncwarp();
		for (uint32_t c = 0; c < total; c += 256) {
			uint32_t off[8], qq[8];
			uint64_t idx[8];
#pragma unroll
			for (int j = 0; j < 8; ++j) {
				const uint32_t i = c + (uint32_t)j * 32 + lane;
				off[j] = 0;
				qq[j] = 0;
				idx[j] = ~0ull;
				if (i < total) {
					uint32_t lo = 0, hi = 32; /* spre[lo] <= i < spre[lo + 1] */
					while (hi - lo > 1) {
						const uint32_t mid = (lo + hi) >> 1;
						if (spre[wib][mid] <= i)
							lo = mid;
						else
							hi = mid;
					}
					idx[j] = sbase[wib][lo] + (i - spre[wib][lo]);
					qq[j] = sq[wib][lo];
					off[j] = __ldcs(b.req_off + idx[j]);
				}
			}
			uint16_t e[8];
#pragma unroll
			for (int j = 0; j < 8; ++j)
				e[j] = idx[j] != ~0ull ? __ldg(dense + (((uint64_t)qq[j] << sh) + off[j])) : 0;
#pragma unroll
			for (int j = 0; j < 8; ++j)
				if (idx[j] != ~0ull)
					__stcs(b.res + idx[j], e[j]);
		}
		__syncwarp();
	}
}

/* Per block: the entries read go to their slots (shared memory), then out to
 * the sub-batch's entry array in frame order; slots with no request (frames
 * not valid) stay 0. */
__global__ void __launch_bounds__(256) mbk_unscatter_kernel(MbkArgs b)
{
	extern __shared__ uint16_t se[];
	const uint32_t h = b.f.h, blk = blockIdx.x, t = threadIdx.x;
	const uint32_t nreq = b.W * h;
	for (uint32_t j = t; j < nreq; j += blockDim.x)
		se[j] = 0;
	__syncthreads();
	const uint64_t base = (uint64_t)blk * b.cap;
	const uint32_t n = b.btot[blk];
	for (uint32_t i = t; i < n; i += blockDim.x)
		se[__ldcs(b.req_slot + base + i)] = __ldcs(b.res + base + i);
	__syncthreads();
	const uint64_t w0 = (uint64_t)blk * b.W;
	const uint64_t w1 = min(w0 + b.W, b.T);
	const uint32_t m = (uint32_t)(w1 - w0) * h;
	for (uint32_t j = t; j < m; j += blockDim.x)
		b.e[w0 * h + j] = se[j];
}

/* fo_plus1[r] = frames of read (pair) r: both mates. */
__global__ void mbk_frames_kernel(const uint64_t *off, const uint64_t *off2, uint64_t n,
		unsigned k, uint64_t *fo_plus1)
{
	for (uint64_t r = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; r < n;
			r += (uint64_t)gridDim.x * blockDim.x) {
		const uint64_t l1 = off[r + 1] - off[r];
		const uint64_t l2 = off2 ? off2[r + 1] - off2[r] : 0;
		fo_plus1[r] = (l1 >= k ? l1 - k + 1 : 0) + (l2 >= k ? l2 - k + 1 : 0);
	}
}

} // namespace bbt

using namespace bbt;

#define MIBF_TRY(ctx, call)                                                                \
	do {                                                                                   \
		cudaError_t e_ = (call);                                                           \
		if (e_ != cudaSuccess)                                                             \
			return mibf_fail((ctx), e_ == cudaErrorMemoryAllocation ? BBT_ERR_NOMEM        \
					: BBT_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_));  \
	} while (0)

static uint32_t tally_slots(uint32_t nids)
{
	return (nids + 31) & ~31u;
}

static int pick_h(unsigned h)
{
	return h <= 1 ? 1 : h <= 2 ? 2 : h <= 3 ? 3 : h <= 4 ? 4 : h <= 6 ? 6 : h <= 8 ? 8 : 16;
}

/* Frames per lane per step (BBT_MIBF_FPL for the dense layout, whose probes
 * are single reads; one for the rank layout).  Two frames per lane measured
 * slower than one on the 500-target workload. */
#ifndef BBT_MIBF_FPL
#define BBT_MIBF_FPL 1
#endif
template <int H, bool D>
struct Fpl {
	static constexpr int value = (D && H <= 4) ? BBT_MIBF_FPL : 1;
};

template <int H, bool D, bool B, bool P = false>
static cudaError_t launch_h(const MibfArgs &a, int grid, size_t smem, cudaStream_t s)
{
	mibf_query_kernel<H, D, Fpl<H, D>::value, B, P><<<grid, kQueryThreads, smem, s>>>(a);
	return cudaGetLastError();
}

/* Blocks per SM of a variant with smem bytes of shared memory (also sets the
 * variant's shared-memory limit, which must precede its launch). */
template <int H, bool D, bool B, bool P = false>
static int occupancy_h(size_t smem)
{
	auto kern = mibf_query_kernel<H, D, Fpl<H, D>::value, B, P>;
	cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
	int nb = 0;
	cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, kern, kQueryThreads, smem);
	return nb > 0 ? nb : 1;
}

template <bool D, bool B, bool P = false>
static cudaError_t launch_query_db(const MibfArgs &a, int hsel, int grid, size_t smem,
		cudaStream_t s)
{
	switch (hsel) {
	case 1: return launch_h<1, D, B, P>(a, grid, smem, s);
	case 2: return launch_h<2, D, B, P>(a, grid, smem, s);
	case 3: return launch_h<3, D, B, P>(a, grid, smem, s);
	case 4: return launch_h<4, D, B, P>(a, grid, smem, s);
	case 6: return launch_h<6, D, B, P>(a, grid, smem, s);
	case 8: return launch_h<8, D, B, P>(a, grid, smem, s);
	default: return launch_h<16, D, B, P>(a, grid, smem, s);
	}
}

template <bool D, bool B, bool P = false>
static int query_occupancy_db(int hsel, size_t smem)
{
	switch (hsel) {
	case 1: return occupancy_h<1, D, B, P>(smem);
	case 2: return occupancy_h<2, D, B, P>(smem);
	case 3: return occupancy_h<3, D, B, P>(smem);
	case 4: return occupancy_h<4, D, B, P>(smem);
	case 6: return occupancy_h<6, D, B, P>(smem);
	case 8: return occupancy_h<8, D, B, P>(smem);
	default: return occupancy_h<16, D, B, P>(smem);
	}
}

/* pre: the bucketed query's tally kernel (dense layout only) */
static cudaError_t launch_query(const MibfArgs &a, bool dense, bool big, int hsel, int grid,
		size_t smem, cudaStream_t s, bool pre = false)
{
	if (pre)
		return big ? launch_query_db<true, true, true>(a, hsel, grid, smem, s)
		           : launch_query_db<true, false, true>(a, hsel, grid, smem, s);
	if (big)
		return dense ? launch_query_db<true, true>(a, hsel, grid, smem, s)
		             : launch_query_db<false, true>(a, hsel, grid, smem, s);
	return dense ? launch_query_db<true, false>(a, hsel, grid, smem, s)
	             : launch_query_db<false, false>(a, hsel, grid, smem, s);
}

static int query_occupancy(bool dense, bool big, int hsel, size_t smem, bool pre = false)
{
	if (pre)
		return big ? query_occupancy_db<true, true, true>(hsel, smem)
		           : query_occupancy_db<true, false, true>(hsel, smem);
	if (big)
		return dense ? query_occupancy_db<true, true>(hsel, smem)
		             : query_occupancy_db<false, true>(hsel, smem);
	return dense ? query_occupancy_db<true, false>(hsel, smem)
	             : query_occupancy_db<false, false>(hsel, smem);
}

/* Exclusive scan of n 64-bit counts into out (cub). */
static int scan_counts(bbt_mibf *ctx, const unsigned long long *in, unsigned long long *out,
		uint64_t n)
{
	size_t tmp_bytes = 0;
	cub::DeviceScan::ExclusiveSum(nullptr, tmp_bytes, in, out, (int64_t)n);
	void *tmp = nullptr;
	if (cudaMalloc(&tmp, tmp_bytes) != cudaSuccess)
		return mibf_fail(ctx, BBT_ERR_NOMEM, "cudaMalloc(scan)");
	cub::DeviceScan::ExclusiveSum(tmp, tmp_bytes, in, out, (int64_t)n);
	cudaError_t e = cudaDeviceSynchronize();
	cudaFree(tmp);
	if (e != cudaSuccess)
		return mibf_fail(ctx, BBT_ERR_CUDA, std::string("scan: ") + cudaGetErrorString(e));
	return BBT_OK;
}

/* Rank blocks (32 bytes per 224 bits) from the raw bit vector. */
static int build_blocks(bbt_mibf *ctx, const uint32_t *d_raw)
{
	const uint64_t m = ctx->hd.m, nwords = m / 32;
	const uint64_t nblocks = (m + kBlockBits - 1) / kBlockBits;
	const uint64_t nsuper = (nblocks >> kSuperShift) + 1;
	unsigned long long *d_pop = nullptr, *d_rank = nullptr;
	int rc = BBT_OK;
	if (cudaMalloc(&d_pop, nblocks * 8) != cudaSuccess ||
			cudaMalloc(&d_rank, nblocks * 8) != cudaSuccess ||
			cudaMalloc(&ctx->d_blocks, nblocks * 32) != cudaSuccess ||
			cudaMalloc(&ctx->d_super, nsuper * 8) != cudaSuccess)
		rc = mibf_fail(ctx, BBT_ERR_NOMEM, "cudaMalloc(rank blocks)");
	const int grid = ctx->num_sms * 8;
	if (rc == BBT_OK) {
		mibf_block_pop_kernel<<<grid, 256>>>(d_raw, nwords, nblocks, d_pop);
		rc = scan_counts(ctx, d_pop, d_rank, nblocks);
	}
	if (rc == BBT_OK) {
		mibf_block_build_kernel<<<grid, 256>>>(d_raw, nwords, nblocks, d_rank, ctx->d_super,
				ctx->d_blocks);
		cudaError_t e = cudaDeviceSynchronize();
		if (e != cudaSuccess)
			rc = mibf_fail(ctx, BBT_ERR_CUDA, std::string("rank blocks: ") +
					cudaGetErrorString(e));
	}
	cudaFree(d_pop);
	cudaFree(d_rank);
	return rc;
}

/* Dense ID map from the raw bit vector and the ID array. */
static int build_dense(bbt_mibf *ctx, const uint32_t *d_raw, const std::vector<uint16_t> &ids)
{
	const uint64_t m = ctx->hd.m, nw = m / 64, pop = ctx->hd.pop;
	unsigned long long *d_pop = nullptr, *d_rank = nullptr;
	uint16_t *d_ids = nullptr;
	int rc = BBT_OK;
	if (cudaMalloc(&d_pop, nw * 8) != cudaSuccess || cudaMalloc(&d_rank, nw * 8) != cudaSuccess ||
			cudaMalloc(&d_ids, std::max<uint64_t>(pop, 1) * 2) != cudaSuccess ||
			cudaMalloc(&ctx->d_dense, m * 2) != cudaSuccess)
		rc = mibf_fail(ctx, BBT_ERR_NOMEM, "cudaMalloc(dense ID map)");
	if (rc == BBT_OK && pop &&
			cudaMemcpy(d_ids, ids.data(), pop * 2, cudaMemcpyHostToDevice) != cudaSuccess)
		rc = mibf_fail(ctx, BBT_ERR_CUDA, "cudaMemcpy(IDs)");
	const int grid = ctx->num_sms * 8;
	if (rc == BBT_OK) {
		mibf_word_pop_kernel<<<grid, 256>>>((const uint64_t *)d_raw, nw, d_pop);
		rc = scan_counts(ctx, d_pop, d_rank, nw);
	}
	if (rc == BBT_OK) {
		mibf_dense_build_kernel<<<grid, 256>>>((const uint64_t *)d_raw, m, d_rank, d_ids,
				(uint32_t)ctx->names.size(), (uint32_t *)ctx->d_dense);
		cudaError_t e = cudaDeviceSynchronize();
		if (e != cudaSuccess)
			rc = mibf_fail(ctx, BBT_ERR_CUDA, std::string("dense ID map: ") +
					cudaGetErrorString(e));
	}
	cudaFree(d_pop);
	cudaFree(d_rank);
	cudaFree(d_ids);
	return rc;
}

/* Upload the bit vector, then build the layout the parameters ask for. */
static int load_device(bbt_mibf *ctx, const std::string &sdsl, const std::vector<uint16_t> &ids)
{
	const uint64_t m = ctx->hd.m, bytes = m / 8, pop = ctx->hd.pop;
	FILE *f = fopen(sdsl.c_str(), "rb");
	if (!f)
		return mibf_fail(ctx, BBT_ERR_IO, "Error: " + sdsl + " File cannot be opened");
	uint32_t *d_raw = nullptr;
	if (cudaMalloc(&d_raw, bytes) != cudaSuccess) {
		fclose(f);
		return mibf_fail(ctx, BBT_ERR_NOMEM, "cudaMalloc(bit vector)");
	}
	std::vector<char> buf(std::min<uint64_t>(bytes, 64ull << 20));
	int rc = BBT_OK;
	for (uint64_t done = 0; done < bytes && rc == BBT_OK;) {
		const size_t n = (size_t)std::min<uint64_t>(buf.size(), bytes - done);
		if (fread(buf.data(), 1, n, f) != n)
			rc = mibf_fail(ctx, BBT_ERR_FORMAT, sdsl + ": shorter than BitVectorSize / 8");
		else if (cudaMemcpy((char *)d_raw + done, buf.data(), n, cudaMemcpyHostToDevice) !=
				cudaSuccess)
			rc = mibf_fail(ctx, BBT_ERR_CUDA, "cudaMemcpy(bit vector)");
		done += n;
	}
	fclose(f);
	int layout = ctx->p.layout;
	if (rc == BBT_OK && layout == BBT_MIBF_LAYOUT_AUTO) {
		size_t free_b = 0, total_b = 0;
		cudaMemGetInfo(&free_b, &total_b);
		const double need = 2.0 * m + 2.0 * pop + m / 8.0 + (1ull << 30);
		layout = need < 0.7 * (double)free_b ? BBT_MIBF_LAYOUT_DENSE : BBT_MIBF_LAYOUT_RANK;
	}
	if (rc == BBT_OK && layout == BBT_MIBF_LAYOUT_DENSE) {
		rc = build_dense(ctx, d_raw, ids);
	} else if (rc == BBT_OK) {
		rc = build_blocks(ctx, d_raw);
		if (rc == BBT_OK && cudaMalloc(&ctx->d_ids, std::max<uint64_t>(pop, 1) * 2) != cudaSuccess)
			rc = mibf_fail(ctx, BBT_ERR_NOMEM, "cudaMalloc(IDs)");
		if (rc == BBT_OK && pop &&
				cudaMemcpy(ctx->d_ids, ids.data(), pop * 2, cudaMemcpyHostToDevice) != cudaSuccess)
			rc = mibf_fail(ctx, BBT_ERR_CUDA, "cudaMemcpy(IDs)");
	}
	cudaFree(d_raw);
	return rc;
}

/* Zeroed per-warp tally tables for a query grid of num_sms x
 * kMibfBigBlocksPerSm blocks (contexts with more than kMibfSmemIds IDs). */
static int alloc_gtally(bbt_mibf *ctx, unsigned long long **p, uint64_t *warps)
{
	const uint64_t T = tally_slots((uint32_t)ctx->names.size());
	const uint64_t w = (uint64_t)ctx->num_sms * kMibfBigBlocksPerSm * (kQueryThreads / 32);
	const size_t bytes = w * 3 * T * sizeof(unsigned long long);
	if (cudaMalloc(p, bytes) != cudaSuccess) {
		*p = nullptr;
		return mibf_fail(ctx, BBT_ERR_NOMEM, "cudaMalloc(per-warp tally tables, " +
				std::to_string(bytes >> 20) + " MB)");
	}
	if (cudaMemset(*p, 0, bytes) != cudaSuccess)
		return mibf_fail(ctx, BBT_ERR_CUDA, "cudaMemset(per-warp tally tables)");
	*warps = w;
	return BBT_OK;
}

static bool big_ids(const bbt_mibf *ctx)
{
	return ctx->names.size() > kMibfSmemIds;
}

extern "C" int bbt_mibf_close(bbt_mibf *ctx)
{
	if (!ctx)
		return BBT_OK;
	if (!ctx->host_only) {
		cudaSetDevice(ctx->dev);
		cudaFree(ctx->d_blocks);
		cudaFree(ctx->d_super);
		cudaFree(ctx->d_ids);
		cudaFree(ctx->d_dense);
		cudaFree(ctx->d_tables);
		cudaFree(ctx->d_counts);
		cudaFree(ctx->d_work);
		cudaFree(ctx->d_flags);
		cudaFree(ctx->d_stat);
		cudaFree(ctx->d_gtally);
		cudaFree(ctx->d_minc);
		cudaFree(ctx->d_fcmax);
		cudaFree(ctx->d_hits);
		cudaFree(ctx->d_nhits);
		cudaFree(ctx->d_sat);
		cudaFree(ctx->d_bk_fo);
		cudaFreeHost(ctx->h_bk_samples);
		cudaFree(ctx->d_bk_samples);
		for (int m = 0; m < 2; ++m) {
			cudaFree(ctx->d_bk_codes[m]);
			cudaFree(ctx->d_bk_cvalid[m]);
		}
		cudaFree(ctx->d_bk_valid);
		cudaFree(ctx->d_bk_e);
		cudaFree(ctx->d_bk_off);
		cudaFree(ctx->d_bk_slot);
		cudaFree(ctx->d_bk_res);
		cudaFree(ctx->d_bk_cnt);
		cudaFree(ctx->d_bk_loc);
		cudaFree(ctx->d_bk_btot);
		cudaFree(ctx->d_bk_tmp);
		for (int c = 0; c < 2; ++c) {
			for (int m = 0; m < 2; ++m) {
				cudaFree(ctx->c_seq[c][m]);
				cudaFree(ctx->c_valid[c][m]);
				cudaFree(ctx->c_off[c][m]);
				cudaFreeHost(ctx->h_coff[c][m]);
			}
			if (ctx->c_copied[c])
				cudaEventDestroy(ctx->c_copied[c]);
			if (ctx->c_computed[c])
				cudaEventDestroy(ctx->c_computed[c]);
		}
		if (ctx->h2d)
			cudaStreamDestroy(ctx->h2d);
		if (ctx->d2h)
			cudaStreamDestroy(ctx->d2h);
		if (ctx->ev0)
			cudaEventDestroy(ctx->ev0);
		if (ctx->ev1)
			cudaEventDestroy(ctx->ev1);
		if (ctx->stream)
			cudaStreamDestroy(ctx->stream);
	}
	delete ctx;
	return BBT_OK;
}

static size_t counts_len(const bbt_mibf *ctx)
{
	return 2 * (ctx->names.size() + 2) + 2;
}

extern "C" int bbt_mibf_open(const char *bf_path, const bbt_mibf_params *params, bbt_mibf **out)
{
	if (!out || !bf_path)
		return mibf_fail(nullptr, BBT_ERR_ARG, "bbt_mibf_open: need a path and an out pointer");
	*out = nullptr;
	int ndev = 0;
	if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
		return mibf_fail(nullptr, BBT_ERR_NODEVICE, "no CUDA device is available");
	bbt_mibf *ctx = new bbt_mibf();
	if (params)
		ctx->p = *params;
	else
		bbt_mibf_default_params(&ctx->p);
	ctx->dev = ctx->p.device;
	auto bail = [&](int rc) {
		mibf_fail(nullptr, rc, ctx->err);
		bbt_mibf_close(ctx);
		return rc;
	};
	if (cudaSetDevice(ctx->dev) != cudaSuccess) {
		ctx->host_only = true;
		mibf_fail(ctx, BBT_ERR_NODEVICE, "cannot use CUDA device " + std::to_string(ctx->dev));
		return bail(BBT_ERR_NODEVICE);
	}
	cudaDeviceGetAttribute(&ctx->num_sms, cudaDevAttrMultiProcessorCount, ctx->dev);
	std::vector<uint16_t> ids;
	int rc = mibf_load_host(ctx, bf_path, &ids);
	if (rc)
		return bail(rc);
	if (cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess ||
			cudaEventCreate(&ctx->ev0) != cudaSuccess || cudaEventCreate(&ctx->ev1) != cudaSuccess)
		return bail(mibf_fail(ctx, BBT_ERR_CUDA, "cannot create a stream"));
	rc = load_device(ctx, mibf_sdsl_path(bf_path), ids);
	if (rc)
		return bail(rc);
	std::vector<uint16_t>().swap(ids);
	std::vector<unsigned long long> tabs = mibf_seed_tables(ctx->hd.seeds, ctx->hd.k);
	if (BBT_MIBF_PAIR_TABLES) {
		/* pair entry (p, c0 | c1 << 2) = entry (2p, c0) ^ entry (2p + 1, c1) */
		const size_t nse = tabs.size() / (32 * 4 * 2);
		std::vector<unsigned long long> pairs(nse * 16 * 16 * 2, 0ull);
		for (size_t sd = 0; sd < nse; ++sd)
			for (int pp = 0; pp < 16; ++pp)
				for (int c = 0; c < 16; ++c)
					for (int half = 0; half < 2; ++half) {
						const unsigned long long *a0 = &tabs[((sd * 32 + 2 * pp) * 4 + (c & 3)) * 2];
						const unsigned long long *a1 =
								&tabs[((sd * 32 + 2 * pp + 1) * 4 + (c >> 2)) * 2];
						pairs[((sd * 16 + pp) * 16 + c) * 2 + half] = a0[half] ^ a1[half];
					}
		tabs.swap(pairs);
	}
	const size_t nc = counts_len(ctx) + 1; /* + reads */
	if (cudaMalloc(&ctx->d_tables, tabs.size() * 8) != cudaSuccess ||
			cudaMalloc(&ctx->d_counts, 2 * nc * 8) != cudaSuccess ||
			cudaMalloc(&ctx->d_work, 8) != cudaSuccess ||
			cudaMalloc(&ctx->d_flags, 4) != cudaSuccess ||
			cudaMalloc(&ctx->d_stat, 3 * 8) != cudaSuccess ||
			cudaMalloc(&ctx->d_fcmax, (1 + 2048) * 4) != cudaSuccess)
		return bail(mibf_fail(ctx, BBT_ERR_NOMEM, "cudaMalloc(context)"));
	cudaMemcpy(ctx->d_tables, tabs.data(), tabs.size() * 8, cudaMemcpyHostToDevice);
	cudaMemset(ctx->d_counts, 0, 2 * nc * 8);
	if (big_ids(ctx) && (rc = alloc_gtally(ctx, &ctx->d_gtally, &ctx->gtally_warps)) != BBT_OK)
		return bail(rc);
	if (cudaDeviceSynchronize() != cudaSuccess)
		return bail(mibf_fail(ctx, BBT_ERR_CUDA, "loading the miBF failed"));
	*out = ctx;
	return BBT_OK;
}

/* Make minCount rows present for the frame counts in fcs (sorted, unique). */
static int ensure_min_count(bbt_mibf *ctx, const std::vector<uint32_t> &fcs, cudaStream_t s)
{
	if (fcs.empty())
		return BBT_OK;
	const unsigned nids = (unsigned)ctx->names.size();
	const uint32_t need_rows = fcs.back() + 1;
	std::lock_guard<std::mutex> lk(ctx->mc_mu);
	if (ctx->minc_have.size() < need_rows) {
		ctx->minc_have.resize(need_rows, 0);
		ctx->h_minc.resize((size_t)need_rows * nids, 0);
	}
	std::vector<uint32_t> missing;
	for (uint32_t fc : fcs)
		if (fc && !ctx->minc_have[fc])
			missing.push_back(fc);
	if (missing.empty() && ctx->minc_rows >= need_rows)
		return BBT_OK;
	const long long nm = (long long)missing.size();
#pragma omp parallel for schedule(dynamic, 16)
	for (long long t = 0; t < nm * (long long)nids; ++t) {
		const uint32_t fc = missing[t / nids];
		const unsigned id = (unsigned)(t % nids);
		ctx->h_minc[(size_t)fc * nids + id] = id == 0 ? 0u
				: mibf_min_count(fc, ctx->frame_prob[id], ctx->p.score, nids);
	}
	for (uint32_t fc : missing)
		ctx->minc_have[fc] = 1;
	if (ctx->minc_rows < need_rows) {
		uint32_t rows = std::max<uint32_t>(need_rows, ctx->minc_rows * 2);
		rows = std::max<uint32_t>(rows, 256);
		uint32_t *d = nullptr;
		MIBF_TRY(ctx, cudaMalloc(&d, (size_t)rows * nids * 4));
		MIBF_TRY(ctx, cudaStreamSynchronize(s));
		cudaFree(ctx->d_minc);
		ctx->d_minc = d;
		ctx->minc_rows = rows;
		if (ctx->h_minc.size() < (size_t)rows * nids) {
			ctx->h_minc.resize((size_t)rows * nids, 0);
			ctx->minc_have.resize(rows, 0);
		}
		MIBF_TRY(ctx, cudaMemcpyAsync(d, ctx->h_minc.data(), (size_t)rows * nids * 4,
				cudaMemcpyHostToDevice, s));
		MIBF_TRY(ctx, cudaStreamSynchronize(s));
		return BBT_OK;
	}
	for (uint32_t fc : missing)
		MIBF_TRY(ctx, cudaMemcpyAsync(ctx->d_minc + (size_t)fc * nids,
				ctx->h_minc.data() + (size_t)fc * nids, nids * 4, cudaMemcpyHostToDevice, s));
	MIBF_TRY(ctx, cudaStreamSynchronize(s));
	return BBT_OK;
}

int bbt::mibf_reserve_rows(bbt_mibf *ctx, uint32_t rows)
{
	const unsigned nids = (unsigned)ctx->names.size();
	std::lock_guard<std::mutex> lk(ctx->mc_mu);
	if (ctx->minc_rows >= rows)
		return BBT_OK;
	uint32_t *d = nullptr;
	MIBF_TRY(ctx, cudaDeviceSynchronize());
	MIBF_TRY(ctx, cudaMalloc(&d, (size_t)rows * nids * 4));
	if (ctx->h_minc.size() < (size_t)rows * nids) {
		ctx->h_minc.resize((size_t)rows * nids, 0);
		ctx->minc_have.resize(rows, 0);
	}
	MIBF_TRY(ctx, cudaMemcpy(d, ctx->h_minc.data(), (size_t)rows * nids * 4,
			cudaMemcpyHostToDevice));
	cudaFree(ctx->d_minc);
	ctx->d_minc = d;
	ctx->minc_rows = rows;
	return BBT_OK;
}

static std::vector<uint32_t> host_frame_counts(const bbt_batch *b, unsigned k);

int bbt::mibf_rows_for(bbt_mibf *ctx, const uint64_t *off, const uint64_t *off2, uint64_t n)
{
	bbt_batch b;
	memset(&b, 0, sizeof b);
	b.offsets = off;
	b.offsets2 = off2;
	b.seq2 = off2 ? "" : nullptr;
	b.n_reads = n;
	std::vector<uint32_t> fcs = host_frame_counts(&b, ctx->hd.k);
	if (!fcs.empty() && fcs.back() >= ctx->minc_rows)
		return mibf_fail(ctx, BBT_ERR_ARG, "a read is longer than the minCount rows reserved "
				"for serving");
	return ensure_min_count(ctx, fcs, ctx->stream);
}

static std::vector<uint32_t> host_frame_counts(const bbt_batch *b, unsigned k)
{
	std::vector<uint32_t> fcs;
	std::vector<uint8_t> seen;
	for (uint64_t r = 0; r < b->n_reads; ++r) {
		const uint64_t l1 = b->offsets[r + 1] - b->offsets[r];
		const uint64_t l2 = b->seq2 ? b->offsets2[r + 1] - b->offsets2[r] : 0;
		const uint64_t fc = l1 >= k ? l1 - k + 1 : (l2 >= k ? l2 - k + 1 : 0);
		if (fc >= seen.size())
			seen.resize(fc + 1, 0);
		if (!seen[fc]) {
			seen[fc] = 1;
			fcs.push_back((uint32_t)fc);
		}
	}
	std::sort(fcs.begin(), fcs.end());
	return fcs;
}

static int device_frame_counts(bbt_mibf *ctx, const bbt_batch *b, cudaStream_t s,
		std::vector<uint32_t> &fcs)
{
	MIBF_TRY(ctx, cudaMemsetAsync(ctx->d_fcmax, 0, (1 + 2048) * 4, s));
	mibf_frame_counts_kernel<<<ctx->num_sms * 4, 256, 0, s>>>(b->offsets,
			b->seq2 ? b->offsets2 : nullptr, b->n_reads, ctx->hd.k, ctx->d_fcmax);
	std::vector<unsigned int> h(1 + 2048);
	MIBF_TRY(ctx, cudaMemcpyAsync(h.data(), ctx->d_fcmax, h.size() * 4, cudaMemcpyDeviceToHost,
			s));
	MIBF_TRY(ctx, cudaStreamSynchronize(s));
	const uint32_t mx = h[0];
	for (uint32_t fc = 0; fc < 65536 && fc <= mx; ++fc)
		if ((h[1 + (fc >> 5)] >> (fc & 31)) & 1u)
			fcs.push_back(fc);
	if (mx >= 65536) /* rare: rows for every longer count up to the maximum */
		for (uint32_t fc = 65536; fc <= mx; ++fc)
			fcs.push_back(fc);
	return BBT_OK;
}

/* Device scratch of at least n elements (contents not kept). */
template <class T>
static int mbk_grow(bbt_mibf *ctx, T **p, uint64_t &cap, uint64_t n)
{
	if (n <= cap)
		return BBT_OK;
	cudaFree(*p);
	*p = nullptr;
	cap = 0;
	MIBF_TRY(ctx, cudaMalloc(p, std::max<uint64_t>(n, 1) * sizeof(T)));
	cap = n;
	return BBT_OK;
}

template <int H>
static cudaError_t mbk_launch_hash(const MbkArgs &b, size_t smem, cudaStream_t s)
{
	cudaError_t e = cudaFuncSetAttribute(mbk_hash_kernel<H>,
			cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
	if (e != cudaSuccess)
		return e;
	mbk_hash_kernel<H><<<b.nblk, kMbkThreads, smem, s>>>(b);
	return cudaGetLastError();
}

static cudaError_t mbk_hash(const MbkArgs &b, int hsel, size_t smem, cudaStream_t s)
{
	switch (hsel) {
	case 1: return mbk_launch_hash<1>(b, smem, s);
	case 2: return mbk_launch_hash<2>(b, smem, s);
	case 3: return mbk_launch_hash<3>(b, smem, s);
	case 4: return mbk_launch_hash<4>(b, smem, s);
	case 6: return mbk_launch_hash<6>(b, smem, s);
	case 8: return mbk_launch_hash<8>(b, smem, s);
	default: return mbk_launch_hash<16>(b, smem, s);
	}
}

/* Whether a call of n reads takes the bucketed query. */
static bool mbk_wanted(const bbt_mibf *ctx, uint64_t n_reads)
{
	if (!ctx->d_dense || n_reads == 0 || ctx->bk_mode == 0)
		return false;
	return ctx->bk_mode == 1 || (2 * ctx->hd.m >= (256ull << 20) && n_reads >= (1ull << 20));
}

/*
 * The bucketed query of n reads (the dense layout): frame offsets and a host
 * plan of sub-batches (samples of the offsets, one short wait), the bases
 * packed, then per sub-batch hash -> resolve -> unscatter -> the query kernel
 * (PRE) over the sub-batch's reads, its results at their place in the call's
 * arrays and its counters added to the batch's.  *done = false when the plan
 * finds a read too long for any sub-batch (the caller then runs the direct
 * kernel).
 */
static int run_query_bucketed(bbt_mibf *ctx, const MibfArgs &a, int hsel, bool big, int grid,
		size_t smem, cudaStream_t s, bool *done)
{
	*done = false;
	const uint64_t n = a.n_reads;
	const unsigned k = a.f.k, h = a.f.h;
	if (mbk_grow(ctx, &ctx->d_bk_fo, ctx->bk_fo_cap, n + 1))
		return BBT_ERR_NOMEM;
	MIBF_TRY(ctx, cudaMemsetAsync(ctx->d_bk_fo, 0, 8, s));
	mbk_frames_kernel<<<ctx->num_sms * 8, 256, 0, s>>>(a.off, a.seq2 ? a.off2 : nullptr, n, k,
			ctx->d_bk_fo + 1);
	MIBF_TRY(ctx, cudaGetLastError());
	size_t tb = 0;
	MIBF_TRY(ctx, cub::DeviceScan::InclusiveSum(nullptr, tb, ctx->d_bk_fo + 1, ctx->d_bk_fo + 1,
			(int64_t)n, s));
	if (tb > ctx->bk_tmp_cap) {
		cudaFree(ctx->d_bk_tmp);
		ctx->d_bk_tmp = nullptr;
		ctx->bk_tmp_cap = 0;
		MIBF_TRY(ctx, cudaMalloc(&ctx->d_bk_tmp, tb));
		ctx->bk_tmp_cap = tb;
	}
	MIBF_TRY(ctx, cub::DeviceScan::InclusiveSum(ctx->d_bk_tmp, tb, ctx->d_bk_fo + 1,
			ctx->d_bk_fo + 1, (int64_t)n, s));
	/* fo[0], fo[S], ..., fo[n], then the end offset of each mate array; S reads
	 * per sample, fewer for small batches */
	const uint64_t S = std::min<uint64_t>(4096, std::max<uint64_t>(1, n / 256)), ns = n / S + 1;
	if (ns + 3 > ctx->bk_samples_cap) {
		cudaFreeHost(ctx->h_bk_samples);
		cudaFree(ctx->d_bk_samples);
		ctx->h_bk_samples = ctx->d_bk_samples = nullptr;
		ctx->bk_samples_cap = 0;
		MIBF_TRY(ctx, cudaMallocHost(&ctx->h_bk_samples, (ns + 3) * 8));
		MIBF_TRY(ctx, cudaMalloc(&ctx->d_bk_samples, (ns + 3) * 8));
		ctx->bk_samples_cap = ns + 3;
	}
	MIBF_TRY(ctx, launch_bk_samples(ctx->d_bk_fo, n, S, ctx->d_bk_samples, ns, ctx->num_sms, s));
	MIBF_TRY(ctx, launch_bk_samples(ctx->d_bk_fo + n, 0, 0, ctx->d_bk_samples + ns, 1,
			ctx->num_sms, s));
	const uint32_t mates = a.seq2 ? 2 : 1;
	const uint64_t *offm[2] = {a.off, a.off2};
	const uint8_t *seqm[2] = {a.seq, a.seq2};
	for (uint32_t m = 0; m < mates; ++m)
		MIBF_TRY(ctx, launch_bk_samples(offm[m] + n, 0, 0, ctx->d_bk_samples + ns + 1 + m, 1,
				ctx->num_sms, s));
	MIBF_TRY(ctx, cudaMemcpyAsync(ctx->h_bk_samples, ctx->d_bk_samples, (ns + 1 + mates) * 8,
			cudaMemcpyDeviceToHost, s));
	MIBF_TRY(ctx, cudaStreamSynchronize(s));
	const uint64_t *hs = ctx->h_bk_samples;
	struct Cut {
		uint64_t r0, r1, f0, f1;
	};
	std::vector<Cut> cuts;
	const uint64_t most = std::max<uint64_t>(ctx->bk_max_frames, 1ull << 16);
	auto pt = [&](uint64_t j) { return j < ns ? j * S : n; };
	for (uint64_t j = 0; pt(j) < n;) {
		uint64_t jj = j;
		while (jj + 1 <= ns && hs[jj + 1] - hs[j] <= most)
			++jj;
		if (jj == j)
			return BBT_OK; /* S reads above a sub-batch: the direct kernel */
		/* reads without frames still get their (empty) results and summary */
		cuts.push_back({pt(j), pt(jj), hs[j], hs[jj]});
		j = jj;
	}
	/* the bases as 2-bit codes */
	PackedBases pk[2];
	memset(pk, 0, sizeof pk);
	for (uint32_t m = 0; m < mates; ++m) {
		const uint64_t len = hs[ns + 1 + m];
		if (a.packed) { /* the batch's own code words and validity bits */
			pk[m].words = reinterpret_cast<const uint32_t *>(seqm[m]);
			pk[m].nwords = (len + 15) / 16;
			pk[m].valid = a.valid[m];
			pk[m].nvalid = a.valid[m] ? (len + 31) / 32 : 0;
			continue;
		}
		if (mbk_grow(ctx, &ctx->d_bk_codes[m], ctx->bk_codes_cap[m], 2 * (len / 32 + 2)) ||
				mbk_grow(ctx, &ctx->d_bk_cvalid[m], ctx->bk_cvalid_cap[m], len / 32 + 2))
			return BBT_ERR_NOMEM;
		MIBF_TRY(ctx, launch_bk_pack(seqm[m], len, ctx->d_bk_codes[m], ctx->d_bk_cvalid[m],
				ctx->num_sms, s));
		pk[m].words = ctx->d_bk_codes[m];
		pk[m].nwords = 2 * (len / 32 + 2);
		pk[m].valid = ctx->d_bk_cvalid[m];
		pk[m].nvalid = len / 32 + 2;
	}
	unsigned bshift = std::max<unsigned>(ctx->bk_bshift, 12);
	while (((ctx->hd.m + (1ull << bshift) - 1) >> bshift) > kMbkMaxBuckets)
		++bshift;
	const uint32_t nbkt = (uint32_t)((ctx->hd.m + (1ull << bshift) - 1) >> bshift);
	const uint32_t W = std::max<uint32_t>(kMbkThreads, kMbkRequests / h / kMbkThreads *
			kMbkThreads);
	const size_t hsmem = mbk_hash_smem(a.f.nse, W, h, nbkt);
	int res_per_sm = 0;
	MIBF_TRY(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&res_per_sm, mbk_resolve_kernel,
			256, 0));
	for (const Cut &c : cuts) {
		const uint64_t T = c.f1 - c.f0;
		const uint32_t nblk = (uint32_t)((T + W - 1) / W);
		const uint64_t cap = (uint64_t)W * h, pool = (uint64_t)nblk * cap;
		if (mbk_grow(ctx, &ctx->d_bk_valid, ctx->bk_valid_cap, T / 32 + 2) ||
				mbk_grow(ctx, &ctx->d_bk_e, ctx->bk_e_cap, T * h) ||
				mbk_grow(ctx, &ctx->d_bk_off, ctx->bk_off_cap, pool) ||
				mbk_grow(ctx, &ctx->d_bk_slot, ctx->bk_slot_cap, pool) ||
				mbk_grow(ctx, &ctx->d_bk_res, ctx->bk_res_cap, pool) ||
				mbk_grow(ctx, &ctx->d_bk_cnt, ctx->bk_cnt_cap, (uint64_t)nbkt * nblk) ||
				mbk_grow(ctx, &ctx->d_bk_loc, ctx->bk_loc_cap, (uint64_t)nbkt * nblk) ||
				mbk_grow(ctx, &ctx->d_bk_btot, ctx->bk_btot_cap, nblk))
			return BBT_ERR_NOMEM;
		MbkArgs b;
		memset(&b, 0, sizeof b);
		b.f = a.f;
		b.tables = a.tables;
		b.pk[0] = pk[0];
		b.pk[1] = pk[1];
		b.off = a.off;
		b.off2 = a.seq2 ? a.off2 : nullptr;
		b.r0 = c.r0;
		b.nr = c.r1 - c.r0;
		b.fo = ctx->d_bk_fo;
		b.fo0 = c.f0;
		b.T = T;
		b.W = W;
		b.nblk = nblk;
		b.nbkt = nbkt;
		b.bshift = bshift;
		b.valid = ctx->d_bk_valid;
		b.e = ctx->d_bk_e;
		b.cnt = ctx->d_bk_cnt;
		b.loc = ctx->d_bk_loc;
		b.btot = ctx->d_bk_btot;
		b.cap = cap;
		b.req_off = ctx->d_bk_off;
		b.req_slot = ctx->d_bk_slot;
		b.res = ctx->d_bk_res;
		if (T > 0) {
			MIBF_TRY(ctx, mbk_hash(b, hsel, hsmem, s));
			b.next = a.work;
			MIBF_TRY(ctx, cudaMemsetAsync(a.work, 0, 8, s));
			mbk_resolve_kernel<<<ctx->num_sms * std::max(res_per_sm, 1), 256, 0, s>>>(b,
					a.f.dense);
			MIBF_TRY(ctx, cudaGetLastError());
			mbk_unscatter_kernel<<<nblk, 256, cap * sizeof(uint16_t), s>>>(b);
			MIBF_TRY(ctx, cudaGetLastError());
		}
		MibfArgs q = a;
		q.n_reads = c.r1 - c.r0;
		q.off = a.off + c.r0;
		q.off2 = a.seq2 ? a.off2 + c.r0 : a.off2;
		q.hits = a.hits + c.r0 * a.max_hits;
		q.n_hits = a.n_hits + c.r0;
		q.sat = a.sat + c.r0;
		q.pre_e = ctx->d_bk_e;
		q.pre_valid = ctx->d_bk_valid;
		q.pre_fo = ctx->d_bk_fo + c.r0;
		q.pre_fo0 = c.f0;
		MIBF_TRY(ctx, cudaMemsetAsync(a.work, 0, 8, s));
		MIBF_TRY(ctx, launch_query(q, true, big, hsel, grid, smem, s, true));
	}
	*done = true;
	return BBT_OK;
}

/* A batch may be classified in several launches (chunks of its reads, their
 * results at their place in the batch's arrays): the first clears the batch's
 * counters and overflow flag, the last commits the counters. */
enum { kQueryBegin = 1, kQueryEnd = 2, kQueryWhole = 3 };

/* The bases of a call: ASCII, or 2-bit code words (bbt_batch BBT_BASES_2BIT)
 * with validity bits per mate array (NULL: every base is ACGT). */
struct MibfEncoding {
	bool packed = false;
	const uint32_t *valid[2] = {nullptr, nullptr};
};

static int run_query_sc(bbt_mibf *ctx, uint64_t n_reads, const uint8_t *seq, const uint64_t *off,
		const uint8_t *seq2, const uint64_t *off2, bbt_mibf_hit *hits, uint32_t max_hits,
		uint32_t *n_hits, uint32_t *sat, cudaStream_t s, const MibfScratch &sc, bool timed,
		int phase = kQueryWhole, uint64_t total_reads = ~0ull, MibfEncoding enc = MibfEncoding())
{
	if (total_reads == ~0ull)
		total_reads = n_reads;
	const unsigned nids = (unsigned)ctx->names.size();
	const size_t nc = counts_len(ctx);
	unsigned long long *batch_counts = sc.counts;
	MibfArgs a;
	a.f.blocks = ctx->d_blocks;
	a.f.super = ctx->d_super;
	a.f.ids = ctx->d_ids;
	a.f.dense = ctx->d_dense;
	a.f.m = ctx->hd.m;
	a.f.minv = ~0ull / ctx->hd.m;
	a.f.h = ctx->hd.h;
	a.f.k = ctx->hd.k;
	a.f.kmer_mode = ctx->hd.seeds.empty();
	a.f.nse = a.f.kmer_mode ? 1 : ctx->hd.h;
	a.f.nids = nids;
	a.seq = seq;
	a.off = off;
	a.seq2 = seq2;
	a.off2 = off2;
	a.packed = enc.packed ? 1 : 0;
	a.valid[0] = enc.valid[0];
	a.valid[1] = seq2 ? enc.valid[1] : enc.valid[0];
	a.n_reads = n_reads;
	a.minc = ctx->d_minc;
	a.need = ctx->need;
	a.min_nonsat = ctx->p.min_nonsat;
	a.best_agree = ctx->p.best_hit_agree;
	a.skip_empty_summary = (seq2 && ctx->p.hit_only) ? 1 : 0;
	a.multi = ctx->p.multi_thresh;
	a.tables = ctx->d_tables;
	a.hits = hits;
	a.max_hits = max_hits;
	a.n_hits = n_hits;
	a.sat = sat;
	a.counts = batch_counts;
	a.work = sc.work;
	a.flags = sc.flags;
	a.stat = sc.stat;
	a.T = tally_slots(nids);
	const bool big = big_ids(ctx);
	a.gtally = big ? sc.gtally : nullptr;
	const int hsel = pick_h(ctx->hd.h);
	const size_t smem = mibf_smem_bytes(a.f.nse, a.T, kQueryThreads / 32, big);
	const bool dense = ctx->d_dense != nullptr;
	int per_sm = query_occupancy(dense, big, hsel, smem);
	if (big)
		per_sm = std::min(per_sm, kMibfBigBlocksPerSm);
	const int grid = ctx->num_sms * per_sm;
	if (big && (!sc.gtally || (uint64_t)grid * (kQueryThreads / 32) > sc.gtally_warps))
		return mibf_fail(ctx, BBT_ERR_ARG, "the per-warp tally tables are missing or too small");
	if (phase & kQueryBegin) {
		MIBF_TRY(ctx, cudaMemsetAsync(batch_counts, 0, nc * 8, s));
		MIBF_TRY(ctx, cudaMemsetAsync(sc.flags, 0, 4, s));
		MIBF_TRY(ctx, cudaMemsetAsync(sc.stat, 0, 3 * 8, s));
		if (timed)
			MIBF_TRY(ctx, cudaEventRecord(ctx->ev0, s));
	}
	bool bucketed = false;
	if (sc.work == ctx->d_work && mbk_wanted(ctx, n_reads)) {
		const int pre_sm = query_occupancy(true, big, hsel, smem, true);
		const int pre_grid = ctx->num_sms * (big ? std::min(pre_sm, kMibfBigBlocksPerSm) : pre_sm);
		int rc = run_query_bucketed(ctx, a, hsel, big, pre_grid, smem, s, &bucketed);
		if (rc)
			return rc;
	}
	if (!bucketed) {
		MIBF_TRY(ctx, cudaMemsetAsync(sc.work, 0, 8, s));
		if (n_reads)
			MIBF_TRY(ctx, launch_query(a, dense, big, hsel, grid, smem, s));
	}
	if (phase & kQueryEnd) {
		if (timed)
			MIBF_TRY(ctx, cudaEventRecord(ctx->ev1, s));
		mibf_commit_kernel<<<1, 256, 0, s>>>(batch_counts, ctx->d_counts, (uint32_t)nc, sc.flags,
				total_reads);
		MIBF_TRY(ctx, cudaGetLastError());
	}
	return BBT_OK;
}

/* The context's own scratch (single-stream entry points). */
static MibfScratch ctx_scratch(bbt_mibf *ctx)
{
	MibfScratch sc;
	sc.work = ctx->d_work;
	sc.counts = ctx->d_counts + counts_len(ctx) + 1;
	sc.stat = ctx->d_stat;
	sc.flags = ctx->d_flags;
	sc.gtally = ctx->d_gtally;
	sc.gtally_warps = ctx->gtally_warps;
	return sc;
}

static MibfEncoding batch_encoding(const bbt_batch *b)
{
	MibfEncoding e;
	e.packed = b->encoding == BBT_BASES_2BIT;
	if (e.packed) {
		e.valid[0] = b->valid;
		e.valid[1] = b->valid2;
	}
	return e;
}

static int run_query(bbt_mibf *ctx, const bbt_batch *b, const uint8_t *seq, const uint64_t *off,
		const uint8_t *seq2, const uint64_t *off2, bbt_mibf_hit *hits, uint32_t max_hits,
		uint32_t *n_hits, uint32_t *sat, cudaStream_t s)
{
	return run_query_sc(ctx, b->n_reads, seq, off, seq2, off2, hits, max_hits, n_hits, sat, s,
			ctx_scratch(ctx), true, kQueryWhole, ~0ull, batch_encoding(b));
}

int bbt::mibf_scratch_init(bbt_mibf *ctx, MibfScratch &sc)
{
	MIBF_TRY(ctx, cudaSetDevice(ctx->dev));
	MIBF_TRY(ctx, cudaMalloc(&sc.work, 8));
	MIBF_TRY(ctx, cudaMalloc(&sc.counts, counts_len(ctx) * 8));
	MIBF_TRY(ctx, cudaMalloc(&sc.stat, 3 * 8));
	MIBF_TRY(ctx, cudaMalloc(&sc.flags, 4));
	if (big_ids(ctx))
		return alloc_gtally(ctx, &sc.gtally, &sc.gtally_warps);
	return BBT_OK;
}

void bbt::mibf_scratch_free(MibfScratch &sc)
{
	cudaFree(sc.work);
	cudaFree(sc.counts);
	cudaFree(sc.stat);
	cudaFree(sc.flags);
	cudaFree(sc.gtally);
	sc.gtally = nullptr;
	sc.gtally_warps = 0;
	sc = MibfScratch();
}

int bbt::mibf_classify_slot(bbt_mibf *ctx, uint64_t n, const uint8_t *seq, const uint64_t *off,
		const uint8_t *seq2, const uint64_t *off2, bbt_mibf_hit *hits, uint32_t max_hits,
		uint32_t *n_hits, uint32_t *sat, cudaStream_t s, MibfScratch &sc)
{
	return run_query_sc(ctx, n, seq, off, seq2, off2, hits, max_hits, n_hits, sat, s, sc, false);
}

/* Chunk slots of the host-batch pipeline, for chunks of up to `reads` reads
 * and `bases` bases per mate array. */
static int grow_chunks(bbt_mibf *ctx, uint64_t bases, uint64_t reads)
{
	if (!ctx->h2d) {
		MIBF_TRY(ctx, cudaStreamCreateWithFlags(&ctx->h2d, cudaStreamNonBlocking));
		MIBF_TRY(ctx, cudaStreamCreateWithFlags(&ctx->d2h, cudaStreamNonBlocking));
		for (int c = 0; c < 2; ++c) {
			MIBF_TRY(ctx, cudaEventCreateWithFlags(&ctx->c_copied[c], cudaEventDisableTiming));
			MIBF_TRY(ctx, cudaEventCreateWithFlags(&ctx->c_computed[c], cudaEventDisableTiming));
		}
	}
	if (bases <= ctx->c_bases_cap && reads <= ctx->c_reads_cap)
		return BBT_OK;
	const uint64_t nb = std::max(bases, ctx->c_bases_cap), nr = std::max(reads, ctx->c_reads_cap);
	MIBF_TRY(ctx, cudaDeviceSynchronize());
	ctx->c_bases_cap = ctx->c_reads_cap = 0;
	for (int c = 0; c < 2; ++c)
		for (int m = 0; m < 2; ++m) {
			cudaFree(ctx->c_seq[c][m]);
			cudaFree(ctx->c_valid[c][m]);
			cudaFree(ctx->c_off[c][m]);
			cudaFreeHost(ctx->h_coff[c][m]);
			ctx->c_seq[c][m] = nullptr;
			ctx->c_valid[c][m] = nullptr;
			ctx->c_off[c][m] = nullptr;
			ctx->h_coff[c][m] = nullptr;
			MIBF_TRY(ctx, cudaMalloc(&ctx->c_seq[c][m], std::max<uint64_t>(nb, 16)));
			/* packed batches: the chunk's validity words, from a 32-base boundary */
			MIBF_TRY(ctx, cudaMalloc(&ctx->c_valid[c][m], (nb / 32 + 4) * 4));
			MIBF_TRY(ctx, cudaMalloc(&ctx->c_off[c][m], (nr + 1) * 8));
			MIBF_TRY(ctx, cudaMallocHost(&ctx->h_coff[c][m], (nr + 1) * 8));
		}
	ctx->c_bases_cap = nb;
	ctx->c_reads_cap = nr;
	return BBT_OK;
}

/* Reads per chunk of the host-batch pipeline, and bases per mate array. */
constexpr uint64_t kChunkReads = 1ull << 20;
constexpr uint64_t kChunkBases = 256ull << 20;

/*
 * Host batch: the reads go in chunks through two slots.  Chunk c is
 * classified on the context's stream while chunk c + 1's bases and offsets
 * are copied in on a second stream and chunk c - 1's results go out on a
 * third, so the copies overlap the classification.  The chunks' launches
 * share the batch's counters, committed once after the last (none if a read
 * overflowed max_hits), so results and summary equal one launch's.
 */
static int classify_host_chunks(bbt_mibf *ctx, const bbt_batch *b, bbt_mibf_result *res,
		cudaStream_t s)
{
	const uint64_t n = b->n_reads;
	if (n == 0) {
		ctx->last_kernel_ms = 0;
		return BBT_OK;
	}
	const bool paired = b->seq2 != nullptr;
	const bool packed = b->encoding == BBT_BASES_2BIT;
	auto bases = [&](uint64_t lo, uint64_t hi) {
		uint64_t x = b->offsets[hi] - b->offsets[lo];
		if (paired)
			x = std::max(x, b->offsets2[hi] - b->offsets2[lo]);
		return x;
	};
	std::vector<uint64_t> cuts(1, 0);
	uint64_t most_reads = 1, most_bases = 16;
	while (cuts.back() < n) {
		const uint64_t r0 = cuts.back();
		uint64_t r1 = std::min(n, r0 + kChunkReads);
		if (r1 - r0 > 1 && bases(r0, r1) > kChunkBases) {
			uint64_t lo = r0 + 1, hi = r1;
			while (lo < hi) {
				const uint64_t mid = (lo + hi + 1) / 2;
				if (bases(r0, mid) <= kChunkBases)
					lo = mid;
				else
					hi = mid - 1;
			}
			r1 = lo;
		}
		most_reads = std::max(most_reads, r1 - r0);
		most_bases = std::max(most_bases, bases(r0, r1));
		cuts.push_back(r1);
	}
	int rc = grow_chunks(ctx, most_bases, most_reads);
	if (rc)
		return rc;
	/* device result arrays for the whole batch */
	if (n > ctx->res_cap_reads || res->max_hits > ctx->res_cap_hits ||
			n * res->max_hits > ctx->res_cap_reads * (uint64_t)ctx->res_cap_hits) {
		const uint64_t nr = std::max<uint64_t>(n, ctx->res_cap_reads);
		const uint32_t nh = std::max<uint32_t>(res->max_hits, ctx->res_cap_hits);
		cudaFree(ctx->d_hits);
		cudaFree(ctx->d_nhits);
		cudaFree(ctx->d_sat);
		ctx->d_hits = nullptr;
		ctx->d_nhits = ctx->d_sat = nullptr;
		ctx->res_cap_reads = 0;
		ctx->res_cap_hits = 0;
		MIBF_TRY(ctx, cudaMalloc(&ctx->d_hits, std::max<uint64_t>(nr * nh, 1) *
				sizeof(bbt_mibf_hit)));
		MIBF_TRY(ctx, cudaMalloc(&ctx->d_nhits, std::max<uint64_t>(nr, 1) * 4));
		MIBF_TRY(ctx, cudaMalloc(&ctx->d_sat, std::max<uint64_t>(nr, 1) * 4));
		ctx->res_cap_reads = nr;
		ctx->res_cap_hits = nh;
	}
	const size_t nchunks = cuts.size() - 1;
	/* input of chunk c into slot c % 2 (after the launch that last read it) */
	auto copy_in = [&](size_t c) -> int {
		const int sl = (int)(c & 1);
		const uint64_t r0 = cuts[c], r1 = cuts[c + 1], cnt = r1 - r0;
		if (c >= 2)
			MIBF_TRY(ctx, cudaStreamWaitEvent(ctx->h2d, ctx->c_computed[sl], 0));
		/* the pinned offsets of chunk c - 2 have been copied */
		MIBF_TRY(ctx, cudaEventSynchronize(ctx->c_copied[sl]));
		for (int m = 0; m < (paired ? 2 : 1); ++m) {
			const char *seq = m ? b->seq2 : b->seq;
			const uint64_t *off = m ? b->offsets2 : b->offsets;
			uint64_t *ho = ctx->h_coff[sl][m];
			/* packed: the chunk's code and validity words from the 32-base
			 * boundary at or before its first base */
			const uint64_t o0 = packed ? off[r0] & ~31ull : off[r0];
			for (uint64_t i = 0; i <= cnt; ++i)
				ho[i] = off[r0 + i] - o0;
			if (packed && off[r1] > o0) {
				const uint32_t *w = reinterpret_cast<const uint32_t *>(seq);
				const uint32_t *v = m ? b->valid2 : b->valid;
				MIBF_TRY(ctx, cudaMemcpyAsync(ctx->c_seq[sl][m], w + o0 / 16,
						(off[r1] - o0 + 15) / 16 * 4, cudaMemcpyHostToDevice, ctx->h2d));
				if (v)
					MIBF_TRY(ctx, cudaMemcpyAsync(ctx->c_valid[sl][m], v + o0 / 32,
							(off[r1] - o0 + 31) / 32 * 4, cudaMemcpyHostToDevice, ctx->h2d));
			} else if (off[r1] > o0) {
				MIBF_TRY(ctx, cudaMemcpyAsync(ctx->c_seq[sl][m], seq + o0, off[r1] - o0,
						cudaMemcpyHostToDevice, ctx->h2d));
			}
			MIBF_TRY(ctx, cudaMemcpyAsync(ctx->c_off[sl][m], ho, (cnt + 1) * 8,
					cudaMemcpyHostToDevice, ctx->h2d));
		}
		MIBF_TRY(ctx, cudaEventRecord(ctx->c_copied[sl], ctx->h2d));
		return BBT_OK;
	};
	for (int c = 0; c < 2; ++c) /* no copy is pending on either slot */
		MIBF_TRY(ctx, cudaEventRecord(ctx->c_copied[c], ctx->h2d));
	if (nchunks && (rc = copy_in(0)))
		return rc;
	const MibfScratch sc = ctx_scratch(ctx);
	for (size_t c = 0; c < nchunks; ++c) {
		const int sl = (int)(c & 1);
		const uint64_t r0 = cuts[c], cnt = cuts[c + 1] - r0;
		MIBF_TRY(ctx, cudaStreamWaitEvent(s, ctx->c_copied[sl], 0));
		const int phase = (c == 0 ? kQueryBegin : 0) | (c + 1 == nchunks ? kQueryEnd : 0);
		MibfEncoding enc;
		enc.packed = packed;
		enc.valid[0] = packed && b->valid ? ctx->c_valid[sl][0] : nullptr;
		enc.valid[1] = packed && paired && b->valid2 ? ctx->c_valid[sl][1] : nullptr;
		rc = run_query_sc(ctx, cnt, ctx->c_seq[sl][0], ctx->c_off[sl][0],
				paired ? ctx->c_seq[sl][1] : nullptr, paired ? ctx->c_off[sl][1] : nullptr,
				ctx->d_hits + r0 * res->max_hits, res->max_hits, ctx->d_nhits + r0,
				ctx->d_sat + r0, s, sc, true, phase, n, enc);
		if (rc)
			return rc;
		MIBF_TRY(ctx, cudaEventRecord(ctx->c_computed[sl], s));
		if (c + 1 < nchunks && (rc = copy_in(c + 1)))
			return rc;
		/* results of chunk c */
		MIBF_TRY(ctx, cudaStreamWaitEvent(ctx->d2h, ctx->c_computed[sl], 0));
		MIBF_TRY(ctx, cudaMemcpyAsync(res->n_hits + r0, ctx->d_nhits + r0, cnt * 4,
				cudaMemcpyDeviceToHost, ctx->d2h));
		MIBF_TRY(ctx, cudaMemcpyAsync(res->sat_count + r0, ctx->d_sat + r0, cnt * 4,
				cudaMemcpyDeviceToHost, ctx->d2h));
		if (res->max_hits)
			MIBF_TRY(ctx, cudaMemcpyAsync(res->hits + r0 * res->max_hits,
					ctx->d_hits + r0 * res->max_hits,
					cnt * res->max_hits * sizeof(bbt_mibf_hit), cudaMemcpyDeviceToHost, ctx->d2h));
	}
	unsigned int flag = 0;
	MIBF_TRY(ctx, cudaMemcpyAsync(&flag, ctx->d_flags, 4, cudaMemcpyDeviceToHost, s));
	MIBF_TRY(ctx, cudaStreamSynchronize(s));
	MIBF_TRY(ctx, cudaStreamSynchronize(ctx->d2h));
	MIBF_TRY(ctx, cudaStreamSynchronize(ctx->h2d));
	float ms = 0;
	cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
	ctx->last_kernel_ms = ms;
	if (flag)
		return mibf_fail(ctx, BBT_ERR_OVERFLOW, "a read has more significant IDs than max_hits");
	return BBT_OK;
}

extern "C" int bbt_mibf_classify_batch(bbt_mibf *ctx, const bbt_batch *b, bbt_mibf_result *res,
		void *stream)
{
	if (!ctx || !b || !res)
		return mibf_fail(ctx, BBT_ERR_ARG, "bbt_mibf_classify_batch: NULL argument");
	if (ctx->host_only)
		return mibf_fail(ctx, BBT_ERR_ARG, "context was opened without a device");
	if (b->n_reads && (!b->seq || !b->offsets || (b->seq2 && !b->offsets2)))
		return mibf_fail(ctx, BBT_ERR_ARG, "bbt_mibf_classify_batch: batch arrays missing");
	if (!res->n_hits || !res->sat_count || (res->max_hits && !res->hits))
		return mibf_fail(ctx, BBT_ERR_ARG, "bbt_mibf_classify_batch: result arrays missing");
	if (res->location != b->location)
		return mibf_fail(ctx, BBT_ERR_ARG, "batch and result must live on the same side");
	MIBF_TRY(ctx, cudaSetDevice(ctx->dev));
	cudaStream_t s = stream ? (cudaStream_t)stream : ctx->stream;
	int rc;
	if (b->location == BBT_DEVICE) {
		std::vector<uint32_t> fcs;
		rc = device_frame_counts(ctx, b, s, fcs);
		if (rc)
			return rc;
		rc = ensure_min_count(ctx, fcs, s);
		if (rc)
			return rc;
		return run_query(ctx, b, (const uint8_t *)b->seq, b->offsets, (const uint8_t *)b->seq2,
				b->offsets2, res->hits, res->max_hits, res->n_hits, res->sat_count, s);
	}
	/* host batch: chunks through two slots, copies overlapping the launches */
	rc = ensure_min_count(ctx, host_frame_counts(b, ctx->hd.k), s);
	if (rc)
		return rc;
	return classify_host_chunks(ctx, b, res, s);
}

extern "C" int bbt_mibf_sync(bbt_mibf *ctx)
{
	if (!ctx || ctx->host_only)
		return BBT_ERR_ARG;
	MIBF_TRY(ctx, cudaSetDevice(ctx->dev));
	MIBF_TRY(ctx, cudaStreamSynchronize(ctx->stream));
	MIBF_TRY(ctx, cudaDeviceSynchronize());
	float ms = 0;
	if (cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1) == cudaSuccess)
		ctx->last_kernel_ms = ms;
	unsigned int flag = 0;
	MIBF_TRY(ctx, cudaMemcpy(&flag, ctx->d_flags, 4, cudaMemcpyDeviceToHost));
	if (flag)
		return mibf_fail(ctx, BBT_ERR_OVERFLOW, "a read has more significant IDs than max_hits");
	return BBT_OK;
}

extern "C" int bbt_mibf_summary(bbt_mibf *ctx, uint64_t *counts, uint64_t *reads)
{
	if (!ctx || ctx->host_only)
		return BBT_ERR_ARG;
	MIBF_TRY(ctx, cudaSetDevice(ctx->dev));
	const size_t nc = counts_len(ctx);
	std::vector<uint64_t> h(nc + 1);
	MIBF_TRY(ctx, cudaDeviceSynchronize());
	MIBF_TRY(ctx, cudaMemcpy(h.data(), ctx->d_counts, (nc + 1) * 8, cudaMemcpyDeviceToHost));
	if (counts)
		memcpy(counts, h.data(), nc * 8);
	if (reads)
		*reads = h[nc];
	return BBT_OK;
}

extern "C" int bbt_mibf_reset_summary(bbt_mibf *ctx)
{
	if (!ctx || ctx->host_only)
		return BBT_ERR_ARG;
	MIBF_TRY(ctx, cudaSetDevice(ctx->dev));
	MIBF_TRY(ctx, cudaDeviceSynchronize());
	MIBF_TRY(ctx, cudaMemset(ctx->d_counts, 0, (counts_len(ctx) + 1) * 8));
	return BBT_OK;
}

extern "C" int bbt_mibf_summary_tsv(bbt_mibf *ctx, uint64_t read_count, char *buf, size_t cap,
		size_t *len)
{
	std::vector<uint64_t> c(counts_len(ctx));
	int rc = bbt_mibf_summary(ctx, c.data(), nullptr);
	if (rc)
		return rc;
	std::string s = mibf_summary_text(ctx->names, c, read_count);
	if (len)
		*len = s.size();
	if (buf && cap) {
		size_t n = std::min(cap - 1, s.size());
		memcpy(buf, s.data(), n);
		buf[n] = 0;
	}
	return BBT_OK;
}

extern "C" int bbt_mibf_set_bucketing(bbt_mibf *ctx, int mode, unsigned bucket_shift,
		uint64_t max_frames)
{
	if (!ctx || ctx->host_only)
		return BBT_ERR_ARG;
	if (mode < 0 || mode > 2)
		return mibf_fail(ctx, BBT_ERR_ARG, "bbt_mibf_set_bucketing: mode must be 0, 1 or 2");
	if (bucket_shift && (bucket_shift < 12 || bucket_shift > 40))
		return mibf_fail(ctx, BBT_ERR_ARG, "bbt_mibf_set_bucketing: bucket_shift must be in "
				"[12, 40]");
	if (mode == 1 && !ctx->d_dense)
		return mibf_fail(ctx, BBT_ERR_UNSUPPORTED, "bbt_mibf_set_bucketing: the bucketed query "
				"reads the dense layout");
	MIBF_TRY(ctx, cudaSetDevice(ctx->dev));
	MIBF_TRY(ctx, cudaDeviceSynchronize());
	ctx->bk_mode = mode;
	if (bucket_shift)
		ctx->bk_bshift = bucket_shift;
	if (max_frames)
		ctx->bk_max_frames = max_frames;
	return BBT_OK;
}

extern "C" int bbt_mibf_layout(const bbt_mibf *ctx)
{
	if (!ctx || ctx->host_only)
		return BBT_ERR_ARG;
	return ctx->d_dense ? BBT_MIBF_LAYOUT_DENSE : BBT_MIBF_LAYOUT_RANK;
}

extern "C" int bbt_mibf_last_counts(bbt_mibf *ctx, uint64_t *out)
{
	if (!ctx || ctx->host_only || !out)
		return BBT_ERR_ARG;
	MIBF_TRY(ctx, cudaSetDevice(ctx->dev));
	MIBF_TRY(ctx, cudaDeviceSynchronize());
	MIBF_TRY(ctx, cudaMemcpy(out, ctx->d_stat, 3 * 8, cudaMemcpyDeviceToHost));
	return BBT_OK;
}

/* Device time of the last batch's query kernel, in ms. */
extern "C" double bbt_mibf_last_kernel_ms(bbt_mibf *ctx)
{
	return ctx ? ctx->last_kernel_ms : 0.0;
}
