/*
 * bucketed.cu -- the bucketed probe path, for filters much larger than L2.
 *
 * Every Bloom probe is an isolated 4-byte read at a random bit of the filter.
 * When the filter is gigabytes, each such read is a DRAM line fill, and the
 * read-major kernels (classify.cu) are bound by how many of those the memory
 * system serves (about 42 G random reads per second on B200).  This path makes
 * the probes of many reads at once and sorts them by filter address before
 * making them: the filter is cut into buckets of 2^bshift bits that fit L2,
 * each bucket's requests are resolved together, and every line of the bucket
 * is fetched from DRAM about once per round instead of once per probe.
 *
 * The decisions are SeqEval's (Common/SeqEval.h:37-114 and the other scoring
 * methods) exactly: BloomFilter::contains is the AND of h bit tests, made
 * level by level (level l only for frames whose tests 0..l-1 all passed, as
 * contains() short-circuits; or several levels per round when so set, a frame
 * staying a hit only when all pass), and the state machine of
 * seqeval_chunk.cuh then walks each read over the resolved hit bits.  The walk
 * consumes only contains() results, so making more tests than the sequential
 * loop would (frames after a decision, frames in skip windows, a second level
 * after a failed first) changes no result.
 *
 * To keep those extra tests few, a read's frames are resolved in phases: the
 * first phase covers a prefix of every read (most reads that match are
 * accepted early), the next the rest of the reads still undecided.  Per phase:
 *   hash   -- per window block (kBkWinFrames frames of the sub-batch): the
 *             phase's frames of the open reads are shared out evenly among
 *             the block's threads, each rolling ntHash over its share (2-bit
 *             codes, 16 bases per load); a frame's validity, hit and
 *             requesting bits are set, its canonical hash kept, and its
 *             requests of the round's levels counted per bucket, then written
 *             to the block's region of the request pool in bucket order;
 *   resolve-- the (bucket, block) segments in bucket-major order, one warp per
 *             segment: each request's bit is tested out of the bucket held in
 *             L2, its result written as a byte beside it (the frames' hit
 *             bits, spread over the whole sub-batch, are not touched here, so
 *             that the bucket keeps L2 to itself);
 *   emit   -- (the later rounds) per block, the previous round's results
 *             clear the hit bits of the frames that failed, then the frames
 *             still hits request their next levels from their kept hashes,
 *             as above, then resolve;
 * and after the last round (its results applied the same way) one thread per
 * undecided read walks SeqEval over [0, phase end) of its frames.
 */
#include "bucketed.cuh"

#include "bbt.h"
#include "seqeval_chunk.cuh"
#include "window.cuh"

namespace bbt {

namespace {

constexpr uint32_t kNT = kBkWinThreads;
constexpr uint32_t kRun = kBkWinFrames / kNT;  /* frames per counting run: 128 */
constexpr uint32_t kWinWords = kBkWinFrames / 32;
constexpr uint32_t kMaxBuckets = 2048;
static_assert(kBkWinFrames % kNT == 0 && kNT % 32 == 0, "whole runs and warps");

/* First frame of phase boundary q (sixteenths) of a read of F frames. */
__device__ __forceinline__ uint64_t bk_bound(uint64_t F, uint32_t q, uint32_t pmin)
{
	if (q == 0)
		return 0;
	if (q >= kBkPhaseDen)
		return F;
	uint64_t b = (F * q + kBkPhaseDen - 1) / kBkPhaseDen;
	if (b < pmin)
		b = pmin;
	return b < F ? b : F;
}

/* The read (index in the batch's read space) holding sub-batch frame x. */
__device__ __forceinline__ uint64_t bk_find_read(const BucketArgs &b, uint64_t x)
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

/* The phase's frames of read r, clipped to [lo, hi) (sub-batch frames):
 * [pa, pb), empty (pa >= pb) when the read is decided. */
__device__ __forceinline__ void bk_piece(const BucketArgs &b, uint64_t r, uint64_t lo, uint64_t hi,
		uint64_t &pa, uint64_t &pb)
{
	const uint64_t fr0 = b.fo[r] - b.fo0, F = b.fo[r + 1] - b.fo[r];
	pa = max(lo, fr0 + bk_bound(F, b.ph_lo, b.ph_min));
	pb = min(hi, fr0 + bk_bound(F, b.ph_hi, b.ph_min));
	if (b.state[r])
		pb = pa;
}

__device__ __forceinline__ uint64_t seed_fw_code(uint8_t c)
{
	return c == 0 ? kSeedA : c == 1 ? kSeedC : c == 2 ? kSeedG : c == 3 ? kSeedT : 0ull;
}

__device__ __forceinline__ uint64_t seed_rc_code(uint8_t c)
{
	return c == 0 ? kSeedT : c == 1 ? kSeedG : c == 2 ? kSeedC : c == 3 ? kSeedA : 0ull;
}

/* 32 bits of a bit array from bit x on (the array has a spare word at its end). */
__device__ __forceinline__ uint32_t bits_at(const uint32_t *w, uint64_t x)
{
	const uint64_t i = x >> 5;
	const uint32_t s = (uint32_t)(x & 31u);
	const uint32_t lo = w[i];
	return s ? (lo >> s) | (w[i + 1] << (32u - s)) : lo;
}

/* ntHash rolling tables of one k, indexed by (code of the base leaving the
 * k-mer) << 3 | (code of the base entering it), codes 0..3 for ACGT and 4 for
 * any other base or for no base (seed 0):
 *   tf[o, i] = rol(seed_fw(o), k) ^ seed_fw(i)
 *   tr[o, i] = ror(seed_rc(o), 1) ^ rol(seed_rc(i), k - 1)
 * so that a step is fh = rol(fh, 1) ^ tf, rh = ror(rh, 1) ^ tr.  From
 * fh = rh = 0, k steps with no base leaving give the hashes of the first
 * k-mer: fh = XOR_j rol(seed_fw(s_j), k-1-j), rh = XOR_j rol(seed_rc(s_j), j). */
struct RollTables {
	uint64_t tf[64];
	uint64_t tr[64];
};

__device__ void bk_set_tables(RollTables &t, unsigned k)
{
	for (int e = threadIdx.x; e < 64; e += blockDim.x) {
		const uint8_t o = (uint8_t)(e >> 3), i = (uint8_t)(e & 7);
		t.tf[e] = rolk(seed_fw_code(o), k) ^ seed_fw_code(i);
		t.tr[e] = ror1(seed_rc_code(o)) ^ rolk(seed_rc_code(i), k - 1);
	}
}

/* Codes (2 bits per base) and non-ACGT flags (1 bit per base) of 16 bases
 * from base g >= 0 of a packed mate array. */
__device__ __forceinline__ void codes16_at(const PackedBases &p, uint64_t g, uint32_t &c,
		uint32_t &bad)
{
	const uint64_t w = g >> 4;
	const uint32_t lo = w < p.nwords ? __ldg(p.words + w) : 0u;
	const uint32_t hi = w + 1 < p.nwords ? __ldg(p.words + w + 1) : 0u;
	c = __funnelshift_r(lo, hi, (uint32_t)(g & 15u) * 2u);
	if (p.valid) {
		const uint64_t v = g >> 5;
		const uint32_t vlo = v < p.nvalid ? __ldg(p.valid + v) : 0u;
		const uint32_t vhi = v + 1 < p.nvalid ? __ldg(p.valid + v + 1) : 0u;
		bad = ~__funnelshift_r(vlo, vhi, (uint32_t)(g & 31u)) & 0xFFFFu;
	} else {
		bad = 0;
	}
}

/* The same from base g, which may lie before the array (those bases flagged). */
__device__ __forceinline__ void codes16(const PackedBases &p, int64_t g, uint32_t &c, uint32_t &bad)
{
	if (g >= 0) {
		codes16_at(p, (uint64_t)g, c, bad);
		return;
	}
	const int64_t d = -g;
	if (d >= 16) {
		c = 0;
		bad = 0xFFFFu;
		return;
	}
	uint32_t c0, b0;
	codes16_at(p, 0, c0, b0);
	c = c0 << (2u * (uint32_t)d);
	bad = ((b0 << (uint32_t)d) | ((1u << (uint32_t)d) - 1u)) & 0xFFFFu;
}

/* Four ASCII bytes: their 2-bit codes (A0 C1 G2 T3, by bits 1-2 of the byte)
 * in bits 0-7 and a nibble of ACGT flags. */
__device__ __forceinline__ void ascii4(uint32_t w, uint32_t &c8, uint32_t &ok4)
{
	const uint32_t t = ((w >> 1) & 0x03030303u) ^ ((w >> 2) & 0x01010101u);
	c8 = (t & 3u) | ((t >> 6) & 0xCu) | ((t >> 12) & 0x30u) | ((t >> 18) & 0xC0u);
	const uint32_t u = w & 0xDFDFDFDFu;
	const uint32_t v = __vcmpeq4(u, 0x41414141u) | __vcmpeq4(u, 0x43434343u) |
			__vcmpeq4(u, 0x47474747u) | __vcmpeq4(u, 0x54545454u);
	ok4 = ((v >> 7) & 1u) | ((v >> 14) & 2u) | ((v >> 21) & 4u) | ((v >> 28) & 8u);
}

/* One thread per 32 bases: code words 2j, 2j + 1 and validity word j.  Bases
 * at or past len are flagged and coded 0. */
__global__ void bk_pack_kernel(const uint8_t *ascii, uint64_t len, uint32_t *words,
		uint32_t *valid, uint64_t nvalid)
{
	const bool vec = (reinterpret_cast<uintptr_t>(ascii) & 15u) == 0;
	for (uint64_t j = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; j < nvalid;
			j += (uint64_t)gridDim.x * blockDim.x) {
		uint32_t ok = 0;
		for (uint32_t h = 0; h < 2; ++h) {
			const uint64_t g = j * 32 + h * 16;
			uint32_t q[4] = {0, 0, 0, 0};
			if (vec && g + 16 <= len) {
				const uint4 v = __ldg(reinterpret_cast<const uint4 *>(ascii + g));
				q[0] = v.x;
				q[1] = v.y;
				q[2] = v.z;
				q[3] = v.w;
			} else {
				for (uint32_t i = 0; i < 16 && g + i < len; ++i)
					q[i >> 2] |= (uint32_t)ascii[g + i] << (8u * (i & 3u));
			}
			uint32_t code = 0, ok16 = 0;
			for (uint32_t i = 0; i < 4; ++i) {
				uint32_t c8, k4;
				ascii4(q[i], c8, k4);
				code |= c8 << (8u * i);
				ok16 |= k4 << (4u * i);
			}
			if (g + 16 > len) { /* past the end: flagged, code 0 */
				const uint32_t keep = g >= len ? 0u : (1u << (uint32_t)(len - g)) - 1u;
				ok16 &= keep;
				code &= g >= len ? 0u : (uint32_t)((1ull << (2u * (uint32_t)(len - g))) - 1u);
			}
			words[2 * j + h] = code;
			ok |= ok16 << (16u * h);
		}
		valid[j] = ok;
	}
}

/* In-place exclusive scan of v[0, n) in shared memory by the whole block
 * (blockDim.x == kNT); returns the total.  tmp: 33 words of shared memory. */
__device__ uint32_t block_exscan(uint32_t *v, uint32_t n, uint32_t *tmp)
{
	const uint32_t t = threadIdx.x;
	const uint32_t per = (n + kNT - 1) / kNT;
	const uint32_t a = min(n, t * per), z = min(n, a + per);
	uint32_t sum = 0;
	for (uint32_t i = a; i < z; ++i)
		sum += v[i];
	const uint32_t lane = t & 31u, wid = t >> 5;
	uint32_t inc = sum;
#pragma unroll
	for (uint32_t d = 1; d < 32; d <<= 1) {
		const uint32_t y = __shfl_up_sync(0xffffffffu, inc, d);
		if (lane >= d)
			inc += y;
	}
	if (lane == 31)
		tmp[wid] = inc;
	__syncthreads();
	if (wid == 0) {
		const uint32_t wv = lane < kNT / 32 ? tmp[lane] : 0u;
		uint32_t wi = wv;
#pragma unroll
		for (uint32_t d = 1; d < 32; d <<= 1) {
			const uint32_t y = __shfl_up_sync(0xffffffffu, wi, d);
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
	for (uint32_t i = a; i < z; ++i) {
		const uint32_t x = v[i];
		v[i] = run;
		run += x;
	}
	const uint32_t total = tmp[32];
	__syncthreads();
	return total;
}

/* Shared memory of the hash / emit kernels: the block's validity and
 * requesting bits, counts and first slots of nbkt buckets. */
struct SweepSmem {
	uint32_t *sv, *sa, *hist, *loc;
	__device__ __forceinline__ SweepSmem(uint32_t *base, uint32_t nbkt)
	{
		sv = base;
		sa = base + kWinWords;
		hist = sa + kWinWords;
		loc = hist + nbkt;
	}
};

/* After the block's requests are counted into sm.hist: their first slots per
 * bucket (into sm.loc and the global cnt / loc tables), then each requesting
 * frame of the block writes its requests of levels [level, level + nlevels) to
 * its bucket's slots.  The canonical hashes are read back from b.canon. */
__device__ void bk_scatter(const BucketArgs &b, const SweepSmem &sm, uint32_t *tmp)
{
	const uint32_t blk = blockIdx.x, t = threadIdx.x;
	for (uint32_t q = t; q < b.nbkt; q += kNT)
		sm.loc[q] = sm.hist[q];
	__syncthreads();
	const uint32_t total = block_exscan(sm.loc, b.nbkt, tmp);
	if (t == 0)
		b.btot[blk] = total;
	for (uint32_t q = t; q < b.nbkt; q += kNT) {
		b.cnt[(uint64_t)q * b.nblk + blk] = sm.hist[q];
		b.loc[(uint64_t)q * b.nblk + blk] = sm.loc[q];
		sm.hist[q] = 0;
	}
	__syncthreads();
	const uint64_t w0 = (uint64_t)blk * kBkWinFrames;
	const uint64_t base = (uint64_t)blk * b.cap;
	const unsigned sh = b.bshift, k = b.f.k;
	const uint64_t mask = (1ull << sh) - 1ull;
	const uint32_t lane = t & 31u;
	for (uint32_t w = t >> 5; w < kWinWords; w += kNT / 32) {
		const uint32_t am = sm.sa[w];
		if (!((am >> lane) & 1u))
			continue;
		const uint32_t fid = w * 32 + lane;
		const uint64_t canon = b.canon[w0 + fid];
		for (uint32_t l = b.level; l < b.level + b.nlevels; ++l) {
			const uint64_t pos = reduce(l ? extra_hash(canon, k, l) : canon, b.f.m, b.f.minv);
			const uint32_t q = (uint32_t)(pos >> sh);
			const uint64_t i = base + sm.loc[q] + atomicAdd(&sm.hist[q], 1u);
			b.req_off[i] = (uint32_t)(pos & mask);
			b.req_fid[i] = (uint16_t)fid;
		}
	}
}

/*
 * A phase's first round, per window block [w0, w1) of the sub-batch:
 *  1. each thread counts the phase's frames of open reads in its run of kRun
 *     frames, and a block scan numbers them 0..A-1 in frame order;
 *  2. thread t takes frames [A t / kNT, A (t + 1) / kNT) of that numbering,
 *     finds the first (its run by binary search over the scan, then the read
 *     by walking the run) and rolls ntHash through them read piece by read
 *     piece (k steps with no base leaving start each piece), setting the
 *     frames' validity and requesting bits, keeping the canonical hash of each
 *     requesting frame (valid, not DUST-masked) and counting its requests of
 *     levels [0, nlevels) per bucket;
 *  3. the bits go to the sub-batch arrays (this phase's frames are new there,
 *     so hit bits start equal to the requesting bits), then bk_scatter.
 */
__global__ void __launch_bounds__(kNT) bk_hash_kernel(BucketArgs b)
{
	extern __shared__ uint32_t bk_sm[];
	const SweepSmem sm(bk_sm, b.nbkt);
	__shared__ uint32_t pre[kNT + 1];
	__shared__ uint32_t tmp[33];
	__shared__ RollTables tab;
	const uint32_t blk = blockIdx.x, t = threadIdx.x;
	const uint64_t w0 = (uint64_t)blk * kBkWinFrames;
	const uint64_t w1 = min(w0 + kBkWinFrames, b.T);
	bk_set_tables(tab, b.f.k);
	for (uint32_t w = t; w < kWinWords; w += kNT)
		sm.sv[w] = sm.sa[w] = 0;
	for (uint32_t q = t; q < b.nbkt; q += kNT)
		sm.hist[q] = 0;

	/* 1 */
	const uint64_t end_r = b.r0 + b.nr;
	uint32_t c = 0;
	{
		const uint64_t x0 = w0 + (uint64_t)t * kRun;
		if (x0 < w1) {
			const uint64_t x1 = min(x0 + kRun, w1);
			for (uint64_t r = bk_find_read(b, x0); r < end_r && b.fo[r] - b.fo0 < x1; ++r) {
				uint64_t pa, pb;
				bk_piece(b, r, x0, x1, pa, pb);
				if (pa < pb)
					c += (uint32_t)(pb - pa);
			}
		}
	}
	pre[t] = c;
	__syncthreads();
	const uint32_t A = block_exscan(pre, kNT, tmp);
	if (t == 0)
		pre[kNT] = A;
	__syncthreads();

	/* 2 */
	const uint32_t s0 = (uint32_t)((uint64_t)A * t / kNT);
	const uint32_t s1 = (uint32_t)((uint64_t)A * (t + 1) / kNT);
	const unsigned k = b.f.k;
	uint32_t cw = 0xffffffffu, vacc = 0, aacc = 0;
	if (s0 < s1) {
		uint32_t lo = 0, hi = kNT; /* pre[lo] <= s0 < pre[lo + 1] */
		while (hi - lo > 1) {
			const uint32_t mid = (lo + hi) >> 1;
			if (pre[mid] <= s0)
				lo = mid;
			else
				hi = mid;
		}
		uint32_t o = s0 - pre[lo];
		const uint64_t x0 = w0 + (uint64_t)lo * kRun, x1 = min(x0 + kRun, w1);
		uint64_t r = bk_find_read(b, x0), xs = x1;
		for (; r < end_r && b.fo[r] - b.fo0 < x1; ++r) {
			uint64_t pa, pb;
			bk_piece(b, r, x0, x1, pa, pb);
			if (pa < pb) {
				if (o < pb - pa) {
					xs = pa + o;
					break;
				}
				o -= (uint32_t)(pb - pa);
			}
		}
		uint32_t left = s1 - s0;
		while (left > 0 && r < end_r && xs < w1) {
			const uint64_t fr0 = b.fo[r] - b.fo0;
			uint64_t pa, pb;
			bk_piece(b, r, xs, w1, pa, pb);
			const uint32_t n = (uint32_t)min((uint64_t)left, pb > pa ? pb - pa : (uint64_t)0);
			if (n > 0) {
				const uint32_t mate = r >= b.a.n ? 1u : 0u;
				const uint64_t i = r - (mate ? b.a.n : 0);
				const uint64_t start = b.a.off[mate][i] - b.a.off_base[mate];
				const PackedBases &P = b.pk[mate];
				const uint32_t *dust = b.a.dust[mate];
				const uint64_t qa = pa - fr0;           /* first frame, read coordinates */
				const uint64_t steps = (uint64_t)n + k - 1;
				uint64_t fh = 0, rh = 0;
				int64_t lb = -1; /* last base that is not ACGT, read coordinates */
				for (uint64_t j = qa; j < qa + steps; j += 16) {
					const uint32_t gn = (uint32_t)min((uint64_t)16, qa + steps - j);
					uint32_t cin, bin, cout, bout;
					codes16(P, (int64_t)(start + j), cin, bin);
					codes16(P, (int64_t)(start + j) - (int64_t)k, cout, bout);
					if (j < qa + k) { /* the first k steps: no base leaves */
						const uint64_t wu = qa + k - j;
						bout |= wu >= 16 ? 0xFFFFu : (1u << (uint32_t)wu) - 1u;
					}
#pragma unroll
					for (uint32_t u = 0; u < 16; ++u) {
						if (u < gn) {
							const uint32_t ci = ((bin >> u) & 1u) ? 4u : ((cin >> (2u * u)) & 3u);
							const uint32_t co = ((bout >> u) & 1u) ? 4u : ((cout >> (2u * u)) & 3u);
							const uint32_t e = (co << 3) | ci;
							fh = rol1(fh) ^ tab.tf[e];
							rh = ror1(rh) ^ tab.tr[e];
							const uint64_t jj = j + u;
							if (ci == 4u)
								lb = (int64_t)jj;
							if (jj + 1 >= qa + k) {
								const uint64_t q = jj + 1 - k;
								const uint32_t fid = (uint32_t)(fr0 + q - w0);
								const uint32_t wi = fid >> 5, bit = 1u << (fid & 31u);
								if (wi != cw) {
									if (vacc)
										atomicOr(&sm.sv[cw], vacc);
									if (aacc)
										atomicOr(&sm.sa[cw], aacc);
									vacc = aacc = 0;
									cw = wi;
								}
								if (lb < (int64_t)q) {
									vacc |= bit;
									if (!dust_low(dust, start + q)) {
										aacc |= bit;
										const uint64_t canon = fh < rh ? fh : rh;
										b.canon[w0 + fid] = canon;
										for (uint32_t l = 0; l < b.nlevels; ++l) {
											const uint64_t pos = reduce(
													l ? extra_hash(canon, k, l) : canon,
													b.f.m, b.f.minv);
											atomicAdd(&sm.hist[pos >> b.bshift], 1u);
										}
									}
								}
							}
						}
					}
				}
				left -= n;
			}
			/* the next read with frames in the phase */
			++r;
			xs = r < end_r ? max(xs, b.fo[r] - b.fo0) : w1;
		}
	}
	if (vacc)
		atomicOr(&sm.sv[cw], vacc);
	if (aacc)
		atomicOr(&sm.sa[cw], aacc);
	__syncthreads();

	/* 3 */
	const uint64_t wbase = (uint64_t)blk * kWinWords;
	const uint64_t words = (b.T + 31) / 32;
	for (uint32_t w = t; w < kWinWords; w += kNT)
		if (wbase + w < words) {
			b.vbits[wbase + w] |= sm.sv[w];
			b.hbits[wbase + w] |= sm.sa[w];
			b.abits[wbase + w] = sm.sa[w];
		}
	bk_scatter(b, sm, tmp);
}

/* The previous round's results of block blk applied to its hit bits: sh (the
 * block's words, loaded) loses the bits of the frames with a failed test and
 * goes back to b.hbits. */
__device__ void bk_apply_block(const BucketArgs &b, uint32_t *sh)
{
	const uint32_t blk = blockIdx.x, t = threadIdx.x;
	const uint64_t wbase = (uint64_t)blk * kWinWords;
	const uint64_t words = (b.T + 31) / 32;
	for (uint32_t w = t; w < kWinWords; w += kNT)
		sh[w] = wbase + w < words ? b.hbits[wbase + w] : 0u;
	__syncthreads();
	const uint64_t base = (uint64_t)blk * b.cap;
	const uint32_t n = b.btot[blk];
	for (uint32_t i = t; i < n; i += kNT)
		if (!__ldcs(b.res + base + i)) {
			const uint32_t fid = __ldcs(b.req_fid + base + i);
			atomicAnd(&sh[fid >> 5], ~(1u << (fid & 31u)));
		}
	__syncthreads();
	for (uint32_t w = t; w < kWinWords; w += kNT)
		if (wbase + w < words)
			b.hbits[wbase + w] = sh[w];
}

/* A later round, per window block: the previous round's results applied,
 * then the frames requesting in this phase that are still hits count their
 * requests of levels [level, level + nlevels) per bucket, then bk_scatter. */
__global__ void __launch_bounds__(kNT) bk_emit_kernel(BucketArgs b)
{
	extern __shared__ uint32_t bk_sm[];
	const SweepSmem sm(bk_sm, b.nbkt);
	__shared__ uint32_t tmp[33];
	const uint32_t blk = blockIdx.x, t = threadIdx.x;
	const uint64_t w0 = (uint64_t)blk * kBkWinFrames;
	const uint64_t wbase = (uint64_t)blk * kWinWords;
	const uint64_t words = (b.T + 31) / 32;
	bk_apply_block(b, sm.sv);
	for (uint32_t w = t; w < kWinWords; w += kNT)
		sm.sa[w] = wbase + w < words ? b.abits[wbase + w] & sm.sv[w] : 0u;
	for (uint32_t q = t; q < b.nbkt; q += kNT)
		sm.hist[q] = 0;
	__syncthreads();
	const unsigned sh = b.bshift, k = b.f.k;
	const uint32_t lane = t & 31u;
	for (uint32_t w = t >> 5; w < kWinWords; w += kNT / 32) {
		const uint32_t am = sm.sa[w];
		if (!((am >> lane) & 1u))
			continue;
		const uint64_t canon = b.canon[w0 + w * 32 + lane];
		for (uint32_t l = b.level; l < b.level + b.nlevels; ++l) {
			const uint64_t pos = reduce(l ? extra_hash(canon, k, l) : canon, b.f.m, b.f.minv);
			atomicAdd(&sm.hist[pos >> sh], 1u);
		}
	}
	__syncthreads();
	bk_scatter(b, sm, tmp);
}

__global__ void __launch_bounds__(kNT) bk_apply_kernel(BucketArgs b)
{
	__shared__ uint32_t sh[kWinWords];
	bk_apply_block(b, sh);
}

/* The round's (bucket, block) segments in bucket-major order, taken four at a
 * time from a work counter (so that every warp works at the front and the
 * buckets in flight stay few), one warp per segment and eight requests per
 * lane in flight; the bucket being tested is held in L2, the pool is read once
 * and the results written once (streaming). */
__global__ void __launch_bounds__(256) bk_resolve_kernel(BucketArgs b)
{
	const uint32_t lane = threadIdx.x & 31u;
	const uint64_t nseg = (uint64_t)b.nbkt * b.nblk;
	const uint32_t *words = b.f.words;
	const unsigned sh = b.bshift;
	unsigned long long issued = 0;
	for (;;) {
		unsigned long long g = 0;
		if (lane == 0)
			g = atomicAdd(b.next, 4ull);
		g = __shfl_sync(0xffffffffu, g, 0);
		if (g >= nseg)
			break;
		const uint32_t n4 = lane < 4 && g + lane < nseg ? b.cnt[g + lane] : 0u;
		const uint32_t l4 = lane < 4 && g + lane < nseg ? b.loc[g + lane] : 0u;
		for (uint32_t u = 0; u < 4 && g + u < nseg; ++u) {
			const uint64_t cur = g + u;
			const uint32_t n = __shfl_sync(0xffffffffu, n4, u);
			const uint32_t lc = __shfl_sync(0xffffffffu, l4, u);
			if (n == 0)
				continue;
			const uint32_t q = (uint32_t)(cur / b.nblk);
			const uint32_t blk = (uint32_t)(cur - (uint64_t)q * b.nblk);
			const uint64_t base = (uint64_t)blk * b.cap + lc;
			const uint64_t qbase = (uint64_t)q << sh;
			issued += n;
			for (uint32_t c = 0; c < n; c += 256) {
				uint32_t off[8], w[8];
#pragma unroll
				for (int j = 0; j < 8; ++j) {
					const uint32_t i = c + (uint32_t)j * 32 + lane;
					off[j] = i < n ? __ldcs(b.req_off + base + i) : 0u;
				}
#pragma unroll
				for (int j = 0; j < 8; ++j) {
					const uint32_t i = c + (uint32_t)j * 32 + lane;
					w[j] = i < n ? __ldg(words + ((qbase + off[j]) >> 5)) : 0u;
				}
#pragma unroll
				for (int j = 0; j < 8; ++j) {
					const uint32_t i = c + (uint32_t)j * 32 + lane;
					if (i < n)
						__stcs(b.res + base + i, (uint8_t)((w[j] >> (off[j] & 31u)) & 1u));
				}
			}
		}
	}
	if (b.issued && lane == 0 && issued)
		atomicAdd(b.issued, issued);
}

/* One thread per read of the sub-batch walks the exact state machine over
 * the frames resolved so far. */
template <int MODE>
__global__ void __launch_bounds__(256) bk_walk_kernel(BucketArgs b)
{
	const ClassifyArgs &a = b.a;
	const unsigned k = b.f.k;
	for (uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; t < b.nr;
			t += (uint64_t)gridDim.x * blockDim.x) {
		const uint64_t r = b.r0 + t;
		if (b.state[r])
			continue;
		const uint64_t F = b.fo[r + 1] - b.fo[r];
		if (F == 0) {
			b.state[r] = 1;
			continue;
		}
		const uint32_t mate = r >= a.n ? 1u : 0u;
		const uint64_t i = r - (mate ? a.n : 0);
		const uint64_t len = a.off[mate][i + 1] - a.off[mate][i];
		const uint64_t pb = bk_bound(F, b.ph_hi, b.ph_min);
		const uint64_t xr = b.fo[r] - b.fo0;
		SimpleState st;
		LengthState ls;
		SeqState qs;
		if (MODE == BBT_SCORE_HARMONIC)
			harmonic_init(qs, a.score, a.one_minus, F);
		else if (MODE == BBT_SCORE_BINOMIAL)
			binomial_simple_init(st, a.bthres[(uint64_t)b.fbit * a.bthres_rows + F], F);
		else if (MODE == BBT_SCORE_LENGTH)
			length_init(ls, a.min_len, len, (int)k);
		else
			simple_init(st, a.score, a.one_minus, F);
		int decided = EVAL_OPEN;
		for (uint64_t c = 0; c < pb && !decided; c += 32) {
			const int nf = (int)min((uint64_t)32, pb - c);
			const uint32_t V = bits_at(b.vbits, xr + c) & low_mask(nf);
			const uint32_t H = bits_at(b.hbits, xr + c) & V;
			decided = MODE == BBT_SCORE_LENGTH
					? length_chunk(ls, V, H, (int64_t)c, nf, nullptr)
					: MODE == BBT_SCORE_HARMONIC
					? seq_chunk(qs, V, H, (int64_t)c, nf, (int)k, a.streak_thr, nullptr)
					: simple_chunk<false>(st, V, H, (int32_t)c, nf, (int)k, (int)a.streak_thr,
							nullptr);
		}
		if (decided == EVAL_ACCEPT)
			a.hits[mate][i * a.words + (b.fbit >> 6)] |= 1ull << (b.fbit & 63u);
		if (decided || pb == F)
			b.state[r] = 1;
	}
}

/* out[j] = fo[min(j * stride, total)] for j < n (frame offsets sampled for the
 * host's sub-batch plan). */
__global__ void bk_samples_kernel(const uint64_t *fo, uint64_t total, uint64_t stride,
		uint64_t *out, uint64_t n)
{
	for (uint64_t j = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; j < n;
			j += (uint64_t)gridDim.x * blockDim.x) {
		const uint64_t r = j * stride;
		out[j] = fo[r < total ? r : total];
	}
}

__global__ void bk_frame_counts_kernel(ClassifyArgs a, unsigned k, uint64_t *fo_plus1)
{
	const uint64_t total = a.n * a.mates;
	for (uint64_t r = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; r < total;
			r += (uint64_t)gridDim.x * blockDim.x) {
		const uint32_t mate = r >= a.n ? 1u : 0u;
		const uint64_t i = r - (mate ? a.n : 0);
		const uint64_t len = a.off[mate][i + 1] - a.off[mate][i];
		fo_plus1[r] = len >= k ? len - k + 1 : 0;
	}
}

} // namespace

size_t bk_sweep_smem(uint32_t nbkt)
{
	return (2 * (size_t)kWinWords + 2 * (size_t)nbkt) * sizeof(uint32_t);
}

cudaError_t launch_bk_frame_counts(const ClassifyArgs &a, unsigned k, uint64_t *fo_plus1,
		int num_sms, cudaStream_t s)
{
	const uint64_t total = a.n * a.mates;
	if (total == 0)
		return cudaSuccess;
	const uint64_t need = (total + 255) / 256, cap = (uint64_t)num_sms * 8;
	bk_frame_counts_kernel<<<(unsigned)(need < cap ? need : cap), 256, 0, s>>>(a, k, fo_plus1);
	return cudaGetLastError();
}

cudaError_t launch_bk_samples(const uint64_t *fo, uint64_t total, uint64_t stride, uint64_t *out,
		uint64_t n, int num_sms, cudaStream_t s)
{
	const uint64_t need = (n + 255) / 256, cap = (uint64_t)num_sms * 4;
	bk_samples_kernel<<<(unsigned)(need < cap ? need : cap), 256, 0, s>>>(fo, total, stride, out,
			n);
	return cudaGetLastError();
}

cudaError_t launch_bk_pack(const uint8_t *ascii, uint64_t len, uint32_t *words, uint32_t *valid,
		int num_sms, cudaStream_t s)
{
	const uint64_t nvalid = len / 32 + 2;
	const uint64_t need = (nvalid + 255) / 256, cap = (uint64_t)num_sms * 16;
	bk_pack_kernel<<<(unsigned)(need < cap ? need : cap), 256, 0, s>>>(ascii, len, words, valid,
			nvalid);
	return cudaGetLastError();
}

cudaError_t launch_bk_hash(const BucketArgs &b, cudaStream_t s)
{
	if (b.nblk == 0)
		return cudaSuccess;
	if (b.nbkt > kMaxBuckets || b.level != 0 || b.cap < (uint64_t)kBkWinFrames * b.nlevels)
		return cudaErrorInvalidValue;
	bk_hash_kernel<<<b.nblk, kNT, bk_sweep_smem(b.nbkt), s>>>(b);
	return cudaGetLastError();
}

cudaError_t launch_bk_emit(const BucketArgs &b, cudaStream_t s)
{
	if (b.nblk == 0)
		return cudaSuccess;
	if (b.nbkt > kMaxBuckets || b.cap < (uint64_t)kBkWinFrames * b.nlevels)
		return cudaErrorInvalidValue;
	bk_emit_kernel<<<b.nblk, kNT, bk_sweep_smem(b.nbkt), s>>>(b);
	return cudaGetLastError();
}

cudaError_t launch_bk_resolve(const BucketArgs &b, int num_sms, cudaStream_t s)
{
	if (b.nblk == 0)
		return cudaSuccess;
	/* one resident wave */
	int per_sm = 0;
	cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, bk_resolve_kernel,
			256, 0);
	if (e != cudaSuccess)
		return e;
	e = cudaMemsetAsync(b.next, 0, sizeof(unsigned long long), s);
	if (e != cudaSuccess)
		return e;
	bk_resolve_kernel<<<num_sms * (per_sm > 0 ? per_sm : 1), 256, 0, s>>>(b);
	return cudaGetLastError();
}

cudaError_t launch_bk_apply(const BucketArgs &b, cudaStream_t s)
{
	if (b.nblk == 0)
		return cudaSuccess;
	bk_apply_kernel<<<b.nblk, kNT, 0, s>>>(b);
	return cudaGetLastError();
}

cudaError_t launch_bk_walk(const BucketArgs &b, int num_sms, cudaStream_t s)
{
	if (b.nr == 0)
		return cudaSuccess;
	const uint64_t need = (b.nr + 255) / 256, cap = (uint64_t)num_sms * 8;
	const unsigned grid = (unsigned)(need < cap ? need : cap);
	switch (b.a.scoring) {
	case BBT_SCORE_LENGTH:
		bk_walk_kernel<BBT_SCORE_LENGTH><<<grid, 256, 0, s>>>(b);
		break;
	case BBT_SCORE_HARMONIC:
		bk_walk_kernel<BBT_SCORE_HARMONIC><<<grid, 256, 0, s>>>(b);
		break;
	case BBT_SCORE_BINOMIAL:
		bk_walk_kernel<BBT_SCORE_BINOMIAL><<<grid, 256, 0, s>>>(b);
		break;
	default:
		bk_walk_kernel<BBT_SCORE_SIMPLE><<<grid, 256, 0, s>>>(b);
	}
	return cudaGetLastError();
}

} // namespace bbt
