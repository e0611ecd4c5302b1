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
 * contains() short-circuits), and the state machine of seqeval_chunk.cuh then
 * walks each read over the resolved hit bits.  The walk consumes only
 * contains() results, so making more tests than the sequential loop would (the
 * frames after a decision, frames in skip windows) changes no result.
 *
 * To keep those extra tests few, a read's frames are resolved in phases: the
 * first phase covers a prefix of every read (most reads that match are
 * accepted early), the next the rest of the reads still undecided.  Per phase
 * and round (one hash level, or two: a frame that passed the levels before
 * requests both, and stays a hit when both pass):
 *   count  -- per window block (kBkWinFrames frames of the sub-batch), apply
 *             the previous round's results to the block's hit bits (a frame
 *             with any failed test is no longer a hit), then hash the active
 *             frames (one thread per run of 128 consecutive frames, rolling
 *             ntHash) and count their requests per bucket;
 *   scan   -- the counts in bucket-major order give every (bucket, block) its
 *             place in the request pool;
 *   write  -- hash again and write each request (bit offset in its bucket,
 *             frame id in its block) to its place;
 *   resolve-- a resident grid tests the pool's requests in order, bucket by
 *             bucket, one result bit per request.
 * After the phase's last round the results are applied and one thread per
 * undecided read walks SeqEval over [0, phase end) of its frames.
 */
#include "bucketed.cuh"

#include "bbt.h"
#include "seqeval_chunk.cuh"
#include "window.cuh"

namespace bbt {

namespace {

constexpr uint32_t kRun = kBkWinFrames / kBkWinThreads;  /* frames per thread: 128 */
constexpr uint32_t kWinWords = kBkWinFrames / 32;
constexpr uint32_t kMaxBuckets = 2048;
static_assert(kRun % 32 == 0, "runs are whole hit-bit words");

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
 * any other base (whose seed is 0):
 *   tf[o, i] = rol(seed_fw(o), k) ^ seed_fw(i)
 *   tr[o, i] = ror(seed_rc(o), 1) ^ rol(seed_rc(i), k - 1)
 * so that a step is fh = rol(fh, 1) ^ tf, rh = ror(rh, 1) ^ tr; rc[c] is the
 * plain reverse-complement seed (the first k-mer of a piece). */
struct RollTables {
	uint64_t tf[64];
	uint64_t tr[64];
	uint64_t rc[8];
};

__device__ void bk_set_tables(RollTables &t, unsigned k)
{
	for (int e = threadIdx.x; e < 64; e += blockDim.x) {
		const uint8_t o = (uint8_t)(e >> 3), i = (uint8_t)(e & 7);
		t.tf[e] = rolk(seed_fw_code(o), k) ^ seed_fw_code(i);
		t.tr[e] = ror1(seed_rc_code(o)) ^ rolk(seed_rc_code(i), k - 1);
		if (e < 8)
			t.rc[e] = seed_rc_code((uint8_t)e);
	}
}

/* Sequential 3-bit base codes (0..3 ACGT, 4 other) of one read for one
 * thread, fetched 16 bases per load: the aligned 16-byte block of ASCII bases
 * holding the base (bytes turned into codes and validity bits four at a time),
 * or the 2-bit code word and its validity bits.  Calls ask for non-decreasing
 * j.  (An aligned 16-byte block never crosses a page, so reading all of the
 * block that holds a valid base stays inside mapped memory.) */
struct CodeStream {
	Bases src;
	uint64_t blk;
	uint32_t codes; /* 2 bits per base of the block */
	uint32_t bad;   /* 1 bit per base of the block: not ACGT */

	__device__ __forceinline__ void init(const Bases &s)
	{
		src = s;
		blk = ~0ull;
	}

	/* four ASCII bytes: their 2-bit codes (A0 C1 G2 T3 by bits 1-2 of the
	 * byte) in bits 0-7 and a validity nibble */
	__device__ __forceinline__ static void ascii4(uint32_t w, uint32_t &c8, uint32_t &ok4)
	{
		const uint32_t t = ((w >> 1) & 0x03030303u) ^ ((w >> 2) & 0x01010101u);
		c8 = (t & 3u) | ((t >> 6) & 0xCu) | ((t >> 12) & 0x30u) | ((t >> 18) & 0xC0u);
		const uint32_t u = w & 0xDFDFDFDFu;
		const uint32_t v = __vcmpeq4(u, 0x41414141u) | __vcmpeq4(u, 0x43434343u) |
				__vcmpeq4(u, 0x47474747u) | __vcmpeq4(u, 0x54545454u);
		ok4 = ((v >> 7) & 1u) | ((v >> 14) & 2u) | ((v >> 21) & 4u) | ((v >> 28) & 8u);
	}

	__device__ __forceinline__ uint32_t code(uint64_t j)
	{
		const uint64_t g = src.g0 + j;
		uint32_t o;
		if (src.ascii) {
			const uintptr_t p = reinterpret_cast<uintptr_t>(src.ascii + g);
			const uint64_t bk = p >> 4;
			if (bk != blk) {
				blk = bk;
				const uint4 q = __ldg(reinterpret_cast<const uint4 *>(bk << 4));
				uint32_t c0, c1, c2, c3, k0, k1, k2, k3;
				ascii4(q.x, c0, k0);
				ascii4(q.y, c1, k1);
				ascii4(q.z, c2, k2);
				ascii4(q.w, c3, k3);
				codes = c0 | (c1 << 8) | (c2 << 16) | (c3 << 24);
				bad = ~(k0 | (k1 << 4) | (k2 << 8) | (k3 << 12)) & 0xFFFFu;
			}
			o = (uint32_t)(p & 15u);
		} else {
			const uint64_t bk = g >> 4;
			if (bk != blk) {
				blk = bk;
				codes = __ldg(src.words + bk);
				bad = src.valid ? (~(__ldg(src.valid + (g >> 5)) >> (16u * (uint32_t)(bk & 1u))) &
				                   0xFFFFu)
				                : 0u;
			}
			o = (uint32_t)(g & 15u);
		}
		return ((bad >> o) & 1u) ? 4u : ((codes >> (2u * o)) & 3u);
	}
};

/*
 * One thread's run of frames [x0, x0 + kRun) of window block blk: for every
 * frame of an open read inside the current phase, FIRST computes its validity
 * (ACGT only, not DUST-masked) into vbits / hbits; otherwise a frame is active
 * when its hit bit (shb, the block's words in shared memory) is still set.
 * op(pos, fid) is called for each active frame with the bit its hash of this
 * round's level selects and the frame's id in the block.
 */
template <bool FIRST, class Op>
__device__ void bk_sweep_run(const BucketArgs &b, uint32_t blk, const uint32_t *shb,
		const RollTables &tab, Op op)
{
	const uint64_t w0 = (uint64_t)blk * kBkWinFrames;
	const uint64_t x0 = w0 + (uint64_t)threadIdx.x * kRun;
	if (x0 >= b.T)
		return;
	const uint64_t x1 = min(x0 + kRun, b.T);
	const unsigned k = b.f.k;
	/* FIRST: the run's validity / hit bits, one word at a time (word cw of
	 * the sub-batch), merged into the arrays when the run moves past it; the
	 * run's words belong to this thread */
	uint64_t cw = x0 >> 5;
	uint32_t vacc = 0, hacc = 0, touched = 0;
	auto flush = [&]() {
		if (touched) {
			b.vbits[cw] = (b.vbits[cw] & ~touched) | vacc;
			b.hbits[cw] = (b.hbits[cw] & ~touched) | hacc;
		}
		vacc = hacc = touched = 0;
	};
	uint64_t r = bk_find_read(b, x0);
	for (uint64_t x = x0; x < x1;) {
		while (b.fo[r + 1] - b.fo0 <= x)
			++r;
		const uint64_t fr0 = b.fo[r] - b.fo0, fr1 = b.fo[r + 1] - b.fo0;
		const uint64_t F = fr1 - fr0;
		const uint64_t q0 = x - fr0, q1 = min(x1, fr1) - fr0;
		x = fr0 + q1;
		if (b.state[r])
			continue;
		const uint64_t qa = max(q0, bk_bound(F, b.ph_lo, b.ph_min));
		const uint64_t qb = min(q1, bk_bound(F, b.ph_hi, b.ph_min));
		if (qa >= qb)
			continue;
		const uint32_t mate = r >= b.a.n ? 1u : 0u;
		const uint64_t i = r - (mate ? b.a.n : 0);
		const uint64_t start = b.a.off[mate][i] - b.a.off_base[mate];
		const Bases src = read_bases(b.a, mate, start);
		CodeStream sin, sout; /* the base entering and the base leaving the k-mer */
		sin.init(src);
		sout.init(src);
		/* ntHash of frame qa over its k bases, then rolled one base at a time */
		uint64_t fh = 0, rh = 0;
		int64_t lb = -1; /* last base that is not ACGT, read coordinates */
		for (unsigned j = 0; j < k; ++j) {
			const uint32_t c = sin.code(qa + j);
			fh = rol1(fh) ^ tab.tf[(4u << 3) | c];
			rh ^= rolk(tab.rc[c], j);
			if (c == 4)
				lb = (int64_t)(qa + j);
		}
		for (uint64_t q = qa; q < qb; ++q) {
			if (q > qa) {
				const uint32_t out = sout.code(q - 1);
				const uint32_t in = sin.code(q + k - 1);
				const uint32_t e = (out << 3) | in;
				fh = rol1(fh) ^ tab.tf[e];
				rh = ror1(rh) ^ tab.tr[e];
				if (in == 4)
					lb = (int64_t)(q + k - 1);
			}
			const uint64_t xf = fr0 + q;
			const uint32_t fid = (uint32_t)(xf - w0);
			bool active;
			if (FIRST) {
				const bool valid = lb < (int64_t)q;
				active = valid && !dust_low(b.a.dust[mate], start + q);
				if ((xf >> 5) != cw) {
					flush();
					cw = xf >> 5;
				}
				const uint32_t bit = 1u << (uint32_t)(xf & 31u);
				touched |= bit;
				if (valid)
					vacc |= bit;
				if (active)
					hacc |= bit;
			} else {
				active = (shb[fid >> 5] >> (fid & 31u)) & 1u;
			}
			if (active) {
				const uint64_t canon = fh < rh ? fh : rh;
				for (uint32_t l = b.level; l < b.level + b.nlevels; ++l) {
					const uint64_t v = l ? extra_hash(canon, k, l) : canon;
					op(reduce(v, b.f.m, b.f.minv), fid);
				}
			}
		}
	}
	if (FIRST)
		flush();
}

/* Load the hit bits of window block blk into shb. */
__device__ __forceinline__ void bk_load_window(const BucketArgs &b, uint32_t blk, uint32_t *shb)
{
	const uint64_t wbase = (uint64_t)blk * kWinWords;
	const uint64_t words = (b.T + 31) / 32;
	for (uint32_t w = threadIdx.x; w < kWinWords; w += blockDim.x)
		shb[w] = wbase + w < words ? b.hbits[wbase + w] : 0u;
}

/* Clear the hit bits of the block's frames whose previous-round test missed,
 * and store the block's words back. */
__device__ void bk_apply_window(const BucketArgs &b, uint32_t blk, uint32_t *shb)
{
	for (uint32_t q = 0; q < b.nbkt; ++q) {
		const uint64_t at = (uint64_t)q * b.nblk + blk;
		const uint64_t s0 = b.pseg[at];
		const uint32_t n = (uint32_t)b.pcnt[at];
		for (uint32_t j = threadIdx.x; j < n; j += blockDim.x) {
			const uint64_t i = s0 + j;
			if (!((b.res[i >> 5] >> (i & 31u)) & 1u)) {
				const uint32_t fid = b.req_fid[i];
				atomicAnd(&shb[fid >> 5], ~(1u << (fid & 31u)));
			}
		}
	}
	__syncthreads();
	const uint64_t wbase = (uint64_t)blk * kWinWords;
	const uint64_t words = (b.T + 31) / 32;
	for (uint32_t w = threadIdx.x; w < kWinWords; w += blockDim.x)
		if (wbase + w < words)
			b.hbits[wbase + w] = shb[w];
	__syncthreads();
}

template <bool FIRST>
__global__ void __launch_bounds__(kBkWinThreads) bk_count_kernel(BucketArgs b)
{
	extern __shared__ uint32_t bk_sm[];
	uint32_t *shb = bk_sm;
	uint32_t *hist = bk_sm + kWinWords;
	const uint32_t blk = blockIdx.x;
	__shared__ RollTables tab;
	bk_set_tables(tab, b.f.k);
	for (uint32_t q = threadIdx.x; q < b.nbkt; q += blockDim.x)
		hist[q] = 0;
	if (!FIRST) {
		bk_load_window(b, blk, shb);
		__syncthreads();
		bk_apply_window(b, blk, shb);
	}
	__syncthreads();
	const unsigned sh = b.bshift;
	bk_sweep_run<FIRST>(b, blk, shb, tab, [&](uint64_t pos, uint32_t) {
		atomicAdd(&hist[pos >> sh], 1u);
	});
	__syncthreads();
	for (uint32_t q = threadIdx.x; q < b.nbkt; q += blockDim.x)
		b.cnt[(uint64_t)q * b.nblk + blk] = hist[q];
}

__global__ void __launch_bounds__(kBkWinThreads) bk_write_kernel(BucketArgs b)
{
	extern __shared__ uint32_t bk_sm[];
	uint32_t *shb = bk_sm;
	uint32_t *cur = bk_sm + kWinWords;
	const uint32_t blk = blockIdx.x;
	__shared__ RollTables tab;
	bk_set_tables(tab, b.f.k);
	for (uint32_t q = threadIdx.x; q < b.nbkt; q += blockDim.x)
		cur[q] = 0;
	bk_load_window(b, blk, shb);
	__syncthreads();
	const unsigned sh = b.bshift;
	const uint64_t mask = (1ull << sh) - 1ull;
	bk_sweep_run<false>(b, blk, shb, tab, [&](uint64_t pos, uint32_t fid) {
		const uint32_t q = (uint32_t)(pos >> sh);
		const uint64_t i = b.seg[(uint64_t)q * b.nblk + blk] + atomicAdd(&cur[q], 1u);
		b.req_off[i] = (uint32_t)(pos & mask);
		b.req_fid[i] = (uint16_t)fid;
	});
}

__global__ void __launch_bounds__(kBkWinThreads) bk_apply_kernel(BucketArgs b)
{
	__shared__ uint32_t shb[kWinWords];
	bk_load_window(b, blockIdx.x, shb);
	__syncthreads();
	bk_apply_window(b, blockIdx.x, shb);
}

/* The pool's requests in index order (bucket-major), eight per lane in flight;
 * the bucket being tested is held in L2, the pool is read once (evict-first). */
__global__ void __launch_bounds__(256) bk_resolve_kernel(BucketArgs b)
{
	__shared__ unsigned long long bs[kMaxBuckets + 1];
	for (uint32_t q = threadIdx.x; q <= b.nbkt; q += blockDim.x)
		bs[q] = b.seg[(uint64_t)q * b.nblk];
	__syncthreads();
	const uint64_t R = bs[b.nbkt];
	if (b.issued && blockIdx.x == 0 && threadIdx.x == 0)
		atomicAdd(b.issued, (unsigned long long)R);
	const uint64_t pol = evict_first_policy();
	const int lane = threadIdx.x & 31;
	const uint64_t warps = (uint64_t)gridDim.x * (blockDim.x >> 5);
	const uint32_t *words = b.f.words;
	const unsigned sh = b.bshift;
	for (uint64_t c = (uint64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); c * 256 < R;
			c += warps) {
		uint64_t pos[8];
		uint32_t w[8];
#pragma unroll
		for (int j = 0; j < 8; ++j) {
			const uint64_t i = c * 256 + (uint64_t)j * 32 + lane;
			pos[j] = ~0ull;
			if (i < R) {
				uint32_t lo = 0, hi = b.nbkt; /* bs[lo] <= i < bs[hi] */
				while (hi - lo > 1) {
					const uint32_t mid = (lo + hi) >> 1;
					if (bs[mid] <= i)
						lo = mid;
					else
						hi = mid;
				}
				pos[j] = ((uint64_t)lo << sh) | ld_stream_u32(b.req_off + i, pol);
			}
		}
#pragma unroll
		for (int j = 0; j < 8; ++j)
			w[j] = pos[j] != ~0ull ? __ldg(words + (pos[j] >> 5)) : 0u;
#pragma unroll
		for (int j = 0; j < 8; ++j) {
			const uint32_t hit = __ballot_sync(0xffffffffu,
					pos[j] != ~0ull && ((w[j] >> (pos[j] & 31u)) & 1u));
			const uint64_t i0 = c * 256 + (uint64_t)j * 32;
			if (lane == 0 && i0 < R)
				b.res[i0 >> 5] = hit;
		}
	}
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
	return (kWinWords + (size_t)nbkt) * sizeof(uint32_t);
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

cudaError_t launch_bk_count(const BucketArgs &b, cudaStream_t s)
{
	if (b.nblk == 0)
		return cudaSuccess;
	if (b.nbkt > kMaxBuckets)
		return cudaErrorInvalidValue;
	const size_t smem = bk_sweep_smem(b.nbkt);
	if (b.pcnt) {
		cudaError_t e = cudaFuncSetAttribute(bk_count_kernel<false>,
				cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
		if (e != cudaSuccess)
			return e;
		bk_count_kernel<false><<<b.nblk, kBkWinThreads, smem, s>>>(b);
	} else {
		cudaError_t e = cudaFuncSetAttribute(bk_count_kernel<true>,
				cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
		if (e != cudaSuccess)
			return e;
		bk_count_kernel<true><<<b.nblk, kBkWinThreads, smem, s>>>(b);
	}
	return cudaGetLastError();
}

cudaError_t launch_bk_write(const BucketArgs &b, cudaStream_t s)
{
	if (b.nblk == 0)
		return cudaSuccess;
	const size_t smem = bk_sweep_smem(b.nbkt);
	cudaError_t e = cudaFuncSetAttribute(bk_write_kernel,
			cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
	if (e != cudaSuccess)
		return e;
	bk_write_kernel<<<b.nblk, kBkWinThreads, smem, s>>>(b);
	return cudaGetLastError();
}

cudaError_t launch_bk_resolve(const BucketArgs &b, int num_sms, cudaStream_t s)
{
	if (b.nblk == 0)
		return cudaSuccess;
	if (b.nbkt > kMaxBuckets)
		return cudaErrorInvalidValue;
	bk_resolve_kernel<<<num_sms * 8, 256, 0, s>>>(b);
	return cudaGetLastError();
}

cudaError_t launch_bk_apply(const BucketArgs &b, cudaStream_t s)
{
	if (b.nblk == 0)
		return cudaSuccess;
	bk_apply_kernel<<<b.nblk, kBkWinThreads, 0, s>>>(b);
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
