/*
 * seqeval_chunk.cuh -- SeqEval::evalSimple (Common/SeqEval.h:37-114) and
 * SeqEval::evalMinMatchLen (Common/SeqEval.h:295-332) restated over 32-frame
 * chunks of hit bits.
 *
 * A warp probes the filter for 32 consecutive frames at once (one frame per
 * lane) and ballots the results.  The functions here then advance the
 * reference's sequential state machine over those 32 frames using mask
 * arithmetic (popcounts over prefixes), so the decision, and the frame at
 * which it is taken, are exactly those of the sequential loop.  All inputs are
 * warp-uniform, so every lane runs the same scalar code; the functions are
 * also compiled for the host, where tests drive them against the CPU oracle.
 *
 * Frame model.  Frame p is the k-mer starting at base p of the read,
 * p in [0, len-k].  It is "valid" when the k-mer holds only ACGT: those are the
 * positions ntHashIterator visits.  The reference's gap handling
 * (SeqEval.h:71-77) adds, at the next valid frame, one to antiScore for each
 * skipped invalid frame; that is counted here one frame at a time.  The only
 * observable difference is where a rejection is taken, and a rejection is
 * final either way, so decisions are unchanged.  Leading invalid frames are not
 * counted (the first frame has no gap check, SeqEval.h:52-67).  After a miss
 * that ends a streak of at least streakThreshold hits, the reference walks the
 * visited positions below pos+k adding one per position without probing
 * (SeqEval.h:99-110); invalid frames inside that window before its last valid
 * frame are therefore not counted, and those after it are counted by the next
 * gap check.
 */
#ifndef BBT_SEQEVAL_CHUNK_CUH
#define BBT_SEQEVAL_CHUNK_CUH

#include <math.h>
#include <stdint.h>

#if defined(__CUDACC__)
#define BBT_HD __host__ __device__ __forceinline__
#else
#define BBT_HD inline
#endif

namespace bbt {

BBT_HD int popc32(uint32_t x)
{
#if defined(__CUDA_ARCH__)
	return __popc(x);
#else
	return __builtin_popcount(x);
#endif
}

/* index of the lowest set bit (x != 0) */
BBT_HD int lowbit32(uint32_t x)
{
#if defined(__CUDA_ARCH__)
	return __ffs(x) - 1;
#else
	return __builtin_ctz(x);
#endif
}

/* index of the highest set bit (x != 0) */
BBT_HD int highbit32(uint32_t x)
{
#if defined(__CUDA_ARCH__)
	return 31 - __clz(x);
#else
	return 31 - __builtin_clz(x);
#endif
}

/* number of consecutive set bits from bit 31 down */
BBT_HD int leading_ones32(uint32_t x)
{
#if defined(__CUDA_ARCH__)
	return __clz(~x);
#else
	return ~x ? __builtin_clz(~x) : 32;
#endif
}

/* bits [0, n) set, n in [0, 32] */
BBT_HD uint32_t low_mask(int n)
{
	return n >= 32 ? 0xffffffffu : (n <= 0 ? 0u : ((1u << n) - 1u));
}

/* bits [lo, hi) set */
BBT_HD uint32_t range_mask(int lo, int hi)
{
	return low_mask(hi) & ~low_mask(lo);
}

/* position of the n-th (1-based) set bit of x, which has at least n set bits */
BBT_HD int nth_bit(uint32_t x, int n)
{
	for (int i = 1; i < n; ++i)
		x &= x - 1;
	return lowbit32(x);
}

enum { EVAL_OPEN = 0, EVAL_ACCEPT = 1, EVAL_REJECT = 2 };

/*
 * Where a chunk's running totals cross their thresholds.  Frame j of the chunk
 * (restricted to `pre`) accepts when it is a hit and
 *   score2 + popc(H & frames<=j) + popc(P2 & frames<=j) >= thres2,
 * and rejects when it adds to antiScore and anti + popc(A & frames<=j) >=
 * anti_thres.  On the device with WARP every lane evaluates its own frame and
 * two ballots collect the answers (all 32 lanes of the warp must be here);
 * otherwise (the host, or one thread walking a read on its own) the frames are
 * looped over with running sums.
 */
template <bool WARP = true>
BBT_HD void crossing_masks(uint32_t H, uint32_t P2, uint32_t A, uint32_t pre, int32_t score2,
		int32_t anti, int32_t thres2, int32_t anti_thres, uint32_t &acc, uint32_t &rej)
{
	H &= pre;
	P2 &= pre;
	A &= pre;
#if defined(__CUDA_ARCH__)
	if (WARP) {
		unsigned lane;
		asm("mov.u32 %0, %%laneid;" : "=r"(lane));
		const uint32_t le = 0xffffffffu >> (31 - lane);
		const int32_t sc = score2 + __popc(H & le) + __popc(P2 & le);
		const int32_t an = anti + __popc(A & le);
		acc = __ballot_sync(0xffffffffu, ((H >> lane) & 1u) && sc >= thres2);
		rej = __ballot_sync(0xffffffffu, ((A >> lane) & 1u) && an >= anti_thres);
		return;
	}
#endif
	/* one thread: running sums over the 32 frames */
	acc = rej = 0;
	int32_t sc = score2, an = anti;
	for (unsigned j = 0; j < 32; ++j) {
		const uint32_t h = (H >> j) & 1u, a = (A >> j) & 1u;
		sc += (int32_t)(h + ((P2 >> j) & 1u));
		an += (int32_t)a;
		if (h && sc >= thres2)
			acc |= 1u << j;
		if (a && an >= anti_thres)
			rej |= 1u << j;
	}
}

/*
 * State of one (read, filter) evaluation under SIMPLE scoring.
 * score2 is twice the reference's double score (a multiple of 0.5), so
 * "thres <= score" is "score2 >= thres2" with thres2 = ceil(2*thres); anti
 * is antiScore and "antiThres <= antiScore" is "anti >= anti_thres".
 */
struct SimpleState {
	int32_t score2;
	int32_t anti;
	int32_t thres2;
	int32_t anti_thres;
	int32_t streak;       /* hits in the current streak (saturates at 64) */
	int32_t started;      /* a valid frame has been visited */
	int32_t skip_until;   /* frames below this belong to a skip window */
	int32_t in_window;    /* a skip window is open (frames < skip_until) */
	int32_t pending;      /* invalid window frames after its last valid one */
	int32_t decided;      /* EVAL_* */
	int32_t flat;         /* BINOMIAL: every hit adds 1 (2 to score2) */
};

/* Reads are limited to this many frames so that every counter of the state
 * machine (at most twice the frame count) fits in 32 bits. */
constexpr uint64_t kMaxFrames = (1ull << 30) - 1;

/*
 * Thresholds exactly as SeqEval.h:41-45 computes them:
 *   thres     = threshold * (len - k + 1)
 *   antiThres = floor((1 - threshold) * (len - k + 1))
 * with one IEEE double multiply each (one_minus = 1.0 - threshold is
 * computed once by the caller, as the reference's argument is).
 */
BBT_HD void simple_init(SimpleState &s, double threshold, double one_minus,
		uint64_t frames)
{
	double fr = (double)frames;
	double thres = threshold * fr;
	double anti = one_minus * fr;
#if defined(__CUDA_ARCH__)
	thres = __dmul_rn(threshold, fr);
	anti = __dmul_rn(one_minus, fr);
#endif
	double t2 = thres * 2.0; /* exact */
	double c = t2 <= 0.0 ? 0.0 : (double)(int64_t)t2;
	if (c < t2)
		c += 1.0;
	double a = anti;
	double fa = (double)(int64_t)a;
	if (fa > a)
		fa -= 1.0; /* floor for negative values */
	s.score2 = 0;
	s.anti = 0;
	s.thres2 = (int32_t)c;       /* at most 2 * kMaxFrames */
	s.anti_thres = fa < -1.0 ? -1 : (int32_t)fa;
	s.streak = 0;
	s.started = 0;
	s.skip_until = 0;
	s.in_window = 0;
	s.pending = 0;
	s.decided = EVAL_OPEN;
	s.flat = 0;
}

/*
 * SeqEval::evalBinomial (Common/SeqEval.h:218-290) is evalSimple's walk with
 * an integer score: every hit adds 1, "thres <= score" with thres =
 * calcMinCount(frameLen, fpr, minFPR) (computed on the host), and
 * "antiThres <= antiScore" with antiThres = frameLen - thres (unsigned; thres
 * never exceeds frameLen).  In score2's half units: every hit adds 2.
 */
BBT_HD void binomial_simple_init(SimpleState &s, uint32_t thres, uint64_t frames)
{
	s.score2 = 0;
	s.anti = 0;
	s.thres2 = (int32_t)(2u * thres);
	s.anti_thres = (int32_t)(uint32_t)((uint32_t)frames - thres);
	s.streak = 0;
	s.started = 0;
	s.skip_until = 0;
	s.in_window = 0;
	s.pending = 0;
	s.decided = EVAL_OPEN;
	s.flat = 1;
}

/*
 * How many frames the next step should probe (8..cap; cap is 32, or 64 when
 * every lane probes two frames per step).  At the start of a read and while
 * it is on a run of hits, the step is the number of valid frames that could
 * still accept it if all of them hit (a hit that starts a streak adds 1 to
 * score2, any other hit 2), so a read that accepts wastes no probes on frames
 * after its decision; otherwise (a read that is missing, which rarely
 * accepts) the full cap, which keeps the number of dependent steps, and so
 * the latency of a read, as low as before.  At least 8 frames keep several
 * probes in flight per warp.  The decision itself does not depend on the step
 * sizes.
 */
#ifndef BBT_TIGHT_MIN_STEP
#define BBT_TIGHT_MIN_STEP 8
#endif
#ifndef BBT_TIGHT_REJECT
#define BBT_TIGHT_REJECT 0
#endif
BBT_HD int simple_step_frames(const SimpleState &s, int cap = 32)
{
	const int32_t gap = s.thres2 - s.score2;
	if (gap <= 0)
		return cap;
	if (s.started && s.streak == 0) {
		if (!BBT_TIGHT_REJECT)
			return cap;
		/* a missing read: no reject before anti_thres - anti more misses */
		const int32_t agap = s.anti_thres - s.anti;
		return agap < BBT_TIGHT_MIN_STEP ? BBT_TIGHT_MIN_STEP : (agap > cap ? cap : (int)agap);
	}
	const int32_t need = (s.streak > 0 || s.flat) ? (gap + 1) / 2 : 1 + gap / 2;
	return need < BBT_TIGHT_MIN_STEP ? BBT_TIGHT_MIN_STEP : (need > cap ? cap : (int)need);
}

/*
 * Advance over one chunk of 32 frames starting at frame `base`.
 *   V:  valid frames (bit j = frame base+j), already limited to the read
 *   H:  hits among V (only bits the caller probed matter; see below)
 *   nf: frames of the read that exist in this chunk (bits >= nf are past the
 *       end of the read)
 * Frames below s.skip_until are inside a skip window: their H bits are never
 * read, so the caller need not probe them.  Returns s.decided.
 * alg (optional) receives the frames of this chunk that the sequential
 * algorithm probes (the ordinary frames up to the decision or the frame that
 * opens a skip window), for counting algorithmic probes.
 */
template <bool WARP = true>
BBT_HD int simple_chunk(SimpleState &s, uint32_t V, uint32_t H, int32_t base,
		int nf, int k, int streak_thr, uint32_t *alg = nullptr)
{
	if (s.decided)
		return s.decided;
	const uint32_t inread = low_mask(nf);
	V &= inread;
	H &= V;
	/* Fast path: no skip window open.  Frames before the first skip trigger
	 * (a miss after at least streak_thr hits) are settled here, including an
	 * accept or reject among them; a chunk that reaches a trigger undecided
	 * continues in the general loop below, from its start.  (The first
	 * visited frame can never trigger: its streak is 0.) */
	if (!s.in_window && streak_thr >= 1 && streak_thr <= 31) {
		const int st = s.streak;
		/* bit 31-i of lowc is "frame base-1-i was a hit", i < streak */
		const uint32_t lowc = st <= 0 ? 0u : (st >= 32 ? 0xffffffffu : (0xffffffffu << (32 - st)));
		uint32_t run = 0xffffffffu; /* frames preceded by streak_thr hits */
		for (int q = 1; q <= streak_thr; ++q)
			run &= (H << q) | (lowc >> (32 - q));
		const uint32_t M = V & ~H;
		const uint32_t trig = M & run;
		const uint32_t pre = trig ? low_mask(lowbit32(trig)) : inread;
		const uint32_t prevhit = s.flat ? H : (H & ((H << 1) | (st > 0 ? 1u : 0u)));
		/* invalid frames count, except those before the first valid one */
		const uint32_t C = s.started ? (~V & inread)
		                             : (V ? (~V & inread & ~low_mask(lowbit32(V))) : 0u);
		const uint32_t A = M | C;
		const int32_t dS = popc32(H & pre) + popc32(prevhit & pre);
		const int32_t dA = popc32(A & pre);
		if (s.score2 + dS >= s.thres2 || s.anti + dA >= s.anti_thres) {
			uint32_t acc, rej;
			crossing_masks<WARP>(H, prevhit, A, pre, s.score2, s.anti, s.thres2, s.anti_thres, acc,
					rej);
			const int ap = acc ? lowbit32(acc) : 32;
			const int rp = rej ? lowbit32(rej) : 32;
			if (ap < rp) {
				if (alg)
					*alg |= V & low_mask(ap + 1);
				s.decided = EVAL_ACCEPT;
				return s.decided;
			}
			if (rp < 32) {
				if (alg)
					*alg |= V & low_mask(rp + 1);
				s.decided = EVAL_REJECT;
				return s.decided;
			}
		}
		if (!trig) {
			s.score2 += dS;
			s.anti += dA;
			s.started |= V != 0;
			if (alg)
				*alg |= V;
			const uint32_t nonhit = ~H & inread;
			if (nonhit) {
				s.streak = popc32(H & ~low_mask(highbit32(nonhit) + 1));
			} else {
				const int ns = st + nf;
				s.streak = ns > 64 ? 64 : ns;
			}
			return EVAL_OPEN;
		}
	}
	int j = 0;
	while (j < nf) {
		/* ---- skip-window frames ---- */
		if (s.in_window) {
			int32_t we = s.skip_until - base;
			int e = we >= nf ? nf : (int)we;
			if (e > j) {
				uint32_t r = range_mask(j, e);
				uint32_t vw = V & r;
				s.anti += popc32(vw);
				if (vw) {
					int last = highbit32(vw);
					s.pending = popc32(~V & range_mask(last + 1, e));
				} else {
					s.pending += popc32(~V & r);
				}
				if (s.anti >= s.anti_thres) {
					s.decided = EVAL_REJECT;
					return s.decided;
				}
				j = e;
			}
			if (s.skip_until - base <= nf) {
				/* window closed inside the read: its trailing invalid
				 * frames count as the next gap does */
				s.anti += s.pending;
				s.pending = 0;
				s.in_window = 0;
				s.streak = 0;
				if (s.anti >= s.anti_thres) {
					s.decided = EVAL_REJECT;
					return s.decided;
				}
			}
			continue;
		}
		/* ---- ordinary frames [j, nf) ---- */
		const uint32_t rng = range_mask(j, nf);
		const uint32_t Hr = H & rng;
		const uint32_t Mr = V & ~H & rng;
		uint32_t Cr = ~V & rng; /* invalid frames */
		if (!s.started) {
			uint32_t vr = V & rng;
			/* leading invalid frames are not counted */
			Cr = vr ? (Cr & ~low_mask(lowbit32(vr))) : 0u;
		}
		/* ext: bit 32+i is "frame base+i was a hit"; bits below 32 hold the
		 * carried streak ending at frame base+j-1 */
		uint64_t carry = 0;
		{
			int st = s.streak;
			if (st > 0) {
				/* streak frames end at frame j-1 */
				uint64_t ones = st >= 64 ? ~0ull : ((1ull << st) - 1ull);
				carry = ones << (32 + j - (st > 32 + j ? 32 + j : st));
				if (st > 32 + j)
					carry = (1ull << (32 + j)) - 1ull;
			}
		}
		const uint64_t ext = ((uint64_t)Hr << 32) | carry;
		/* hits whose previous frame is a hit of the same streak: these add
		 * 1.0 to the score, the others 0.5 */
		const uint32_t prevhit = s.flat ? Hr : ((uint32_t)((ext << 1) >> 32) & Hr);
		/* skip triggers: a miss after at least streak_thr consecutive hits */
		uint32_t trig;
		if (streak_thr <= 0) {
			trig = Mr;
		} else if (streak_thr <= 32) {
			uint64_t t = ~0ull;
			for (int q = 1; q <= streak_thr; ++q)
				t &= ext << q;
			trig = Mr & (uint32_t)(t >> 32);
		} else {
			trig = 0; /* resolved frame by frame below */
			if (s.streak + popc32(Hr) >= streak_thr) {
				int run = s.streak;
				for (int q = j; q < nf; ++q) {
					uint32_t b = 1u << q;
					if (Hr & b) {
						++run;
					} else if (Mr & b) {
						if (run >= streak_thr) {
							trig = b;
							break;
						}
						run = 0;
					} else {
						run = 0;
					}
				}
			}
		}
		/* the first visited frame never opens a window (SeqEval.h:52-67
		 * has no skip branch), which matters when streak_thr is 0 */
		if (!s.started && (V & rng))
			trig &= ~(1u << lowbit32(V & rng));
		const int t = trig ? lowbit32(trig) : nf;
		const uint32_t pre = range_mask(j, t);
		const uint32_t hp = Hr & pre;
		const uint32_t hp2 = prevhit & pre;
		const uint32_t ap = (Mr | Cr) & pre;
		const int32_t dS = popc32(hp) + popc32(hp2);
		const int32_t dA = popc32(ap);
		int acc_pos = 32, rej_pos = 32;
		if (s.score2 + dS >= s.thres2) {
			int32_t sc = s.score2;
			uint32_t x = hp;
			while (x) {
				int q = lowbit32(x);
				x &= x - 1;
				sc += ((hp2 >> q) & 1u) ? 2 : 1;
				if (sc >= s.thres2) {
					acc_pos = q;
					break;
				}
			}
		}
		if (s.anti + dA >= s.anti_thres) {
			int32_t need = s.anti_thres - s.anti;
			rej_pos = need <= 0 ? (ap ? lowbit32(ap) : 32)
			                    : nth_bit(ap, (int)need);
		}
		if (acc_pos < rej_pos) {
			if (alg)
				*alg |= V & range_mask(j, acc_pos + 1);
			s.decided = EVAL_ACCEPT;
			return s.decided;
		}
		if (rej_pos < 32) {
			if (alg)
				*alg |= V & range_mask(j, rej_pos + 1);
			s.decided = EVAL_REJECT;
			return s.decided;
		}
		if (alg)
			*alg |= V & range_mask(j, t < nf ? t + 1 : nf);
		s.score2 += dS;
		s.anti += dA;
		if (V & pre)
			s.started = 1;
		/* streak at frame t (or at the end of the chunk) */
		{
			uint32_t nonhit = ~hp & pre;
			if (nonhit) {
				int lastbreak = highbit32(nonhit);
				s.streak = popc32(hp & ~low_mask(lastbreak + 1));
			} else {
				int add = popc32(hp);
				s.streak = s.streak + add > 64 ? 64 : s.streak + add;
			}
		}
		if (t >= nf)
			break;
		/* open the skip window at the trigger frame: the trigger frame itself
		 * is its first visited position */
		s.started = 1;
		s.in_window = 1;
		s.pending = 0;
		s.skip_until = base + t + k;
		j = t;
	}
	return s.decided;
}

/*
 * State of one (read, filter) evaluation under LENGTH scoring
 * (evalMinMatchLen): the length of the current run of matching bases.
 */
struct LengthState {
	int64_t match;
	int64_t prev;     /* last visited frame, -1 before the first */
	int64_t min_len;
	int64_t len;      /* read length in bases */
	int32_t k;
	int32_t decided;
};

BBT_HD void length_init(LengthState &s, unsigned min_len, uint64_t len, int k)
{
	s.match = 0;
	s.prev = 0; /* the reference starts prevPos at 0 */
	s.min_len = min_len;
	s.len = (int64_t)len;
	s.k = k;
	s.decided = EVAL_OPEN;
}

/* Advance over one chunk; every valid frame must have been probed.
 *
 * Without alg (no probe accounting) the chunk is settled by runs instead of
 * frame by frame.  The match after a valid frame is k + (its run of
 * consecutive hit frames - 1), or 0 after a miss; a run that touches bit 0
 * continues the previous chunk's match when the last visited frame was the
 * one just before.  The read is accepted iff some frame's match reaches
 * min_len.  The reference's reject test (len - pos + match < min_len before
 * a frame) only fires when no later frame can reach min_len, so the decision
 * does not depend on where it fires: here a chunk rejects when the frames
 * left cannot reach min_len even as one run continuing this chunk's last
 * one. */
BBT_HD int length_chunk(LengthState &s, uint32_t V, uint32_t H, int64_t base,
		int nf, uint32_t *alg = nullptr)
{
	if (s.decided)
		return s.decided;
	V &= low_mask(nf);
	if (!alg) {
		H &= V;
		const bool carry = s.match > 0 && s.prev == base - 1;
		uint32_t x = H;
		while (x) {
			const int a = lowbit32(x);
			const uint32_t rest = ~(H >> a); /* zero bits from a upwards */
			const int run = rest ? lowbit32(rest) : 32 - a;
			const int64_t m0 = (a == 0 && carry) ? s.match + 1 : (int64_t)s.k;
			if (m0 + run - 1 >= s.min_len)
				return s.decided = EVAL_ACCEPT;
			x &= ~range_mask(a, a + run);
		}
		if (V) {
			const int last = highbit32(V);
			if ((H >> last) & 1u) {
				const int run = leading_ones32(H << (31 - last));
				const int a = last - run + 1;
				s.match = (a == 0 && carry) ? s.match + run : (int64_t)s.k + run - 1;
			} else {
				s.match = 0;
			}
			s.prev = base + last;
		}
		const int64_t rem = s.len - s.k + 1 - (base + nf);
		const bool cont = nf > 0 && ((H >> (nf - 1)) & 1u);
		const int64_t best = cont ? s.match + rem : (rem > 0 ? s.k + rem - 1 : 0);
		if (best < s.min_len)
			return s.decided = EVAL_REJECT;
		return EVAL_OPEN;
	}
	uint32_t x = V;
	while (x) {
		int q = lowbit32(x);
		x &= x - 1;
		int64_t pos = base + q;
		if (s.len - pos + s.match < s.min_len) {
			s.decided = EVAL_REJECT;
			return s.decided;
		}
		if (pos != s.prev + 1)
			s.match = 0;
		if (alg)
			*alg |= 1u << q;
		if ((H >> q) & 1u)
			s.match = s.match == 0 ? s.k : s.match + 1;
		else
			s.match = 0;
		if (s.match >= s.min_len) {
			s.decided = EVAL_ACCEPT;
			return s.decided;
		}
		s.prev = pos;
	}
	return s.decided;
}

/*
 * HARMONIC and BINOMIAL scoring (SeqEval.h:116-193, 218-290): the walk of
 * evalSimple with a score kept in double (HARMONIC: a hit in a streak of s
 * earlier hits adds 1 - 1/(1 + s), a streak's first hit 0.5; BINOMIAL: every
 * hit adds 1 against an integer threshold).  The running score of HARMONIC is
 * a sum of doubles whose rounding depends on the order of the additions, so a
 * chunk is walked frame by frame, exactly as the reference iterates; every
 * lane runs the same walk on the chunk's ballots.
 */
enum { SEQ_HARMONIC = 2, SEQ_BINOMIAL = 3 };

struct SeqState {
	double score;
	double thres;        /* accept when thres <= score */
	double anti_thres;   /* reject when anti_thres <= anti */
	uint32_t anti;
	uint32_t streak;
	int64_t prev;        /* last iterated frame */
	int64_t skip_end;    /* frames below this belong to an open skip window */
	int32_t started;
	int32_t in_skip;
	int32_t mode;        /* SEQ_HARMONIC or SEQ_BINOMIAL */
	int32_t decided;
};

/* thres / antiThres of HARMONIC (as evalSimple computes them). */
BBT_HD void harmonic_init(SeqState &s, double threshold, double one_minus, uint64_t frames)
{
	double fr = (double)frames;
	double thres = threshold * fr;
	double anti = one_minus * fr;
#if defined(__CUDA_ARCH__)
	thres = __dmul_rn(threshold, fr);
	anti = __dmul_rn(one_minus, fr);
#endif
	s.score = 0.0;
	s.thres = thres;
	s.anti_thres = floor(anti);
	s.anti = 0;
	s.streak = 0;
	s.prev = 0;
	s.skip_end = 0;
	s.started = 0;
	s.in_skip = 0;
	s.mode = SEQ_HARMONIC;
	s.decided = EVAL_OPEN;
}

/* BINOMIAL: thres = calcMinCount(frameLen, fpr, minFPR), computed on the host. */
BBT_HD void binomial_init(SeqState &s, uint32_t thres, uint32_t frame_len)
{
	s.score = 0.0;
	s.thres = (double)thres;
	s.anti_thres = (double)(uint32_t)(frame_len - thres); /* unsigned, as upstream */
	s.anti = 0;
	s.streak = 0;
	s.prev = 0;
	s.skip_end = 0;
	s.started = 0;
	s.in_skip = 0;
	s.mode = SEQ_BINOMIAL;
	s.decided = EVAL_OPEN;
}

/* Frames below this are not probed (an open skip window). */
BBT_HD int64_t seq_probe_from(const SeqState &s)
{
	return s.in_skip ? s.skip_end : 0;
}

BBT_HD double harmonic_add(double score, uint32_t streak)
{
#if defined(__CUDA_ARCH__)
	if (streak == 0)
		return __dadd_rn(score, 0.5);
	return __dadd_rn(score, __dsub_rn(1.0, __ddiv_rn(1.0, __dadd_rn(1.0, (double)streak))));
#else
	if (streak == 0)
		return score + 0.5;
	return score + (1.0 - 1.0 / (1.0 + (double)streak));
#endif
}

/* Walk the valid frames of one chunk (frame j = base + j, j < nf); H holds the
 * hits of the frames probed (those at or after seq_probe_from when the chunk
 * began).  alg receives the frames the reference probes. */
BBT_HD int seq_chunk(SeqState &s, uint32_t V, uint32_t H, int64_t base, int nf, int k,
		uint32_t streak_thr, uint32_t *alg = nullptr)
{
	if (s.decided)
		return s.decided;
	V &= low_mask(nf);
	H &= V;
	int from = 0;
	/* Without probe accounting, runs of misses outside a skip window are
	 * settled at once: each visited frame adds its gap and 1 to antiScore, so
	 * a run adds (last frame - previous frame) and leaves the streak at 0,
	 * and a rejection inside it is final before the next hit.  Only a miss
	 * right after a streak of streak_thr hits (it opens a skip window) goes to
	 * the frame-by-frame walk below. */
	if (!alg && s.started && !s.in_skip && streak_thr >= 1) {
		for (;;) {
			const uint32_t hm = H & ~low_mask(from);
			const int h = hm ? lowbit32(hm) : nf;
			const uint32_t mm = V & ~H & range_mask(from, h);
			if (mm) {
				const int64_t p0 = base + lowbit32(mm);
				if (p0 == s.prev + 1 && s.streak >= streak_thr)
					break; /* opens a skip window */
				const int64_t pl = base + highbit32(mm);
				s.anti += (uint32_t)(pl - s.prev);
				s.prev = pl;
				s.streak = 0;
				if (s.anti_thres <= (double)s.anti)
					return s.decided = EVAL_REJECT;
			}
			if (h >= nf)
				return EVAL_OPEN;
			const int64_t p = base + h;
			if (p != s.prev + 1) {
				s.anti += (uint32_t)(p - s.prev - 1);
				if (s.anti_thres <= (double)s.anti)
					return s.decided = EVAL_REJECT;
				s.streak = 0;
			}
			s.score = s.mode == SEQ_BINOMIAL ? s.score + 1.0 : harmonic_add(s.score, s.streak);
			if (s.thres <= s.score)
				return s.decided = EVAL_ACCEPT;
			s.prev = p;
			++s.streak;
			from = h + 1;
		}
	}
	uint32_t x = V & ~low_mask(from);
	while (x) {
		const int q = lowbit32(x);
		x &= x - 1;
		const int64_t p = base + q;
		if (s.in_skip && p < s.skip_end) { /* iterated inside a skip window, not probed */
			if (s.anti_thres <= (double)(++s.anti))
				return s.decided = EVAL_REJECT;
			s.prev = p;
			continue;
		}
		s.in_skip = 0;
		const bool hit = (H >> q) & 1u;
		if (!s.started) { /* the first frame: no gap check, no skip window */
			s.started = 1;
			if (alg)
				*alg |= 1u << q;
			if (hit) {
				s.score = s.mode == SEQ_BINOMIAL ? s.score + 1.0 : harmonic_add(s.score, 0);
				if (s.thres <= s.score)
					return s.decided = EVAL_ACCEPT;
				++s.streak;
			} else if (s.anti_thres <= (double)(++s.anti)) {
				return s.decided = EVAL_REJECT;
			}
			s.prev = p;
			continue;
		}
		if (p != s.prev + 1) {
			s.anti += (uint32_t)(p - s.prev - 1);
			if (s.anti_thres <= (double)s.anti)
				return s.decided = EVAL_REJECT;
			s.streak = 0;
		}
		if (alg) /* the reference probes the frame only after the gap check */
			*alg |= 1u << q;
		if (hit) {
			s.score = s.mode == SEQ_BINOMIAL ? s.score + 1.0 : harmonic_add(s.score, s.streak);
			if (s.thres <= s.score)
				return s.decided = EVAL_ACCEPT;
			s.prev = p;
			++s.streak;
		} else {
			if (s.streak >= streak_thr) { /* the window starts at this frame */
				s.in_skip = 1;
				s.skip_end = (int64_t)(uint32_t)((uint32_t)p + (uint32_t)k);
			}
			if (s.anti_thres <= (double)(++s.anti))
				return s.decided = EVAL_REJECT;
			s.prev = p;
			s.streak = 0;
		}
	}
	return s.decided;
}

/*
 * SeqEval::evalScore (Common/SeqEval.h:534-560): the exhaustive walks that
 * score a read against one filter without stopping early (BESTHIT and SCORES
 * modes).
 *   SIMPLE   evalSimpleScore (:334-376): +0.5 for a hit that starts a streak,
 *            +1 for a hit that continues one;
 *   HARMONIC evalHarmonicScore (:378-419): +0.5, then +1 - 1/(1 + streak);
 *   BINOMIAL evalBinomialScore (:450-491): +1 per hit (the count then goes
 *            through the binomial upper tail);
 * in all three a frame after an N gap (pos != prevPos + 1) starts a new streak,
 * and a miss that ends a streak of at least streakThreshold hits leaves the
 * frames below pos + k unprobed (they still move prevPos).  SIMPLE and
 * HARMONIC divide the sum by len - k + 1 (normalizeScore, :33-35).
 *   LENGTH   evalMinMatchLenScore (:421-448): every frame is probed; the value
 *            is the length of the run of hits that reaches the last frame (k
 *            for its first hit, +1 per further hit; a miss or a gap ends it).
 * Unlike evalSimple there is no first-frame special case: prevPos starts at 0
 * and the streak at 0, so the first frame's gap check changes nothing.
 */
enum { SCORE_SIMPLE = 0, SCORE_LENGTH = 1, SCORE_HARMONIC = 2, SCORE_BINOMIAL = 3 };

struct ScoreState {
	double score;        /* SIMPLE / HARMONIC sum; BINOMIAL hit count */
	uint32_t streak;
	uint32_t run;        /* LENGTH: the current match length */
	int64_t prev;        /* last iterated frame */
	int64_t skip_end;    /* frames below this are iterated without a probe */
};

BBT_HD void score_init(ScoreState &s)
{
	s.score = 0.0;
	s.streak = 0;
	s.run = 0;
	s.prev = 0;
	s.skip_end = 0;
}

/* Walk the valid frames of one chunk (frame j = base + j, j < nf); H holds the
 * hits of the frames probed (every frame for LENGTH, otherwise those at or
 * after skip_end when the chunk began).
 *
 * The walk goes by runs rather than frame by frame.  LENGTH only needs the
 * run of hits that reaches the chunk's last valid frame.  Otherwise: frames
 * inside an open skip window are passed over; a run of misses leaves the
 * streak at 0, and only its first frame can open a window (right after a
 * streak of streak_thr hits); a run of consecutive hits adds, for SIMPLE,
 * 0.5 for a first hit and 1 for each other (all partial sums are multiples
 * of 0.5, exact in a double, so one addition gives the sequential result),
 * for BINOMIAL 1 per hit, and for HARMONIC its terms one at a time in the
 * reference's order.  streak_thr = 0 (every miss opens a window) is walked
 * frame by frame. */
BBT_HD void score_chunk(ScoreState &s, uint32_t V, uint32_t H, int64_t base, int nf, int k,
		uint32_t streak_thr, int mode)
{
	V &= low_mask(nf);
	if (!V)
		return;
	H &= V;
	if (mode == SCORE_LENGTH) {
		const int last = highbit32(V);
		if ((H >> last) & 1u) {
			const int run = leading_ones32(H << (31 - last));
			const bool carry = last - run + 1 == 0 && s.run > 0 && s.prev == base - 1;
			s.run = carry ? s.run + (uint32_t)run : (uint32_t)k + (uint32_t)run - 1u;
		} else {
			s.run = 0;
		}
		s.prev = base + last;
		return;
	}
	if (streak_thr == 0) {
		uint32_t x = V;
		while (x) {
			const int q = lowbit32(x);
			x &= x - 1;
			const int64_t p = base + q;
			if (p < s.skip_end) {
				s.prev = p;
				continue;
			}
			if (p != s.prev + 1)
				s.streak = 0;
			if ((H >> q) & 1u) {
				s.score = mode == SCORE_HARMONIC ? harmonic_add(s.score, s.streak)
				        : mode == SCORE_BINOMIAL ? s.score + 1.0
				                                 : s.score + (s.streak ? 1.0 : 0.5);
				++s.streak;
			} else {
				s.skip_end = (int64_t)(uint32_t)((uint32_t)p + (uint32_t)k);
				s.streak = 0;
			}
			s.prev = p;
		}
		return;
	}
	int j = 0;
	for (;;) {
		/* frames inside an open skip window: iterated, not probed */
		const int64_t se = s.skip_end - base;
		if (se > j) {
			const int e = se >= nf ? nf : (int)se;
			const uint32_t w = V & range_mask(j, e);
			if (w)
				s.prev = base + highbit32(w);
			j = e;
			if (j >= nf)
				return;
		}
		const uint32_t hm = H & ~low_mask(j);
		const int h = hm ? lowbit32(hm) : nf;
		const uint32_t mm = V & ~H & range_mask(j, h);
		if (mm) {
			const int m0 = lowbit32(mm);
			const int64_t p0 = base + m0;
			if (p0 == s.prev + 1 && s.streak >= streak_thr) {
				/* the window starts at this miss */
				s.skip_end = (int64_t)(uint32_t)((uint32_t)p0 + (uint32_t)k);
				s.streak = 0;
				s.prev = p0;
				j = m0 + 1;
				continue;
			}
			s.streak = 0;
			s.prev = base + highbit32(mm);
		}
		if (h >= nf)
			return;
		if (base + h != s.prev + 1)
			s.streak = 0;
		if (mode == SCORE_HARMONIC) {
			s.score = harmonic_add(s.score, s.streak);
			++s.streak;
			s.prev = base + h;
			j = h + 1;
		} else {
			const uint32_t rest = ~(H >> h);
			const int run = rest ? lowbit32(rest) : 32 - h;
			const double add = mode == SCORE_BINOMIAL ? (double)run
			                 : (s.streak ? (double)run : (double)run - 0.5);
			s.score = s.score + add;
			s.streak += (uint32_t)run;
			s.prev = base + h + run - 1;
			j = h + run;
		}
		if (j >= nf)
			return;
	}
}

/* The value of 0.0 / 0.0 on x86-64 (the negative default NaN), which is what
 * normalizeScore returns for a read of k - 1 bases. */
BBT_HD double x86_default_nan()
{
#if defined(__CUDA_ARCH__)
	return __longlong_as_double((long long)0xFFF8000000000000ull);
#else
	union {
		uint64_t u;
		double d;
	} v;
	v.u = 0xFFF8000000000000ull;
	return v.d;
#endif
}

/* normalizeScore (Common/SeqEval.h:33-35): score / (len - k + 1), the divisor
 * in size_t arithmetic (it wraps for len < k - 1; for len = k - 1 it is 0,
 * and so is the score: 0 / 0). */
BBT_HD double score_normalize(double score, uint64_t len, unsigned k)
{
	const uint64_t d = len - (uint64_t)k + 1u;
	if (d == 0)
		return x86_default_nan();
#if defined(__CUDA_ARCH__)
	return __ddiv_rn(score, __ull2double_rn(d));
#else
	return score / (double)d;
#endif
}

} // namespace bbt

#endif
