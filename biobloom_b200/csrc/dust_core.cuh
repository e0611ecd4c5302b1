/*
 * dust_core.cuh -- the SDUST scan of one read (dust.cu), compiled for the
 * device and for the host, where tests run it against the oracle.
 *
 * dust_scan follows Common/sdust.c (sdust_core, shift_window, find_perfect,
 * save_masked_regions) step for step, except that find_perfect keeps the
 * running maximum with a forward-only pointer and merges new perfect
 * intervals after the scan (see the comment there); it reports each masked
 * interval [a, b) to `mask` as the reference's result list grows (a new
 * interval, or the extension of the last one when they touch).
 */
#ifndef BBT_DUST_CORE_CUH
#define BBT_DUST_CORE_CUH

#include <stdint.h>

#if defined(__CUDACC__)
#define BBT_DHD __host__ __device__ __forceinline__
#else
#define BBT_DHD inline
#endif

namespace bbt {

struct DustPerfect {
	int start, finish, r, l;
};

BBT_DHD int dust_code(uint8_t c)
{
	switch (c) {
	case 'A': case 'a': return 0;
	case 'C': case 'c': return 1;
	case 'G': case 'g': return 2;
	case 'T': case 't': return 3;
	default: return 4;
	}
}

/* sdust over one read; false when the perfect list would exceed pcap
 * entries.  seq(i) returns base i (i = 0, 1, ... in order); ring: W bytes. */
template <class SeqFn, class MaskFn>
BBT_DHD bool dust_scan(SeqFn &&seq, uint64_t len, int T, int W, DustPerfect *perf,
		int pcap, uint8_t *ring, MaskFn &&mask)
{
	uint16_t cw[64], cv[64];
	for (int i = 0; i < 64; ++i)
		cw[i] = cv[i] = 0;
	int rw = 0, rv = 0, L = 0;
	int head = 0, size = 0;
	const int rcap = W; /* the window never holds more than W - 2 triplets */
	int np = 0;
	bool have_res = false;
	int res_f = 0;  /* finish of the last masked interval */
	/* ring index of window entry i (head, i < rcap) */
	auto slot = [&](int i) -> int {
		const int x = head + i;
		return x >= rcap ? x - rcap : x;
	};
	auto at = [&](int i) -> int { return ring[slot(i)]; };
	/* save_masked_regions */
	auto save = [&](int start) {
		if (np == 0 || perf[np - 1].start >= start)
			return;
		const DustPerfect p = perf[np - 1];
		if (have_res && p.start <= res_f) {
			const int nf = res_f > p.finish ? res_f : p.finish;
			if (nf > res_f)
				mask(res_f, nf);
			res_f = nf;
		} else {
			mask(p.start, p.finish);
			have_res = true;
			res_f = p.finish;
		}
		int i = np - 1;
		while (i >= 0 && perf[i].start < start)
			--i;
		np = i + 1;
	};
	int l = 0;
	unsigned t = 0;
	const int n = (int)len;
	for (int i = 0; i <= n; ++i) {
		const int b = i < n ? dust_code(seq(i)) : 4;
		if (b < 4) {
			++l;
			t = (t << 2 | (unsigned)b) & 63u;
			if (l < 3)
				continue;
			const int start = (l - W > 0 ? l - W : 0) + (i + 1 - l);
			save(start);
			/* shift_window */
			if (size >= W - 2) {
				const int s = ring[head];
				head = head + 1 == rcap ? 0 : head + 1;
				--size;
				rw -= --cw[s];
				if (L > size) {
					--L;
					rv -= --cv[s];
				}
			}
			ring[slot(size)] = (uint8_t)t;
			++size;
			++L;
			rw += cw[t]++;
			rv += cv[t]++;
			if (cv[t] * 10 > T * 2) {
				int s;
				do {
					s = at(size - L);
					rv -= --cv[s];
					--L;
				} while (s != (int)t);
			}
			if (rw * 10 <= L * T)
				continue;
			/* find_perfect.  The reference rescans the list from its head for
			 * every window suffix (O(W |perf|) per base); the same maximum is
			 * kept here with one pointer that only moves forward, because the
			 * suffixes come by decreasing start and the list is ordered by
			 * decreasing start.  Only ratios r/l are compared, so which of two
			 * equal-ratio entries holds the maximum does not matter.  New
			 * entries go to the top of the array (downwards) and are merged in
			 * after the scan at the positions the reference inserts them:
			 * after every older entry whose start is not smaller. */
			uint16_t c[64];
			for (int q = 0; q < 64; ++q)
				c[q] = cv[q];
			int r = rv, max_r = 0, max_l = 0;
			int jp = 0, nn = 0;
			for (int k = size - L - 1; k >= 0; --k) {
				const int tk = at(k);
				r += c[tk]++;
				const int new_r = r, new_l = size - k - 1;
				if (new_r * 10 <= T * new_l)
					continue;
				for (; jp < np && perf[jp].start >= k + start; ++jp) {
					const DustPerfect &p = perf[jp];
					if (max_r == 0 || p.r * max_l > max_r * p.l) {
						max_r = p.r;
						max_l = p.l;
					}
				}
				if (max_r == 0 || new_r * max_l >= max_r * new_l) {
					max_r = new_r;
					max_l = new_l;
					if (np + 2 * nn + 2 > pcap)
						return false;
					/* l (<= W <= 1024) and the insertion point among the older
					 * entries (< 2^21) share the l field until the merge */
					DustPerfect &e = perf[pcap - 1 - nn];
					e.start = k + start;
					e.finish = size + 2 + start;
					e.r = new_r;
					e.l = (int)((unsigned)jp << 11 | (unsigned)new_l);
					++nn;
				}
			}
			if (nn) {
				/* backward merge into [0, np + nn) */
				int w = np + nn - 1, io = np - 1;
				for (int ei = nn - 1; ei >= 0; --ei) {
					DustPerfect e = perf[pcap - 1 - ei];
					const int pos = (int)((unsigned)e.l >> 11);
					e.l = (int)((unsigned)e.l & 2047u);
					while (io >= pos)
						perf[w--] = perf[io--];
					perf[w--] = e;
				}
				np += nn;
			}
		} else {
			int start = (l - W + 1 > 0 ? l - W + 1 : 0) + (i + 1 - l);
			while (np)
				save(start++);
			l = 0;
			t = 0;
		}
	}
	return true;
}

} // namespace bbt

#endif
