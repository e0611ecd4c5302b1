/*
 * maker.cu -- Bloom filter construction on the device (biobloommaker's
 * BloomFilterGenerator::generate, BioBloomMaker/BloomFilterGenerator.cpp:54-73,
 * BloomFilterGenerator.h:108-188, with BloomFilterInfo sizing,
 * Common/BloomFilterInfo.h:57-76, and the hash-count rule of
 * BioBloomMaker.cpp:360-373).
 *
 * Every valid k-mer of every sequence sets its h bits with atomicOr.  The bit
 * array does not depend on insertion order, so it equals the sequential
 * maker's.  The counts of the .txt file do: BloomFilter::insertAndCheck
 * (loadFilter, BloomFilterGenerator.h:170-174) counts a k-mer as redundant
 * when all its bits were already set, which in a sequential insertion is when
 * every bit it maps to was first set by an earlier k-mer.  So with k-mers
 * numbered in insertion order (records in file order, k-mers left to right),
 * first[b] = the lowest number mapping to bit b is taken with atomicMin, and
 * k-mer i is new exactly when first[b] == i for one of its bits.  Those counts
 * are the reference's for a one-threaded run (and for any run whose records
 * each fit one thread, as a single-record genome does); its multi-threaded
 * runs race between records.  first[] covers the filter in slices of at most
 * 2^31 bits, each slice a pass over all k-mers.
 */
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <string>
#include <vector>

#include "bbt.h"
#include "bbt_device.cuh"
#include "ctx.hpp"
#include "formats.hpp"

namespace bbt {
namespace {

constexpr int kMakerSeg = 64; /* frames per thread */

enum MakerPass { kInsert, kFirst, kFresh };

/* One pass over the frames [0, nframes) of chunk s (bases [0, nframes + k - 1)
 * resident), numbered idx0 + q:
 *   kInsert: set the h bits; counts[0] += valid k-mers;
 *   kFirst:  first[b - lo] = min(first[b - lo], number) for bits b in
 *            [lo, lo + span);
 *   kFresh:  mark the k-mer new (bit `number` of fresh) when some bit b in
 *            the slice has first[b - lo] == number. */
template <int PASS, class IdxT>
__global__ void maker_kernel(const uint8_t *__restrict__ s, uint64_t nframes, uint64_t idx0,
		unsigned k, unsigned h, uint32_t *words, uint64_t m, uint64_t minv, IdxT *first,
		uint64_t lo, uint64_t span, uint32_t *fresh, unsigned long long *counts)
{
	const uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
	const uint64_t q0 = t * kMakerSeg;
	unsigned long long valid = 0;
	if (q0 < nframes) {
		const uint64_t qe = min(q0 + kMakerSeg, nframes);
		uint64_t fh = 0, rh = 0;
		int64_t lb = -1;
		for (unsigned i = 0; i < k; ++i) {
			uint8_t c = s[q0 + i];
			fh = rol1(fh) ^ seed_fw(c);
			if (!base_ok(c))
				lb = (int64_t)(q0 + i);
		}
		for (int i = (int)k - 1; i >= 0; --i)
			rh = rol1(rh) ^ seed_rc(s[q0 + i]);
		const uint64_t fk[4] = {rolk(kSeedA, k), rolk(kSeedC, k), rolk(kSeedG, k), rolk(kSeedT, k)};
		for (uint64_t q = q0;; ) {
			if (lb < (int64_t)q) {
				const uint64_t canon = fh < rh ? fh : rh;
				const uint64_t num = idx0 + q;
				bool is_first = false;
				for (unsigned i = 0; i < h; ++i) {
					const uint64_t v = i ? extra_hash(canon, k, i) : canon;
					const uint64_t b = reduce(v, m, minv);
					if (PASS == kInsert) {
						atomicOr(words + (b >> 5), 1u << (b & 31));
					} else if (b >= lo && b - lo < span) {
						if (PASS == kFirst)
							atomicMin(first + (b - lo), (IdxT)num);
						else
							is_first = is_first || first[b - lo] == (IdxT)num;
					}
				}
				valid += 1;
				if (PASS == kFresh && is_first)
					atomicOr(fresh + (num >> 5), 1u << (num & 31));
			}
			if (++q >= qe)
				break;
			uint8_t out = s[q - 1], in = s[q + k - 1];
			uint8_t u = out & 0xDF;
			uint64_t fo = u == 'A' ? fk[0] : u == 'C' ? fk[1] : u == 'G' ? fk[2] : u == 'T' ? fk[3] : 0;
			fh = rol1(fh) ^ fo ^ seed_fw(in);
			rh = ror1(rh) ^ ror1(seed_rc(out)) ^ rolk(seed_rc(in), k - 1);
			if (!base_ok(in))
				lb = (int64_t)(q + k - 1);
		}
	}
	if (PASS == kInsert) {
		for (int o = 16; o; o >>= 1)
			valid += __shfl_xor_sync(0xffffffffu, valid, o);
		if ((threadIdx.x & 31) == 0 && valid)
			atomicAdd(&counts[0], valid);
	}
}

/* counts[1] += set bits of w[0, n). */
__global__ void popcount_kernel(const uint32_t *w, uint64_t n, unsigned long long *counts)
{
	unsigned long long c = 0;
	for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
			i += (uint64_t)gridDim.x * blockDim.x)
		c += __popc(w[i]);
	for (int o = 16; o; o >>= 1)
		c += __shfl_xor_sync(0xffffffffu, c, o);
	if ((threadIdx.x & 31) == 0 && c)
		atomicAdd(&counts[1], c);
}

/* BloomFilterInfo::calcRedunancyFPR (Common/BloomFilterInfo.cpp:289-297) is
 * sum_{i=1}^{n-1} approxFPR(size, i, h) / n; it is evaluated exactly up to
 * 2^20 terms and by Simpson's rule (a smooth, monotone integrand) above. */
double redundancy_fpr(uint64_t size, uint64_t n, unsigned h)
{
	if (n < 2)
		return 0.0;
	auto f = [&](double i) {
		return std::pow(1.0 - std::exp(i * h * std::log1p(-1.0 / (double)size)), (double)h);
	};
	double sum = 0;
	if (n <= (1u << 20)) {
		for (uint64_t i = 1; i < n; ++i)
			sum += f((double)i);
	} else {
		const int N = 1 << 16;
		double a = 1.0, b = (double)(n - 1), dx = (b - a) / N;
		double integ = f(a) + f(b);
		for (int j = 1; j < N; ++j)
			integ += f(a + j * dx) * ((j & 1) ? 4.0 : 2.0);
		integ *= dx / 3.0;
		sum = integ + 0.5 * (f(a) + f(b));
	}
	return sum / (double)n;
}

} // namespace
} // namespace bbt

using namespace bbt;

extern "C" int bbt_make_filter(const char *seq, const uint64_t *offsets, uint64_t n_seqs,
		unsigned k, double fpr, unsigned hash_num, uint64_t entries, const char *stem,
		const char *filter_id, const char *sources, int device)
{
	if (!seq || !offsets || n_seqs == 0 || k == 0 || k > 255 || !stem || !filter_id)
		return fail(nullptr, BBT_ERR_ARG, "bbt_make_filter: invalid argument");
	if (!(fpr > 0 && fpr < 1))
		return fail(nullptr, BBT_ERR_ARG, "bbt_make_filter: FPR must be in (0, 1)");
	uint64_t expected = entries;
	if (!expected)
		for (uint64_t i = 0; i < n_seqs; ++i)
			expected += (offsets[i + 1] - offsets[i]) - k + 1; /* size_t wrap as upstream */
	const unsigned h = hash_num ? hash_num : optimal_hash_num(fpr);
	if (h == 0 || h > 64)
		return fail(nullptr, BBT_ERR_ARG, "bbt_make_filter: hash count out of range");
	const uint64_t m = optimal_size(expected, fpr, h);
	cudaError_t e = cudaSetDevice(device);
	if (e != cudaSuccess)
		return cuda_fail(nullptr, e, "cudaSetDevice");
	uint32_t *d_words = nullptr;
	uint8_t *d_seq = nullptr;
	unsigned long long *d_counts = nullptr;
	void *d_first = nullptr;
	uint32_t *d_fresh = nullptr;
	const uint64_t chunk = 256ull << 20;
	std::vector<uint8_t> host;
	uint64_t nframes_total = 0;
	for (uint64_t r = 0; r < n_seqs; ++r) {
		const uint64_t len = offsets[r + 1] - offsets[r];
		nframes_total += len >= k ? len - k + 1 : 0;
	}
	/* k-mer numbers fit 32 bits (all ones meaning "none") below 2^32 - 1 frames */
	const bool narrow = nframes_total < 0xffffffffull;
	const size_t isz = narrow ? sizeof(uint32_t) : sizeof(unsigned long long);
	const uint64_t span = std::min<uint64_t>(m, 1ull << 31);
	const int npass = 1 + 2 * (int)((m + span - 1) / span);
	int rc = BBT_OK;
#define MK_TRY(call)                                   \
	do {                                               \
		cudaError_t e_ = (call);                       \
		if (e_ != cudaSuccess) {                       \
			rc = cuda_fail(nullptr, e_, #call);        \
			goto out;                                  \
		}                                              \
	} while (0)
	MK_TRY(cudaMalloc(&d_words, m / 8));
	MK_TRY(cudaMemset(d_words, 0, m / 8));
	MK_TRY(cudaMalloc(&d_seq, chunk + k));
	MK_TRY(cudaMalloc(&d_counts, 2 * sizeof(unsigned long long)));
	MK_TRY(cudaMemset(d_counts, 0, 2 * sizeof(unsigned long long)));
	MK_TRY(cudaMalloc(&d_first, span * isz));
	MK_TRY(cudaMalloc(&d_fresh, (nframes_total / 32 + 1) * sizeof(uint32_t)));
	MK_TRY(cudaMemset(d_fresh, 0, (nframes_total / 32 + 1) * sizeof(uint32_t)));
	/* the insertion pass, then per slice of bits the first-number pass and the
	 * new-k-mer pass; each pass streams every sequence through d_seq */
	for (int pass = 0; pass < npass; ++pass) {
		const uint64_t lo = pass == 0 ? 0 : (uint64_t)((pass - 1) / 2) * span;
		const uint64_t sp = pass == 0 ? 0 : std::min(span, m - lo);
		if (pass & 1)
			MK_TRY(cudaMemset(d_first, 0xff, sp * isz));
		uint64_t idx0 = 0;
		for (uint64_t r = 0; r < n_seqs; ++r) {
			const uint64_t len = offsets[r + 1] - offsets[r];
			if (len < k)
				continue;
			const uint64_t frames = len - k + 1;
			for (uint64_t f0 = 0; f0 < frames; f0 += chunk) {
				const uint64_t nfr = std::min(chunk, frames - f0);
				MK_TRY(cudaMemcpy(d_seq, seq + offsets[r] + f0, nfr + k - 1,
						cudaMemcpyHostToDevice));
				const uint64_t threads = (nfr + kMakerSeg - 1) / kMakerSeg;
				const unsigned bs = 256, grid = (unsigned)((threads + bs - 1) / bs);
				const uint64_t i0 = idx0 + f0, minv = ~0ull / m;
				if (pass == 0) {
					maker_kernel<kInsert, uint32_t><<<grid, bs>>>(d_seq, nfr, i0, k, h, d_words,
							m, minv, nullptr, 0, 0, nullptr, d_counts);
				} else if (narrow) {
					uint32_t *fi = (uint32_t *)d_first;
					if (pass & 1)
						maker_kernel<kFirst, uint32_t><<<grid, bs>>>(d_seq, nfr, i0, k, h,
								nullptr, m, minv, fi, lo, sp, nullptr, nullptr);
					else
						maker_kernel<kFresh, uint32_t><<<grid, bs>>>(d_seq, nfr, i0, k, h,
								nullptr, m, minv, fi, lo, sp, d_fresh, nullptr);
				} else {
					unsigned long long *fi = (unsigned long long *)d_first;
					if (pass & 1)
						maker_kernel<kFirst, unsigned long long><<<grid, bs>>>(d_seq, nfr, i0, k,
								h, nullptr, m, minv, fi, lo, sp, nullptr, nullptr);
					else
						maker_kernel<kFresh, unsigned long long><<<grid, bs>>>(d_seq, nfr, i0, k,
								h, nullptr, m, minv, fi, lo, sp, d_fresh, nullptr);
				}
				MK_TRY(cudaGetLastError());
			}
			idx0 += frames;
		}
	}
	popcount_kernel<<<256, 256>>>(d_fresh, nframes_total / 32 + 1, d_counts);
	MK_TRY(cudaGetLastError());
	{
		unsigned long long cnt[2];
		MK_TRY(cudaMemcpy(cnt, d_counts, sizeof cnt, cudaMemcpyDeviceToHost));
		/* counted: cnt[0] valid k-mers, cnt[1] new ones; below cnt[0] new and
		 * cnt[1] redundant */
		const unsigned long long fresh_n = cnt[1];
		cnt[1] = cnt[0] - fresh_n;
		cnt[0] = fresh_n;
		host.resize(m / 8);
		MK_TRY(cudaMemcpy(host.data(), d_words, m / 8, cudaMemcpyDeviceToHost));
		BfHeader hd;
		hd.m = m;
		hd.h = h;
		hd.k = k;
		/* the reference maker stores a BloomFilter built from (size, hash
		 * count, k) (BloomFilterGenerator.cpp:63-71), whose FPR and entry
		 * fields the header carries as 0; the counts go to the .txt file */
		hd.dfpr = 0;
		hd.n_entry = 0;
		hd.t_entry = 0;
		std::string bf = std::string(stem) + ".bf";
		FILE *f = fopen(bf.c_str(), "wb");
		if (!f) {
			rc = fail(nullptr, BBT_ERR_IO, "cannot write " + bf);
			goto out;
		}
		bool ok = write_bf_header(f, hd) == 0 && fwrite(host.data(), 1, host.size(), f) == host.size();
		ok = (fclose(f) == 0) && ok;
		if (!ok) {
			rc = fail(nullptr, BBT_ERR_IO, "cannot write " + bf);
			goto out;
		}
		InfoFile info;
		info.filter_id = filter_id;
		info.kmer_size = k;
		info.fpr = fpr;
		info.hash_num = h;
		info.expected = expected;
		info.sources = sources ? sources : "";
		info.size = m;
		info.num_entries = cnt[0];
		info.approx_fpr = approx_fpr(m, cnt[0], h);
		info.redundant = cnt[1];
		info.redundant_fpr = redundancy_fpr(m, cnt[0], h);
		if (!write_info(std::string(stem) + ".txt", info))
			rc = fail(nullptr, BBT_ERR_IO, std::string("cannot write ") + stem + ".txt");
	}
out:
	cudaFree(d_words);
	cudaFree(d_seq);
	cudaFree(d_counts);
	cudaFree(d_first);
	cudaFree(d_fresh);
	return rc;
#undef MK_TRY
}
