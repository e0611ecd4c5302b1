/*
 * mibf_make.cu -- building a miBF on the GPU (bbt_mibf_make).
 *
 * Replaces MIBFGen::generate (BioBloomMaker/MIBFGen.hpp:131-430), restated as
 * three order-free passes over every (sequence, frame):
 *   1. set bit v mod m of each of the frame's h values (atomicOr);
 *   2. rank the bit vector (popcount + exclusive scan), then offer the
 *      sequence's ID to each value's slot: the slot keeps the largest
 *      (priority(slot, id) << 16 | id) (atomicMax), priority = the top 16 bits
 *      of splitmix64's finalizer of (slot ^ id * 0x9e3779b97f4a7c15);
 *   3. for a frame none of whose h slots its ID owns, set the saturation bit
 *      (0x8000) of all h slots (atomicOr on the 32-bit word holding the ID).
 * Because no pass depends on the order of the updates, the files are the same
 * on every run and equal to the oracle's sequential build.
 */
#include <cuda_runtime.h>

#include <cub/device/device_scan.cuh>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <string>
#include <vector>

#include "bbt_device.cuh"
#include "mibf_ctx.hpp"
#include "window.cuh"

namespace bbt {

struct MakeArgs {
	const uint8_t *seq;
	const uint64_t *off;
	const uint16_t *sid;
	uint64_t n_seqs, total;
	uint32_t k, h, nse;
	int kmer_mode;
	uint64_t m, minv;
	const unsigned long long *tables;
};

__device__ __forceinline__ uint64_t mix64(uint64_t z)
{
	z += 0x9e3779b97f4a7c15ULL;
	z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
	z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
	return z ^ (z >> 31);
}

/* Sequence holding position q: the last i with off[i] <= q. */
__device__ __forceinline__ uint64_t seq_of(const uint64_t *off, uint64_t n, uint64_t q)
{
	uint64_t lo = 0, hi = n; /* off[lo] <= q < off[hi] */
	while (hi - lo > 1) {
		const uint64_t mid = (lo + hi) >> 1;
		if (off[mid] <= q)
			lo = mid;
		else
			hi = mid;
	}
	return lo;
}

/* The frame at global position q: false if it crosses the end of its sequence
 * or holds a base that is not ACGT; else its h values and its sequence ID. */
__device__ __forceinline__ bool frame_values(const MakeArgs &a, const ulonglong2 *tab, uint64_t q,
		uint64_t *vals, uint32_t &id)
{
	const uint64_t i = seq_of(a.off, a.n_seqs, q);
	if (q + a.k > a.off[i + 1])
		return false;
	uint64_t w = 0;
	for (uint32_t j = 0; j < a.k; ++j) {
		const uint8_t c = base_code(a.seq[q + j]);
		if (c > 3)
			return false;
		w |= (uint64_t)c << (2 * j);
	}
	id = a.sid[i];
	for (uint32_t s = 0; s < a.nse; ++s) {
		uint64_t F = 0, R = 0;
		const ulonglong2 *t = tab + s * 128;
		for (uint32_t j = 0; j < a.k; ++j) {
			const ulonglong2 e = t[j * 4 + ((w >> (2 * j)) & 3u)];
			F ^= e.x;
			R ^= e.y;
		}
		vals[s] = F < R ? F : R;
	}
	if (a.kmer_mode)
		for (uint32_t v = 1; v < a.h; ++v)
			vals[v] = extra_hash(vals[0], a.k, v);
	return true;
}

__device__ __forceinline__ void load_tables(const MakeArgs &a, unsigned long long *sm)
{
	for (uint32_t i = threadIdx.x; i < a.nse * 256; i += blockDim.x)
		sm[i] = a.tables[i];
	__syncthreads();
}

__global__ void make_pass1(MakeArgs a, uint32_t *raw)
{
	extern __shared__ __align__(16) unsigned long long sm[];
	load_tables(a, sm);
	const ulonglong2 *tab = reinterpret_cast<const ulonglong2 *>(sm);
	uint64_t vals[kMibfMaxSeeds];
	for (uint64_t q = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; q < a.total;
			q += (uint64_t)gridDim.x * blockDim.x) {
		uint32_t id;
		if (!frame_values(a, tab, q, vals, id))
			continue;
		for (uint32_t v = 0; v < a.h; ++v) {
			const uint64_t p = reduce(vals[v], a.m, a.minv);
			atomicOr(raw + (p >> 5), 1u << (p & 31));
		}
	}
}

__device__ __forceinline__ uint64_t slot_of(const uint32_t *raw, const unsigned long long *rank,
		uint64_t p)
{
	const uint64_t w = ((const uint64_t *)raw)[p >> 6];
	const uint64_t below = (p & 63) ? (w & ((1ull << (p & 63)) - 1)) : 0ull;
	return rank[p >> 6] + (uint64_t)__popcll(below);
}

__global__ void make_pass2(MakeArgs a, const uint32_t *raw, const unsigned long long *rank,
		uint32_t *best)
{
	extern __shared__ __align__(16) unsigned long long sm[];
	load_tables(a, sm);
	const ulonglong2 *tab = reinterpret_cast<const ulonglong2 *>(sm);
	uint64_t vals[kMibfMaxSeeds];
	for (uint64_t q = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; q < a.total;
			q += (uint64_t)gridDim.x * blockDim.x) {
		uint32_t id;
		if (!frame_values(a, tab, q, vals, id))
			continue;
		for (uint32_t v = 0; v < a.h; ++v) {
			const uint64_t slot = slot_of(raw, rank, reduce(vals[v], a.m, a.minv));
			const uint32_t pr = (uint32_t)(mix64(slot ^ ((uint64_t)id * 0x9e3779b97f4a7c15ULL)) >> 48);
			atomicMax(best + slot, (pr << 16) | id);
		}
	}
}

__global__ void make_ids(const uint32_t *best, uint64_t pop, uint16_t *ids)
{
	for (uint64_t s = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; s < pop;
			s += (uint64_t)gridDim.x * blockDim.x)
		ids[s] = (uint16_t)(best[s] & 0xFFFFu);
}

__global__ void make_pass3(MakeArgs a, const uint32_t *raw, const unsigned long long *rank,
		uint16_t *ids)
{
	extern __shared__ __align__(16) unsigned long long sm[];
	load_tables(a, sm);
	const ulonglong2 *tab = reinterpret_cast<const ulonglong2 *>(sm);
	uint64_t vals[kMibfMaxSeeds];
	uint32_t *ids32 = reinterpret_cast<uint32_t *>(ids);
	for (uint64_t q = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; q < a.total;
			q += (uint64_t)gridDim.x * blockDim.x) {
		uint32_t id;
		if (!frame_values(a, tab, q, vals, id))
			continue;
		bool owned = false;
		for (uint32_t v = 0; v < a.h; ++v) {
			const uint64_t slot = slot_of(raw, rank, reduce(vals[v], a.m, a.minv));
			vals[v] = slot;
			/* the low 15 bits do not change in this pass; bit 15 may */
			const uint32_t word = ((volatile uint32_t *)ids32)[slot >> 1];
			const uint32_t e = (slot & 1) ? word >> 16 : word & 0xFFFFu;
			owned |= (e & 0x7FFFu) == id;
		}
		if (!owned)
			for (uint32_t v = 0; v < a.h; ++v)
				atomicOr(ids32 + (vals[v] >> 1), (uint32_t)kMibfSat << (16 * (vals[v] & 1)));
	}
}

__global__ void word_pop(const uint64_t *raw, uint64_t n, unsigned long long *pop)
{
	for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
			i += (uint64_t)gridDim.x * blockDim.x)
		pop[i] = (unsigned long long)__popcll(raw[i]);
}

} // namespace bbt

using namespace bbt;

namespace {

struct DevBuf {
	void *p = nullptr;
	~DevBuf() { cudaFree(p); }
};

int make_fail(const std::string &msg, int code)
{
	return mibf_fail(nullptr, code, msg);
}

} // namespace

#define MK_TRY(call)                                                                       \
	do {                                                                                   \
		cudaError_t e_ = (call);                                                           \
		if (e_ != cudaSuccess)                                                             \
			return make_fail(std::string(#call) + ": " + cudaGetErrorString(e_),           \
					e_ == cudaErrorMemoryAllocation ? BBT_ERR_NOMEM : BBT_ERR_CUDA);     \
	} while (0)

extern "C" int bbt_mibf_make(const char *seq, const uint64_t *offsets, const uint16_t *seq_id,
		uint64_t n_seqs, const char *const *names, unsigned n_names, const char *const *seeds,
		unsigned n_seeds, unsigned k, unsigned hash_num, double occupancy, int location,
		const char *prefix, int device)
{
	if (!seq || !offsets || !seq_id || n_seqs == 0 || !prefix || !names)
		return make_fail("bbt_mibf_make: missing argument", BBT_ERR_ARG);
	if (k == 0 || k > kMibfMaxK)
		return make_fail("bbt_mibf_make: k must be between 1 and 32", BBT_ERR_ARG);
	if (n_seeds > kMibfMaxSeeds || (!n_seeds && (hash_num == 0 || hash_num > kMibfMaxSeeds)))
		return make_fail("bbt_mibf_make: 1 to 16 seeds or hash functions", BBT_ERR_ARG);
	if (!(occupancy > 0.0 && occupancy < 1.0))
		return make_fail("bbt_mibf_make: occupancy must be in (0, 1)", BBT_ERR_ARG);
	MibfHeader hd;
	hd.k = k;
	for (unsigned i = 0; i < n_seeds; ++i) {
		std::string s = seeds[i] ? seeds[i] : "";
		if (s.size() != k || s.find_first_not_of("01") != std::string::npos)
			return make_fail("bbt_mibf_make: seeds are '0'/'1' strings of length k", BBT_ERR_ARG);
		hd.seeds.push_back(s);
	}
	hd.h = n_seeds ? n_seeds : hash_num;
	MK_TRY(cudaSetDevice(device));
	int sms = 0;
	cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
	/* offsets / IDs on the host, for sizing */
	std::vector<uint64_t> h_off(n_seqs + 1);
	if (location == BBT_DEVICE)
		MK_TRY(cudaMemcpy(h_off.data(), offsets, (n_seqs + 1) * 8, cudaMemcpyDeviceToHost));
	else
		memcpy(h_off.data(), offsets, (n_seqs + 1) * 8);
	uint64_t expected = 0;
	for (uint64_t i = 0; i < n_seqs; ++i)
		expected += (h_off[i + 1] - h_off[i]) - k + 1; /* size_t arithmetic, as MIBFGen */
	const double mb = std::ceil((double)expected * hd.h / -std::log(1.0 - occupancy));
	uint64_t m = (uint64_t)mb;
	m += (64 - m % 64) % 64;
	if (m == 0)
		m = 64;
	hd.m = m;
	const uint64_t base = h_off[0], total = h_off[n_seqs] - base;
	DevBuf dseq, doff, dsid, draw, drank, dpop, dtmp, dbest, dids, dtab;
	const uint8_t *d_seq = (const uint8_t *)seq;
	const uint64_t *d_off = offsets;
	const uint16_t *d_sid = seq_id;
	std::vector<uint64_t> rel(n_seqs + 1);
	for (uint64_t i = 0; i <= n_seqs; ++i)
		rel[i] = h_off[i] - base;
	MK_TRY(cudaMalloc(&doff.p, (n_seqs + 1) * 8));
	MK_TRY(cudaMemcpy(doff.p, rel.data(), (n_seqs + 1) * 8, cudaMemcpyHostToDevice));
	d_off = (const uint64_t *)doff.p;
	if (location != BBT_DEVICE) {
		MK_TRY(cudaMalloc(&dseq.p, std::max<uint64_t>(total, 1)));
		MK_TRY(cudaMemcpy(dseq.p, seq + base, total, cudaMemcpyHostToDevice));
		MK_TRY(cudaMalloc(&dsid.p, n_seqs * 2));
		MK_TRY(cudaMemcpy(dsid.p, seq_id, n_seqs * 2, cudaMemcpyHostToDevice));
		d_seq = (const uint8_t *)dseq.p;
		d_sid = (const uint16_t *)dsid.p;
	} else {
		d_seq = (const uint8_t *)seq + base;
	}
	std::vector<unsigned long long> tabs = mibf_seed_tables(hd.seeds, k);
	MK_TRY(cudaMalloc(&dtab.p, tabs.size() * 8));
	MK_TRY(cudaMemcpy(dtab.p, tabs.data(), tabs.size() * 8, cudaMemcpyHostToDevice));
	MakeArgs a;
	a.seq = d_seq;
	a.off = d_off;
	a.sid = d_sid;
	a.n_seqs = n_seqs;
	a.total = total;
	a.k = k;
	a.h = hd.h;
	a.kmer_mode = hd.seeds.empty();
	a.nse = a.kmer_mode ? 1 : hd.h;
	a.m = m;
	a.minv = ~0ull / m;
	a.tables = (const unsigned long long *)dtab.p;
	const size_t smem = (size_t)a.nse * 2048;
	const int grid = sms * 8;
	const uint64_t nwords = m / 64;
	MK_TRY(cudaMalloc(&draw.p, m / 8));
	MK_TRY(cudaMemset(draw.p, 0, m / 8));
	make_pass1<<<grid, 256, smem>>>(a, (uint32_t *)draw.p);
	MK_TRY(cudaGetLastError());
	MK_TRY(cudaMalloc(&dpop.p, nwords * 8));
	MK_TRY(cudaMalloc(&drank.p, (nwords + 1) * 8));
	word_pop<<<grid, 256>>>((const uint64_t *)draw.p, nwords, (unsigned long long *)dpop.p);
	size_t tmp_bytes = 0;
	cub::DeviceScan::ExclusiveSum(nullptr, tmp_bytes, (unsigned long long *)dpop.p,
			(unsigned long long *)drank.p, (int64_t)nwords);
	MK_TRY(cudaMalloc(&dtmp.p, tmp_bytes));
	cub::DeviceScan::ExclusiveSum(dtmp.p, tmp_bytes, (unsigned long long *)dpop.p,
			(unsigned long long *)drank.p, (int64_t)nwords);
	MK_TRY(cudaDeviceSynchronize());
	unsigned long long last_rank = 0, last_pop = 0;
	MK_TRY(cudaMemcpy(&last_rank, (unsigned long long *)drank.p + nwords - 1, 8,
			cudaMemcpyDeviceToHost));
	MK_TRY(cudaMemcpy(&last_pop, (unsigned long long *)dpop.p + nwords - 1, 8,
			cudaMemcpyDeviceToHost));
	const uint64_t pop = last_rank + last_pop;
	hd.pop = pop;
	cudaFree(dpop.p);
	dpop.p = nullptr;
	cudaFree(dtmp.p);
	dtmp.p = nullptr;
	MK_TRY(cudaMalloc(&dbest.p, std::max<uint64_t>(pop, 1) * 4));
	MK_TRY(cudaMemset(dbest.p, 0, std::max<uint64_t>(pop, 1) * 4));
	make_pass2<<<grid, 256, smem>>>(a, (const uint32_t *)draw.p,
			(const unsigned long long *)drank.p, (uint32_t *)dbest.p);
	MK_TRY(cudaGetLastError());
	MK_TRY(cudaMalloc(&dids.p, (std::max<uint64_t>(pop, 1) + 1) * 2));
	MK_TRY(cudaMemset(dids.p, 0, (std::max<uint64_t>(pop, 1) + 1) * 2));
	make_ids<<<grid, 256>>>((const uint32_t *)dbest.p, pop, (uint16_t *)dids.p);
	MK_TRY(cudaDeviceSynchronize());
	cudaFree(dbest.p);
	dbest.p = nullptr;
	make_pass3<<<grid, 256, smem>>>(a, (const uint32_t *)draw.p,
			(const unsigned long long *)drank.p, (uint16_t *)dids.p);
	MK_TRY(cudaDeviceSynchronize());
	/* files */
	const std::string pre = prefix;
	FILE *f = fopen((pre + ".bf").c_str(), "wb");
	if (!f)
		return make_fail("cannot write " + pre + ".bf", BBT_ERR_IO);
	int rc = write_mibf_header(f, hd);
	std::vector<uint16_t> hbuf;
	const uint64_t step = 1ull << 26;
	for (uint64_t done = 0; rc == 0 && done < pop;) {
		const uint64_t n = std::min(step, pop - done);
		hbuf.resize(n);
		if (cudaMemcpy(hbuf.data(), (uint16_t *)dids.p + done, n * 2, cudaMemcpyDeviceToHost) !=
				cudaSuccess || fwrite(hbuf.data(), 2, n, f) != n)
			rc = -1;
		done += n;
	}
	if (fclose(f) || rc)
		return make_fail("cannot write " + pre + ".bf", BBT_ERR_IO);
	f = fopen((pre + ".sdsl").c_str(), "wb");
	if (!f)
		return make_fail("cannot write " + pre + ".sdsl", BBT_ERR_IO);
	std::vector<uint64_t> wbuf;
	for (uint64_t done = 0; rc == 0 && done < nwords;) {
		const uint64_t n = std::min(step, nwords - done);
		wbuf.resize(n);
		if (cudaMemcpy(wbuf.data(), (uint64_t *)draw.p + done, n * 8, cudaMemcpyDeviceToHost) !=
				cudaSuccess || fwrite(wbuf.data(), 8, n, f) != n)
			rc = -1;
		done += n;
	}
	if (fclose(f) || rc)
		return make_fail("cannot write " + pre + ".sdsl", BBT_ERR_IO);
	std::ofstream ids(pre + "_ids.txt");
	for (unsigned i = 0; i < n_names; ++i)
		ids << (i + 1) << "\t" << (names[i] ? names[i] : "") << "\n";
	if (!ids)
		return make_fail("cannot write " + pre + "_ids.txt", BBT_ERR_IO);
	return BBT_OK;
}
