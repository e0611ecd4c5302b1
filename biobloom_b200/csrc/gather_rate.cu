/*
 * gather_rate.cu -- the random-gather ceilings of the GPU the library runs on.
 *
 * Every Bloom probe is an isolated 4-byte read at a random position of a bit
 * array.  How many such reads the GPU serves per second depends on where the
 * array lives: inside L2 (126 MB on B200) every read is an L2 sector access;
 * in HBM each read costs a DRAM line fill.  bbt_measure_gather times random
 * 4-byte gathers into a table of a given size, in the access pattern of a
 * probe-resolving kernel: 4-byte positions streamed from device memory (read
 * once, marked evict-first so they do not push the table out of L2), eight
 * independent gathers in flight per thread, one bit kept per gather and the
 * bits of 32 gathers written as one word.  Warps take their chunks of
 * gathers from a counter, as the persistent classify kernel takes reads: on
 * B200 a grid-stride loop over a grid of exactly one resident wave served
 * random gathers into a 2 GB table at 39.7 G/s, the same grid taking chunks
 * from a counter at 50.8 G/s (and a grid of two or more waves in a
 * grid-stride loop at 48.8 G/s); each gather is a 128-byte DRAM line fill
 * either way (122.6 bytes of DRAM reads per gather), so the counter-driven
 * rate is ~6.2 TB/s of line fills.  Used to choose how large a filter range
 * one probe pass may cover and to state the ceilings the kernels are measured
 * against.
 */
#include <cuda_runtime.h>

#include <algorithm>
#include <vector>

#include "bbt.h"
#include "bbt_device.cuh"
#include "ctx.hpp"

namespace bbt {
namespace {

constexpr int kPerThread = 8;

__device__ __forceinline__ uint64_t mix64d(uint64_t z)
{
	z += 0x9e3779b97f4a7c15ULL;
	z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
	z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
	return z ^ (z >> 31);
}

/* positions[i] = a random bit of the table (bits = entries * 32) */
__global__ void positions_kernel(uint32_t *pos, uint64_t n, uint64_t bits, uint64_t seed)
{
	for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
			i += (uint64_t)gridDim.x * blockDim.x)
		pos[i] = (uint32_t)(mix64d(seed ^ i) % bits);
}

/* A warp takes kTake consecutive chunks per visit to the counter (lane 0
 * takes them): with one chunk per visit the counter itself limited tables
 * held in L2 (~204 G gathers/s). */
constexpr int kTake = 8;
__device__ __forceinline__ uint64_t next_take(unsigned long long *next, int lane)
{
	unsigned long long w = 0;
	if (lane == 0)
		w = atomicAdd(next, 1ull);
	return __shfl_sync(0xffffffffu, w, 0);
}

/* Resolve-shaped gathers: chunk c of 32 * kPerThread positions per warp. */
__global__ void __launch_bounds__(256) gather_stream_kernel(const uint32_t *__restrict__ pos,
		uint64_t n, const uint32_t *__restrict__ table, uint32_t *__restrict__ out,
		unsigned long long *next)
{
	const uint64_t pol = evict_first_policy();
	const int lane = threadIdx.x & 31;
	const uint64_t chunk = 32ull * kPerThread;
	for (uint64_t t = next_take(next, lane); t * kTake * chunk < n; t = next_take(next, lane))
	for (uint64_t w = t * kTake; w < (t + 1) * kTake && w * chunk < n; ++w) {
		const uint64_t base = w * chunk;
		uint32_t p[kPerThread], v[kPerThread];
#pragma unroll
		for (int j = 0; j < kPerThread; ++j) {
			const uint64_t i = base + (uint64_t)j * 32 + lane;
			p[j] = i < n ? ld_stream_u32(pos + i, pol) : 0u;
		}
#pragma unroll
		for (int j = 0; j < kPerThread; ++j)
			v[j] = __ldg(table + (p[j] >> 5));
#pragma unroll
		for (int j = 0; j < kPerThread; ++j) {
			const uint32_t bits = __ballot_sync(0xffffffffu, (v[j] >> (p[j] & 31u)) & 1u);
			const uint64_t word = (base >> 5) + j;
			if (lane == 0 && word * 32 < n)
				out[word] = bits;
		}
	}
}

/* Gathers at positions generated in the kernel (no position stream). */
__global__ void __launch_bounds__(256) gather_hash_kernel(uint64_t n, uint64_t bits,
		uint64_t seed, const uint32_t *__restrict__ table, uint32_t *__restrict__ out,
		unsigned long long *next)
{
	const int lane = threadIdx.x & 31;
	const uint64_t chunk = 32ull * kPerThread;
	for (uint64_t t = next_take(next, lane); t * kTake * chunk < n; t = next_take(next, lane))
	for (uint64_t w = t * kTake; w < (t + 1) * kTake && w * chunk < n; ++w) {
		const uint64_t base = w * chunk;
		uint64_t p[kPerThread];
		uint32_t v[kPerThread];
#pragma unroll
		for (int j = 0; j < kPerThread; ++j)
			p[j] = mix64d(seed ^ (base + (uint64_t)j * 32 + lane)) % bits;
#pragma unroll
		for (int j = 0; j < kPerThread; ++j)
			v[j] = __ldg(table + (p[j] >> 5));
		uint32_t acc = 0;
#pragma unroll
		for (int j = 0; j < kPerThread; ++j)
			acc ^= __ballot_sync(0xffffffffu, (v[j] >> (p[j] & 31u)) & 1u);
		if (lane == 0)
			out[w] = acc;
	}
}

} // namespace
} // namespace bbt

using namespace bbt;

extern "C" int bbt_measure_gather(int device, uint64_t table_bytes, uint64_t n_gathers,
		int position_stream, int reps, double *gathers_per_s)
{
	if (!gathers_per_s || table_bytes < 4096 || table_bytes > (1ull << 37) || n_gathers == 0 ||
			reps < 1)
		return fail(nullptr, BBT_ERR_ARG, "bbt_measure_gather: bad arguments");
	if (position_stream && table_bytes > (1ull << 29))
		return fail(nullptr, BBT_ERR_ARG, "bbt_measure_gather: streamed positions are 32-bit "
				"bit offsets (table of at most 512 MB)");
	cudaError_t e = cudaSetDevice(device);
	if (e != cudaSuccess)
		return cuda_fail(nullptr, e, "cudaSetDevice");
	int sms = 0;
	cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
	const uint64_t entries = table_bytes / 4;
	const uint64_t bits = entries * 32;
	uint32_t *table = nullptr, *pos = nullptr, *out = nullptr;
	unsigned long long *next = nullptr;
	cudaEvent_t e0 = nullptr, e1 = nullptr;
	std::vector<float> ms;
	int rc = BBT_OK;
#define GR_TRY(x) do { if ((e = (x)) != cudaSuccess) { rc = cuda_fail(nullptr, e, #x); goto done; } } while (0)
	GR_TRY(cudaMalloc(&table, entries * 4));
	GR_TRY(cudaMemset(table, 0x5a, entries * 4));
	GR_TRY(cudaMalloc(&out, (n_gathers / 32 + 1) * 4));
	GR_TRY(cudaMalloc(&next, sizeof(unsigned long long)));
	if (position_stream) {
		GR_TRY(cudaMalloc(&pos, n_gathers * 4));
		positions_kernel<<<sms * 8, 256>>>(pos, n_gathers, bits, 12345);
		GR_TRY(cudaGetLastError());
	}
	GR_TRY(cudaEventCreate(&e0));
	GR_TRY(cudaEventCreate(&e1));
	for (int r = 0; r < reps + 1; ++r) {
		GR_TRY(cudaMemset(next, 0, sizeof(unsigned long long)));
		GR_TRY(cudaEventRecord(e0));
		if (position_stream)
			gather_stream_kernel<<<sms * 8, 256>>>(pos, n_gathers, table, out, next);
		else
			gather_hash_kernel<<<sms * 8, 256>>>(n_gathers, bits, 777 + r, table, out, next);
		GR_TRY(cudaGetLastError());
		GR_TRY(cudaEventRecord(e1));
		GR_TRY(cudaEventSynchronize(e1));
		float t = 0;
		GR_TRY(cudaEventElapsedTime(&t, e0, e1));
		if (r)  /* the first launch warms the table into L2 */
			ms.push_back(t);
	}
	std::sort(ms.begin(), ms.end());
	*gathers_per_s = (double)n_gathers / (ms[ms.size() / 2] * 1e-3);
done:
#undef GR_TRY
	if (e0)
		cudaEventDestroy(e0);
	if (e1)
		cudaEventDestroy(e1);
	cudaFree(table);
	cudaFree(pos);
	cudaFree(out);
	cudaFree(next);
	return rc;
}
