/*
 * dust.cu -- SDUST low-complexity masking on the GPU (-D, -T, -W).
 *
 * With opt::dust the reference builds an SDust object per evaluated read
 * (Common/SDust.hpp), which runs sdust (Common/sdust.c: the symmetric DUST
 * algorithm of Morgulis et al., J Comput Biol 2006, as minimap2 implements
 * it) over the read, and SeqEval then treats every frame whose start lies in
 * a masked interval as a miss without probing the filter
 * (Common/SeqEval.h:53,78,132,...).
 *
 * Here one thread runs the same sequential algorithm per read (the algorithm
 * is a scan with a sliding window and a list of pending "perfect intervals";
 * reads are independent, so the batch is the parallel dimension) and sets,
 * for every masked base position, a bit in a per-mate bit array indexed like
 * the batch's bases.  The classification kernels read that bit for each
 * frame they evaluate.
 *
 * The list of pending perfect intervals is short for ordinary sequence but
 * grows with the square of the window on long homopolymers and short tandem
 * repeats (thousands of entries for W = 64).  Pass 1 keeps it in a small
 * per-thread array; a read that outgrows it is queued and recomputed from
 * the start by pass 2, whose threads each own a slice of global memory large
 * enough for any read (W^2 + 2W + 64 entries: the list, plus the entries one
 * window step adds before they are merged in).  A read outgrowing even that is
 * reported through an error counter and fails the call.
 *
 * The algorithm, in the reference's terms: words are the triplets of
 * consecutive A/C/G/T bases (either case); the window holds the last W - 2
 * triplets; a set of triplets scores sum over kinds of c(c-1)/2.  cw / rw
 * count the whole window; cv / rv count its longest suffix (L triplets) in
 * which no kind occurs more than 2T/10 times.  When 10 rw > L T the window
 * may hold perfect intervals (suffixes with 10 r > T l whose score is at
 * least that of every perfect interval starting inside them); they are kept
 * by descending start.  One whose start falls out of the window is saved as
 * masked, merged with the previous masked interval when they touch.  A base
 * that is not A/C/G/T, and the end of the read, flush the pending intervals
 * but leave the window as it is.
 */
#include "dust.cuh"
#include "dust_core.cuh"

namespace bbt {

namespace {

constexpr int kLocalPerfect = 160;  /* pass-1 capacity of the perfect list (and of the
                                       entries a window step adds before they merge) */

/* Set bits [a, b) of the read's mask (positions clamped to the read). */
__device__ void mask_range(uint32_t *mask, uint64_t base, int64_t a, int64_t b, uint64_t len)
{
	if (a < 0)
		a = 0;
	if (b > (int64_t)len)
		b = (int64_t)len;
	for (int64_t p = a; p < b;) {
		const uint64_t g = base + (uint64_t)p;
		const uint32_t bit = (uint32_t)(g & 31u);
		const int64_t n = min((int64_t)(32u - bit), b - p);
		const uint32_t bits = (n == 32 ? 0xffffffffu : ((1u << n) - 1u)) << bit;
		atomicOr(mask + (g >> 5), bits);
		p += n;
	}
}

/* Bases in order, eight at a time: one aligned 8-byte load per 8 bases
 * (each thread scans its own read, so byte loads would not coalesce). */
struct BaseStream {
	const uint8_t *p;
	uint64_t word = 0;
	int64_t word_at = -1; /* address / 8 of the word held */
	__device__ __forceinline__ uint8_t operator()(int i)
	{
		const uintptr_t a = (uintptr_t)(p + i);
		const int64_t w = (int64_t)(a >> 3);
		if (w != word_at) {
			word = __ldg(reinterpret_cast<const unsigned long long *>(a & ~(uintptr_t)7));
			word_at = w;
		}
		return (uint8_t)(word >> ((a & 7u) * 8u));
	}
};

__device__ bool dust_read(const uint8_t *__restrict__ seq, uint64_t len, int T, int W,
		DustPerfect *perf, int pcap, uint8_t *ring, uint32_t *mask, uint64_t mask_base)
{
	BaseStream bs{seq};
	return dust_scan(bs, len, T, W, perf, pcap, ring, [&](int a, int b) {
		mask_range(mask, mask_base, a, b, len);
	});
}

__device__ __forceinline__ void read_at(const DustArgs &a, uint64_t r, const uint8_t *&s,
		uint64_t &len, uint32_t *&mask, uint64_t &base)
{
	const uint32_t mate = r >= a.n ? 1u : 0u;
	const uint64_t i = r - (mate ? a.n : 0);
	const uint64_t *off = a.off[mate];
	base = off[i] - a.off_base[mate];
	len = off[i + 1] - off[i];
	s = a.seq[mate] + base;
	mask = a.mask[mate];
}

__global__ void __launch_bounds__(128) dust_pass1_kernel(DustArgs a)
{
	DustPerfect perf[kLocalPerfect];
	uint8_t ring[kDustMaxWindow];
	const uint64_t total = a.n * a.mates;
	for (uint64_t r = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; r < total;
			r += (uint64_t)gridDim.x * blockDim.x) {
		const uint8_t *s;
		uint64_t len, base;
		uint32_t *mask;
		read_at(a, r, s, len, mask, base);
		if (!dust_read(s, len, a.T, a.W, perf, kLocalPerfect, ring, mask, base)) {
			const unsigned long long q = atomicAdd(a.redo_count, 1ull);
			a.redo[q] = r;
		}
	}
}

__global__ void __launch_bounds__(128) dust_pass2_kernel(DustArgs a)
{
	uint8_t ring[kDustMaxWindow];
	const uint64_t redo_n = *(volatile unsigned long long *)a.redo_count;
	const uint64_t tid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
	DustPerfect *perf = reinterpret_cast<DustPerfect *>(a.scratch) + tid * a.scratch_per_thread;
	for (uint64_t q = tid; q < redo_n; q += (uint64_t)gridDim.x * blockDim.x) {
		const uint8_t *s;
		uint64_t len, base;
		uint32_t *mask;
		read_at(a, a.redo[q], s, len, mask, base);
		if (!dust_read(s, len, a.T, a.W, perf, (int)a.scratch_per_thread, ring, mask, base))
			atomicAdd(a.failed, 1ull);
	}
}

} // namespace

size_t dust_perfect_bytes()
{
	return sizeof(DustPerfect);
}

cudaError_t launch_dust_pass1(const DustArgs &a, int num_sms, cudaStream_t s)
{
	const uint64_t total = a.n * a.mates;
	if (total == 0)
		return cudaSuccess;
	const uint64_t need = (total + 127) / 128;
	const uint64_t cap = (uint64_t)num_sms * 16;
	dust_pass1_kernel<<<(unsigned)(need < cap ? need : cap), 128, 0, s>>>(a);
	return cudaGetLastError();
}

cudaError_t launch_dust_pass2(const DustArgs &a, uint32_t threads, cudaStream_t s)
{
	if (a.n * a.mates == 0)
		return cudaSuccess;
	const uint32_t blocks = (threads + 31) / 32;
	dust_pass2_kernel<<<blocks, 32, 0, s>>>(a);
	return cudaGetLastError();
}

} // namespace bbt
