/*
 * dust_model.cpp -- the SDUST scan of the masking kernel (dust_core.cuh),
 * compiled for the host so that tests can compare it with the oracle's
 * restatement of Common/sdust.c.  TEST INFRASTRUCTURE ONLY.
 */
#include <stdint.h>

#include <vector>

#include "dust_core.cuh"

extern "C" int model_sdust(const char *seq, uint64_t len, int T, int W, int pcap, uint64_t *out,
		int cap)
{
	std::vector<bbt::DustPerfect> perf((size_t)pcap);
	std::vector<uint8_t> ring((size_t)W);
	std::vector<uint64_t> iv;
	const uint8_t *bases = (const uint8_t *)seq;
	const bool ok = bbt::dust_scan([&](int i) { return bases[i]; }, len, T, W, perf.data(), pcap,
			ring.data(), [&](int a, int b) {
				/* an extension of the last interval starts at its finish */
				if (!iv.empty() && (uint32_t)iv.back() == (uint32_t)a)
					iv.back() = (iv.back() & ~0xffffffffull) | (uint32_t)b;
				else
					iv.push_back((uint64_t)(uint32_t)a << 32 | (uint32_t)b);
			});
	if (!ok)
		return -1;
	for (size_t i = 0; i < iv.size() && (int)i < cap; ++i)
		out[i] = iv[i];
	return (int)iv.size();
}
