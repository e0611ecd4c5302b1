/* Shim: btl_bloomfilter/MIBFConstructSupport.hpp (absent from the reference
 * tree) restated over the C oracle (oracle/mibf_oracle.c): the members that
 * MIBFGen::generate and generateBV call (BioBloomMaker/MIBFGen.hpp:131-415).
 * TEST INFRASTRUCTURE ONLY.
 *
 * The passes are the oracle's (mibf_oracle.h): the bit vector of every frame's
 * h values (m = ceil(n * h / -ln(1 - occupancy)) rounded up to 64 bits), then
 * slot owners by the largest (priority(slot, id) << 16 | id), then the
 * saturation bit on all h slots of every (sequence, frame) whose ID owns none
 * of them.  The reference calls them from several OpenMP threads; every update
 * here is an atomic OR or MAX, so the result does not depend on the order. */
#ifndef BBT_SHIM_MIBFCONSTRUCTSUPPORT_HPP
#define BBT_SHIM_MIBFCONSTRUCTSUPPORT_HPP
#include "MIBloomFilter.hpp"
#include "mibf_oracle.h"
#include <cmath>
#include <cstdint>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

template <typename ID, typename H> class MIBFConstructSupport {
public:
	MIBFConstructSupport(size_t expectedEntries, unsigned k, unsigned hashNum, double occupancy,
			const std::vector<std::string> &seeds)
		: m_k(k), m_h(seeds.empty() ? hashNum : (unsigned)seeds.size()), m_seeds(seeds)
	{
		double mb = std::ceil((double)expectedEntries * m_h / -std::log(1.0 - occupancy));
		uint64_t m = (uint64_t)mb;
		m += (64 - m % 64) % 64;
		m_m = m ? m : 64;
		m_bv = (uint64_t *)calloc(m_m / 64, sizeof(uint64_t));
	}
	~MIBFConstructSupport() { free(m_best); }
	size_t getFilterSize() const { return m_m; }

	/* pass 1: set the bits of every frame; returns the frames whose bits
	 * were all set already */
	size_t insertBVColli(H &itr) {
		size_t colli = 0;
		for (; itr != H::end(); ++itr) {
			bool all = true;
			for (unsigned v = 0; v < m_h; ++v) {
				const uint64_t p = (uint64_t)(*itr)[v] % m_m;
				const uint64_t bit = 1ull << (p & 63);
				if (!(__atomic_fetch_or(m_bv + (p >> 6), bit, __ATOMIC_RELAXED) & bit))
					all = false;
			}
			colli += all ? 1 : 0;
		}
		return colli;
	}

	/* rank support and an empty ID array over the finished bit vector */
	MIBloomFilter<ID> *getEmptyMIBF() {
		oracle_mibf f;
		memset(&f, 0, sizeof f);
		f.m = m_m;
		f.h = m_h;
		f.k = m_k;
		f.nseeds = (unsigned)m_seeds.size();
		for (size_t i = 0; i < m_seeds.size() && i < ORACLE_MIBF_MAX_SEEDS; ++i)
			strncpy(f.seeds[i], m_seeds[i].c_str(), 255);
		f.bv = m_bv;
		const uint64_t words = m_m / 64;
		f.rank_word = (uint64_t *)malloc((words + 1) * sizeof(uint64_t));
		uint64_t acc = 0;
		for (uint64_t w = 0; w < words; ++w) {
			f.rank_word[w] = acc;
			acc += (uint64_t)__builtin_popcountll(m_bv[w]);
		}
		f.rank_word[words] = acc;
		f.pop = acc;
		f.ids = (uint16_t *)calloc(acc ? acc : 1, sizeof(uint16_t));
		m_best = (uint32_t *)calloc(acc ? acc : 1, sizeof(uint32_t));
		m_bv = nullptr; /* the filter owns the arrays now */
		MIBloomFilter<ID> *mi = new MIBloomFilter<ID>(f);
		m_f = &mi->rawMutable();
		return mi;
	}

	/* pass 2: offer `id` to the slots of every frame */
	void insertMIBF(MIBloomFilter<ID> &, H &itr, ID id) {
		for (; itr != H::end(); ++itr)
			for (unsigned v = 0; v < m_h; ++v) {
				const uint64_t slot = oracle_mibf_rank(m_f, (uint64_t)(*itr)[v] % m_m);
				const uint32_t cand = ((uint32_t)priority(slot, id) << 16) | (uint32_t)id;
				uint32_t cur = __atomic_load_n(m_best + slot, __ATOMIC_RELAXED);
				while (cand > cur && !__atomic_compare_exchange_n(m_best + slot, &cur, cand,
						true, __ATOMIC_RELAXED, __ATOMIC_RELAXED)) {
				}
			}
	}

	/* pass 3: saturation (the owners of pass 2 are written in first) */
	void insertSaturation(MIBloomFilter<ID> &, H &itr, ID id) {
		std::call_once(m_owners, [this]() {
			for (uint64_t s = 0; s < m_f->pop; ++s)
				m_f->ids[s] = (uint16_t)(m_best[s] & 0xFFFF);
		});
		std::vector<uint64_t> slots(m_h);
		for (; itr != H::end(); ++itr) {
			bool owned = false;
			for (unsigned v = 0; v < m_h; ++v) {
				slots[v] = oracle_mibf_rank(m_f, (uint64_t)(*itr)[v] % m_m);
				const uint16_t e = __atomic_load_n(m_f->ids + slots[v], __ATOMIC_RELAXED);
				if ((e & 0x7FFF) == (uint16_t)id)
					owned = true;
			}
			if (!owned)
				for (unsigned v = 0; v < m_h; ++v)
					__atomic_fetch_or(m_f->ids + slots[v], (uint16_t)ORACLE_MIBF_SAT,
							__ATOMIC_RELAXED);
		}
	}

private:
	static uint16_t priority(uint64_t slot, unsigned id) {
		uint64_t z = slot ^ ((uint64_t)id * 0x9e3779b97f4a7c15ULL);
		z += 0x9e3779b97f4a7c15ULL;
		z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
		z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
		return (uint16_t)((z ^ (z >> 31)) >> 48);
	}
	unsigned m_k, m_h;
	std::vector<std::string> m_seeds;
	uint64_t m_m = 0;
	uint64_t *m_bv = nullptr;
	uint32_t *m_best = nullptr;
	oracle_mibf *m_f = nullptr;
	std::once_flag m_owners;
};
#endif
