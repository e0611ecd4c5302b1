/* Shim: btl_bloomfilter/BloomFilter.hpp restated over the C oracle
 * (oracle/bbt_oracle.c).  The upstream submodule is absent from the
 * reference tree; this class offers the members the reference calls
 * (Common/SeqEval.h, BioBloomCategorizer/BioBloomClassifier.cpp:962,
 * BioBloomMaker/BloomFilterGenerator.*, Tests/BloomFilterTests.cpp). */
#ifndef BBT_SHIM_BLOOMFILTER_HPP
#define BBT_SHIM_BLOOMFILTER_HPP
#include "bbt_oracle.h"
#include <cmath>
#include <cstdlib>
#include <iostream>
#include <string>

/* The reference's headers that include this one (Common/SDust.hpp via
 * Common/SeqEval.h) name std::string unqualified, relying on the submodule's
 * headers to bring namespace std into scope. */
using namespace std;

class BloomFilter {
public:
	BloomFilter() { m_bf.bits = 0; m_bf.m = 0; }
	BloomFilter(size_t size, unsigned hashNum, unsigned kmerSize) {
		if (oracle_bf_create(&m_bf, size, hashNum, kmerSize)) {
			std::cerr << "BloomFilter: allocation failed" << std::endl;
			exit(1);
		}
	}
	explicit BloomFilter(const std::string &path) {
		int rc = oracle_bf_load(&m_bf, path.c_str());
		if (rc) {
			std::cerr << "BloomFilter: cannot load " << path << " (" << rc << ")" << std::endl;
			exit(1);
		}
		m_fpr = getFPR();
	}
	~BloomFilter() { oracle_bf_free(&m_bf); }
	BloomFilter(const BloomFilter &) = delete;
	BloomFilter &operator=(const BloomFilter &) = delete;

	void insert(const size_t *hv) { oracle_bf_insert(&m_bf, (const uint64_t *)hv); }
	bool insertAndCheck(const size_t *hv) {
		return oracle_bf_insert_check(&m_bf, (const uint64_t *)hv) != 0;
	}
	bool contains(const size_t *hv) const {
		return oracle_bf_contains(&m_bf, (const uint64_t *)hv, 0) != 0;
	}
	unsigned getKmerSize() const { return m_bf.k; }
	unsigned getHashNum() const { return m_bf.h; }
	size_t getFilterSize() const { return m_bf.m; }
	size_t getPop() const {
		size_t pop = 0;
		for (size_t i = 0; i < m_bf.m / 8; ++i)
			pop += (size_t)__builtin_popcount(m_bf.bits[i]);
		return pop;
	}
	/* Occupancy raised to the number of hash functions. */
	double getFPR() const {
		return std::pow(double(getPop()) / double(m_bf.m), double(m_bf.h));
	}
	/* the FPR of a filter loaded from a file, computed once at load (SeqEval
	 * calls this for every read it evaluates under BINOMIAL scoring, from
	 * several threads) */
	double getFPRPrecompute() const { return m_fpr >= 0 ? m_fpr : getFPR(); }
	void storeFilter(const std::string &path) const {
		if (oracle_bf_store(&m_bf, path.c_str())) {
			std::cerr << "BloomFilter: cannot write " << path << std::endl;
			exit(1);
		}
	}
	void setEntries(size_t nEntry, size_t tEntry, double dfpr) {
		m_bf.n_entry = nEntry;
		m_bf.t_entry = tEntry;
		m_bf.dfpr = dfpr;
	}
	const oracle_bf &raw() const { return m_bf; }
private:
	oracle_bf m_bf;
	double m_fpr = -1.0; /* FPR computed at load (getFPRPrecompute) */
};
#endif
