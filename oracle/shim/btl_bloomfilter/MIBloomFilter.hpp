/* Shim: btl_bloomfilter/MIBloomFilter.hpp restated over the C oracle
 * (oracle/mibf_oracle.c): the members the reference calls
 * (BioBloomCategorizer/MIBFClassifier.hpp:49-94, 773-834,
 * Tests/ntHashTests.cpp:27). */
#ifndef BBT_SHIM_MIBLOOMFILTER_HPP
#define BBT_SHIM_MIBLOOMFILTER_HPP
#include "mibf_oracle.h"
#include <omp.h>
#include <cstdlib>
#include <fstream>   /* the reference's MIBFClassifier.hpp relies on these */
#include <iostream>
#include <sstream>
#include <string>
#include <vector>

using namespace std;

template <typename T> class MIBloomFilter {
public:
	explicit MIBloomFilter(const std::string &path) {
		int rc = oracle_mibf_load(&m_f, path.c_str());
		if (rc) {
			std::cerr << "MIBloomFilter: cannot load " << path << " (" << rc << ")" << std::endl;
			exit(1);
		}
		std::vector<std::string> s;
		for (unsigned i = 0; i < m_f.nseeds; ++i)
			s.push_back(m_f.seeds[i]);
		m_seedValues = parseSeedString(s);
	}
	/* an empty filter over a finished bit vector (MIBFConstructSupport::
	 * getEmptyMIBF): takes the arrays, IDs all EMPTY */
	MIBloomFilter(const oracle_mibf &f) : m_f(f) {
		std::vector<std::string> s;
		for (unsigned i = 0; i < m_f.nseeds; ++i)
			s.push_back(m_f.seeds[i]);
		m_seedValues = parseSeedString(s);
	}
	~MIBloomFilter() { oracle_mibf_free(&m_f); }
	MIBloomFilter(const MIBloomFilter &) = delete;
	MIBloomFilter &operator=(const MIBloomFilter &) = delete;
	MIBloomFilter(MIBloomFilter &&o) noexcept : m_f(o.m_f), m_seedValues(o.m_seedValues) {
		o.m_f.bv = 0; o.m_f.rank_word = 0; o.m_f.ids = 0;
	}
	unsigned getHashNum() const { return m_f.h; }
	unsigned getKmerSize() const { return m_f.k; }
	const std::vector<std::vector<unsigned> > &getSeedValues() const { return m_seedValues; }
	double calcFrameProbs(std::vector<double> &perFrameProb, unsigned allowedMiss) const {
		return oracle_mibf_frame_probs(&m_f, perFrameProb.data(),
				(unsigned)perFrameProb.size(), allowedMiss);
	}
	/* don't-care ('0') positions of each seed string */
	static std::vector<std::vector<unsigned> > parseSeedString(const std::vector<std::string> &ss) {
		std::vector<std::vector<unsigned> > out;
		for (size_t i = 0; i < ss.size(); ++i) {
			std::vector<unsigned> z;
			for (unsigned j = 0; j < ss[i].size(); ++j)
				if (ss[i][j] != '1')
					z.push_back(j);
			out.push_back(z);
		}
		return out;
	}
	size_t getPop() const { return m_f.pop; }
	size_t getPopSaturated() const {
		size_t n = 0;
		for (uint64_t i = 0; i < m_f.pop; ++i)
			n += (m_f.ids[i] & ORACLE_MIBF_SAT) ? 1 : 0;
		return n;
	}
	/* slots owned per ID (saturated or not) */
	void getIDCounts(std::vector<size_t> &counts) const {
		for (uint64_t i = 0; i < m_f.pop; ++i) {
			const unsigned id = m_f.ids[i] & 0x7FFFu;
			if (id < counts.size())
				++counts[id];
		}
	}
	/* <prefix>.bf + <prefix>.sdsl from the path of the .bf */
	void store(const std::string &bf_path) const {
		std::string prefix = bf_path;
		if (prefix.size() >= 3 && prefix.compare(prefix.size() - 3, 3, ".bf") == 0)
			prefix.resize(prefix.size() - 3);
		if (oracle_mibf_store(&m_f, prefix.c_str())) {
			std::cerr << "MIBloomFilter: cannot store " << bf_path << std::endl;
			exit(1);
		}
	}
	oracle_mibf &rawMutable() { return m_f; }
	size_t size() const { return m_f.m; }
	const oracle_mibf &raw() const { return m_f; }
private:
	oracle_mibf m_f;
	std::vector<std::vector<unsigned> > m_seedValues;
};
#endif
