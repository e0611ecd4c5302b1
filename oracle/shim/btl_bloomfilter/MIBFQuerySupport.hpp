/* Shim: btl_bloomfilter/MIBFQuerySupport.hpp restated over the C oracle
 * (oracle/mibf_oracle.c): per-read ID tallies and the significance / multi-match
 * decision, with the QueryResult fields MIBFClassifier.hpp:652-736 prints. */
#ifndef BBT_SHIM_MIBFQUERYSUPPORT_HPP
#define BBT_SHIM_MIBFQUERYSUPPORT_HPP
#include "MIBloomFilter.hpp"
#include "vendor/stHashIterator.hpp"
#include "vendor/ntHashIterator.hpp"
#include "mibf_oracle.h"
#include <iostream>
#include <string>
#include <utility>
#include <vector>

template <typename T> class MIBFQuerySupport {
public:
	struct QueryResult {
		T id;
		unsigned nonSatFrameCount, solidCount, count, nonSatCount, totalNonSatCount, totalCount;
	};
	MIBFQuerySupport(const MIBloomFilter<T> &filter, const std::vector<double> &perFrameProb,
			double multiThresh, unsigned /*streakThreshold*/, unsigned allowedMiss,
			unsigned minCountNonSatCount, bool bestHitCountAgree)
		: m_filter(&filter), m_nids((unsigned)perFrameProb.size()), m_multi(multiThresh),
		  m_allowedMiss(allowedMiss), m_minNonSat(minCountNonSatCount),
		  m_agree(bestHitCountAgree), m_satCount(0) {}

	template <typename ITR>
	const std::vector<QueryResult> &query(ITR &itr, const std::vector<unsigned> &minCount) {
		return run(itr.seqData(), itr.seqLen(), 0, 0, minCount);
	}
	template <typename ITR>
	const std::vector<QueryResult> &query(ITR &itr1, ITR &itr2,
			const std::vector<unsigned> &minCount) {
		return run(itr1.seqData(), itr1.seqLen(), itr2.seqData(), itr2.seqLen(), minCount);
	}
	const std::vector<QueryResult> &emptyResult() {
		m_results.clear();
		m_satCount = 0;
		return m_results;
	}
	unsigned getSatCount() const { return m_satCount; }
	/* debug-mode helpers used by MIBFClassifier::filterDebug */
	std::vector<unsigned> getMatchSignature(const std::string &, unsigned &evaluated,
			std::vector<std::vector<std::pair<T, bool> > > &) {
		evaluated = 0;
		return std::vector<unsigned>();
	}
	void printAllCounts(const std::vector<std::string> &) {}
private:
	const std::vector<QueryResult> &run(const char *s1, size_t l1, const char *s2, size_t l2,
			const std::vector<unsigned> &minCount) {
		std::vector<uint32_t> mc(m_nids, 0);
		for (size_t i = 0; i < mc.size() && i < minCount.size(); ++i)
			mc[i] = minCount[i];
		std::vector<oracle_qres> out(m_nids ? m_nids : 1);
		uint32_t sat = 0;
		unsigned n = oracle_mibf_query(&m_filter->raw(), s1, l1, s2, l2, mc.data(), m_nids,
				m_multi, m_allowedMiss, m_minNonSat, m_agree ? 1 : 0, out.data(),
				(unsigned)out.size(), &sat, 0);
		m_satCount = sat;
		m_results.clear();
		for (unsigned i = 0; i < n; ++i) {
			QueryResult r;
			r.id = (T)out[i].id;
			r.nonSatFrameCount = out[i].nonSatFrameCount;
			r.solidCount = out[i].solidCount;
			r.count = out[i].count;
			r.nonSatCount = out[i].nonSatCount;
			r.totalNonSatCount = out[i].totalNonSatCount;
			r.totalCount = out[i].totalCount;
			m_results.push_back(r);
		}
		return m_results;
	}
	const MIBloomFilter<T> *m_filter;
	unsigned m_nids;
	double m_multi;
	unsigned m_allowedMiss, m_minNonSat;
	bool m_agree;
	unsigned m_satCount;
	std::vector<QueryResult> m_results;
};
#endif
