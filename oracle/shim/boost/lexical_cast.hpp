/* Shim: boost::lexical_cast via a stringstream round trip (included, unused,
 * by BioBloomMaker/BloomFilterGenerator.cpp). */
#ifndef BBT_SHIM_BOOST_LEXICAL_CAST_HPP
#define BBT_SHIM_BOOST_LEXICAL_CAST_HPP
#include <sstream>
namespace boost {
template <class T, class S> T lexical_cast(const S &s) {
	std::stringstream ss;
	ss << s;
	T t;
	ss >> t;
	return t;
}
}
#endif
