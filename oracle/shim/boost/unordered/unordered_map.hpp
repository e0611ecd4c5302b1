/* Shim: boost::unordered_map is std::unordered_map for the oracle build. */
#ifndef BBT_SHIM_BOOST_UNORDERED_MAP_HPP
#define BBT_SHIM_BOOST_UNORDERED_MAP_HPP
#include <cmath> /* Boost headers pull this in transitively; BloomFilterInfo.h relies on it */
#include <unordered_map>
namespace boost { using std::unordered_map; }
#endif
