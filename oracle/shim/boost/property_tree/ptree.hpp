/* Shim: the subset of boost::property_tree::ptree that
 * Common/BloomFilterInfo.cpp uses: get<T>("section.key"). */
#ifndef BBT_SHIM_PTREE_HPP
#define BBT_SHIM_PTREE_HPP
#include <map>
#include <sstream>
#include <stdexcept>
#include <string>
namespace boost {
namespace property_tree {
class ptree {
public:
	void put(const std::string &path, const std::string &value) { m_kv[path] = value; }
	template <class T> T get(const std::string &path) const {
		std::map<std::string, std::string>::const_iterator it = m_kv.find(path);
		if (it == m_kv.end())
			throw std::runtime_error("No such node (" + path + ")");
		T out;
		std::istringstream in(it->second);
		in >> out;
		if (in.fail())
			throw std::runtime_error("conversion of data to type failed (" + path + ")");
		return out;
	}
private:
	std::map<std::string, std::string> m_kv;
};
template <> inline std::string ptree::get<std::string>(const std::string &path) const {
	std::map<std::string, std::string>::const_iterator it = m_kv.find(path);
	if (it == m_kv.end())
		throw std::runtime_error("No such node (" + path + ")");
	return it->second;
}
}
}
#endif
