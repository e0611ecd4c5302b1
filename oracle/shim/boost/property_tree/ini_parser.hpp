/* Shim: boost::property_tree::ini_parser::read_ini for "[section]" and
 * "key=value" lines; ';' and '#' start comments; keys and values are trimmed. */
#ifndef BBT_SHIM_INI_PARSER_HPP
#define BBT_SHIM_INI_PARSER_HPP
#include "ptree.hpp"
#include <fstream>
namespace boost {
namespace property_tree {
namespace ini_parser {
inline std::string ini_trim(const std::string &s) {
	size_t b = s.find_first_not_of(" \t\r\n");
	if (b == std::string::npos)
		return "";
	size_t e = s.find_last_not_of(" \t\r\n");
	return s.substr(b, e - b + 1);
}
inline void read_ini(const std::string &file, ptree &pt) {
	std::ifstream in(file.c_str());
	if (!in)
		throw std::runtime_error(file + ": cannot open file");
	std::string line, section;
	while (std::getline(in, line)) {
		line = ini_trim(line);
		if (line.empty() || line[0] == ';' || line[0] == '#')
			continue;
		if (line[0] == '[') {
			section = ini_trim(line.substr(1, line.find(']') - 1));
			continue;
		}
		size_t eq = line.find('=');
		if (eq == std::string::npos)
			throw std::runtime_error(file + ": '=' character not found in line");
		std::string key = ini_trim(line.substr(0, eq));
		std::string val = ini_trim(line.substr(eq + 1));
		pt.put(section.empty() ? key : section + "." + key, val);
	}
}
}
}
}
#endif
