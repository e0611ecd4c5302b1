/*
 * formats.cpp -- .bf / .txt reading and writing (layouts in formats.hpp).
 */
#include "formats.hpp"

#include <cmath>
#include <cstring>
#include <fstream>
#include <sstream>

namespace bbt {

const char *read_bf_header(FILE *f, BfHeader &h)
{
	char line[512];
	if (!fgets(line, sizeof line, f) || strcmp(line, "[BTLBloomFilter]\n") != 0)
		return "not a Bloom filter file (missing [BTLBloomFilter] header)";
	bool end = false;
	while (fgets(line, sizeof line, f)) {
		if (!strcmp(line, "[HeaderEnd]\n")) {
			end = true;
			break;
		}
		char key[64];
		char val[256];
		if (sscanf(line, "%63s = %255s", key, val) != 2)
			return "malformed Bloom filter header line";
		if (!strcmp(key, "BloomFilterSize"))
			h.m = strtoull(val, nullptr, 10);
		else if (!strcmp(key, "HashNum"))
			h.h = (unsigned)strtoul(val, nullptr, 10);
		else if (!strcmp(key, "KmerSize"))
			h.k = (unsigned)strtoul(val, nullptr, 10);
		else if (!strcmp(key, "dFPR"))
			h.dfpr = strtod(val, nullptr);
		else if (!strcmp(key, "nEntry"))
			h.n_entry = strtoull(val, nullptr, 10);
		else if (!strcmp(key, "tEntry"))
			h.t_entry = strtoull(val, nullptr, 10);
	}
	if (!end)
		return "truncated Bloom filter header";
	if (h.m == 0 || h.m % 64)
		return "Bloom filter size is not a positive multiple of 64 bits";
	if (h.h == 0 || h.h > 64)
		return "Bloom filter hash count out of range (1..64)";
	if (h.k == 0 || h.k > 255)
		return "Bloom filter k-mer size out of range (1..255)";
	h.payload_offset = ftell(f);
	return nullptr;
}

int write_bf_header(FILE *f, const BfHeader &h)
{
	return fprintf(f, "[BTLBloomFilter]\nFormat = 1\nBloomFilterSize = %llu\nHashNum = %u\n"
			"KmerSize = %u\ndFPR = %.17g\nnEntry = %llu\ntEntry = %llu\n[HeaderEnd]\n",
			(unsigned long long)h.m, h.h, h.k, h.dfpr, (unsigned long long)h.n_entry,
			(unsigned long long)h.t_entry) < 0 ? -1 : 0;
}

static std::string trim(const std::string &s)
{
	size_t b = s.find_first_not_of(" \t\r\n");
	if (b == std::string::npos)
		return "";
	size_t e = s.find_last_not_of(" \t\r\n");
	return s.substr(b, e - b + 1);
}

bool read_ini(const std::string &path, std::map<std::string, std::string> &kv)
{
	std::ifstream in(path);
	if (!in)
		return false;
	std::string line, section;
	while (std::getline(in, line)) {
		line = trim(line);
		if (line.empty() || line[0] == ';' || line[0] == '#')
			continue;
		if (line[0] == '[') {
			section = trim(line.substr(1, line.find(']') - 1));
			continue;
		}
		size_t eq = line.find('=');
		if (eq == std::string::npos)
			continue;
		std::string key = trim(line.substr(0, eq));
		kv[section.empty() ? key : section + "." + key] = trim(line.substr(eq + 1));
	}
	return true;
}

/* Doubles are written with the default ostream format, as the reference's
 * printInfoFile does. */
bool write_info(const std::string &path, const InfoFile &i)
{
	std::ofstream out(path);
	if (!out)
		return false;
	out << "[user_input_options]\nfilter_id=" << i.filter_id << "\nkmer_size=" << i.kmer_size
	    << "\ndesired_false_positve_rate=" << i.fpr << "\nnumber_of_hash_functions="
	    << i.hash_num << "\nexpected_num_entries=" << i.expected << "\nsequence_sources="
	    << i.sources << " \n\n[runtime_options]\nsize=" << i.size << "\nnum_entries="
	    << i.num_entries << "\napproximate_false_positive_rate=" << i.approx_fpr
	    << "\nredundant_sequences=" << i.redundant << "\nredundant_fpr=" << i.redundant_fpr
	    << "\n";
	return (bool)out;
}

uint64_t optimal_size(uint64_t entries, double fpr, unsigned h)
{
	uint64_t v = (uint64_t)(-(double)entries * (double)h
			/ std::log(1.0 - std::pow(fpr, (double)(1 / ((double)h)))));
	return v + (64 - v % 64);
}

unsigned optimal_hash_num(double fpr)
{
	return (unsigned)(-std::log(fpr) / std::log(2));
}

double approx_fpr(uint64_t size, uint64_t entries, unsigned h)
{
	return std::pow(1.0 - std::pow(1.0 - 1.0 / (double)size, (double)entries * h), (double)h);
}

std::string info_path_for(const std::string &bf_path)
{
	if (bf_path.size() < 2)
		return bf_path + "txt";
	return bf_path.substr(0, bf_path.size() - 2) + "txt";
}

} // namespace bbt
