/*
 * formats.hpp -- the on-disk formats of the classification path.
 *
 *  .bf   Bloom filter: a text header of "key = value" lines opened by
 *        "[BTLBloomFilter]" and closed by "[HeaderEnd]" (each line ends in
 *        '\n'), followed by the m/8 payload bytes; bit j is byte j/8,
 *        bit j%8 (least significant first).  Keys: Format, BloomFilterSize (m,
 *        a multiple of 64), HashNum, KmerSize, dFPR, nEntry, tEntry.  The
 *        upstream btl_bloomfilter header layout is not available to this
 *        project; this layout carries the same fields.
 *  .txt  BloomFilterInfo INI sidecar (Common/BloomFilterInfo.cpp:81-116):
 *        [user_input_options] filter_id, kmer_size,
 *        desired_false_positve_rate, number_of_hash_functions,
 *        expected_num_entries, sequence_sources; [runtime_options] size,
 *        num_entries, approximate_false_positive_rate, redundant_sequences,
 *        redundant_fpr.
 */
#ifndef BBT_FORMATS_HPP
#define BBT_FORMATS_HPP

#include <cstdint>
#include <cstdio>
#include <map>
#include <string>

namespace bbt {

struct BfHeader {
	uint64_t m = 0;
	unsigned h = 0;
	unsigned k = 0;
	double dfpr = 0;
	uint64_t n_entry = 0;
	uint64_t t_entry = 0;
	long payload_offset = 0;  /* byte offset of the payload in the file */
};

/* Parse the header of an open .bf file; leaves the stream at the payload.
 * Returns 0, or an error message. */
const char *read_bf_header(FILE *f, BfHeader &h);
int write_bf_header(FILE *f, const BfHeader &h);

/* key -> value of an INI file ("section.key"); returns false if unreadable. */
bool read_ini(const std::string &path, std::map<std::string, std::string> &kv);

struct InfoFile {
	std::string filter_id;
	unsigned kmer_size = 0;
	double fpr = 0;
	unsigned hash_num = 0;
	uint64_t expected = 0;
	std::string sources;
	uint64_t size = 0;
	uint64_t num_entries = 0;
	double approx_fpr = 0;
	uint64_t redundant = 0;
	double redundant_fpr = 0;
};
bool write_info(const std::string &path, const InfoFile &info);

/* Sizing from Common/BloomFilterInfo.h:57-76 and Common/BloomFilterInfo.cpp:172-178. */
uint64_t optimal_size(uint64_t entries, double fpr, unsigned h);
unsigned optimal_hash_num(double fpr);
double approx_fpr(uint64_t size, uint64_t entries, unsigned h);

/* "<path without the trailing 'bf'>txt", as BioBloomClassifier.cpp:957 forms it. */
std::string info_path_for(const std::string &bf_path);

} // namespace bbt

#endif
