/*
 * fastx.hpp -- FASTA/FASTQ reader with the record semantics of kseq_read
 * (Common/kseq.h:177-219), over zlib (plain or gzip input).
 *
 * A record starts at '>' or '@'.  The name runs to the first whitespace byte;
 * the rest of that line is the comment.  Sequence lines are concatenated up to
 * the next line starting with '>', '@' or '+' (empty lines are skipped, one
 * trailing '\r' per line is dropped).  After '+', quality lines are read until
 * the quality is as long as the sequence.  read() returns the sequence length,
 * -1 at end of input, -2 for a truncated / mismatched quality, -3 on a stream
 * error, as kseq_read does.
 */
#ifndef BBT_FASTX_HPP
#define BBT_FASTX_HPP

#include <zlib.h>

#include <string>
#include <vector>

namespace bbt {

class FastxReader {
public:
	explicit FastxReader(const std::string &path);
	~FastxReader();
	bool ok() const { return fp_ != nullptr; }
	/* Appends the sequence to seq (so batches can be built in place). */
	long read(std::string &name, std::string &comment, std::vector<char> &seq,
			std::string &qual);

private:
	int getc_();
	bool fill_();
	gzFile fp_ = nullptr;
	std::vector<unsigned char> buf_;
	size_t begin_ = 0, end_ = 0;
	bool eof_ = false, err_ = false;
	int last_char_ = 0;
};

} // namespace bbt

#endif
