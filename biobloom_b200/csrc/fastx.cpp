/*
 * fastx.cpp -- FASTA/FASTQ reading and the file pipeline behind
 * bbt_filter_files / bbt_filter_pair_files.
 *
 * The pipeline replaces the OpenMP loop of BioBloomClassifier::filter /
 * filterPair (BioBloomClassifier.cpp:33-100, 217-303): a reader thread parses
 * records into one of two pinned batches while the other batch is classified
 * on the device; per-read categories come back for the optional read-status
 * file, and the summary counters stay on the device until the end, when
 * "<prefix>_summary.tsv" is written.
 */
#include "fastx.hpp"

#include <cuda_runtime.h>

#include <condition_variable>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <iostream>
#include <mutex>
#include <thread>
#include <algorithm>

#include "bbt.h"
#include "ctx.hpp"

namespace bbt {

FastxReader::FastxReader(const std::string &path) : buf_(1 << 20)
{
	fp_ = gzopen(path.c_str(), "r");
	if (fp_)
		gzbuffer(fp_, 1 << 20);
}

FastxReader::~FastxReader()
{
	if (fp_)
		gzclose(fp_);
}

bool FastxReader::fill_()
{
	if (eof_)
		return false;
	int n = gzread(fp_, buf_.data(), (unsigned)buf_.size());
	if (n < 0) {
		err_ = true;
		eof_ = true;
		return false;
	}
	if (n == 0) {
		eof_ = true;
		return false;
	}
	begin_ = 0;
	end_ = (size_t)n;
	return true;
}

inline int FastxReader::getc_()
{
	if (begin_ >= end_ && !fill_())
		return err_ ? -3 : -1;
	return buf_[begin_++];
}

long FastxReader::read(std::string &name, std::string &comment, std::vector<char> &seq,
		std::string &qual)
{
	int c;
	if (last_char_ == 0) {
		while ((c = getc_()) >= 0 && c != '>' && c != '@')
			;
		if (c < 0)
			return c;
		last_char_ = c;
	}
	name.clear();
	comment.clear();
	qual.clear();
	/* name: up to the first whitespace */
	bool any = false;
	while ((c = getc_()) >= 0 && !isspace(c)) {
		name.push_back((char)c);
		any = true;
	}
	if (c < 0 && !any)
		return c == -3 ? -3 : -1;
	if (c >= 0 && c != '\n') {
		while ((c = getc_()) >= 0 && c != '\n')
			comment.push_back((char)c);
		if (comment.size() > 1 && comment.back() == '\r')
			comment.pop_back();
	}
	const size_t s0 = seq.size();
	while ((c = getc_()) >= 0 && c != '>' && c != '+' && c != '@') {
		if (c == '\n')
			continue;
		seq.push_back((char)c);
		while ((c = getc_()) >= 0 && c != '\n')
			seq.push_back((char)c);
		if (seq.size() - s0 > 1 && seq.back() == '\r')
			seq.pop_back();
		if (c < 0)
			break;
	}
	if (c == '>' || c == '@')
		last_char_ = c;
	const long slen = (long)(seq.size() - s0);
	if (c != '+')
		return slen; /* FASTA (or end of input) */
	while ((c = getc_()) >= 0 && c != '\n')
		;
	if (c < 0)
		return -2;
	for (;;) {
		bool got = false;
		while ((c = getc_()) >= 0 && c != '\n') {
			qual.push_back((char)c);
			got = true;
		}
		if (qual.size() > 1 && qual.back() == '\r')
			qual.pop_back();
		if (c == -3)
			return -3;
		if (c < 0 && !got)
			break;
		if ((long)qual.size() >= slen || c < 0)
			break;
	}
	last_char_ = 0;
	if ((long)qual.size() != slen)
		return -2;
	return slen;
}

/* One host batch: concatenated bases (pinned), offsets, read names (and,
 * when records are printed, names, comments and qualities of both mates). */
struct HostBatch {
	char *seq[2] = {nullptr, nullptr};
	size_t cap = 0;
	std::vector<uint64_t> off[2];
	std::vector<std::string> names;
	std::vector<std::string> rname[2], rcomment[2], rqual[2];
	std::vector<uint32_t> cat;
	uint64_t n = 0;
	bool last = false;
};

namespace {

struct Pipe {
	std::mutex mu;
	std::condition_variable cv;
	int filled[2] = {0, 0}; /* 1 = ready for the GPU */
	bool stop = false;
	std::string err;
};

/* Fill b from the reader(s); returns false at end of input. */
bool fill_batch(HostBatch &b, FastxReader *r1, FastxReader *r2, uint64_t max_reads,
		uint64_t max_bases, bool keep_names, bool keep_records, std::vector<char> &s1,
		std::vector<char> &s2, std::string &perr)
{
	std::string name, comment, qual, name2, comment2, qual2;
	b.n = 0;
	b.names.clear();
	for (int m = 0; m < 2; ++m) {
		b.rname[m].clear();
		b.rcomment[m].clear();
		b.rqual[m].clear();
	}
	s1.clear();
	s2.clear();
	b.off[0].assign(1, 0);
	b.off[1].assign(1, 0);
	bool more = true;
	while (b.n < max_reads && s1.size() < max_bases && s2.size() < max_bases) {
		const size_t keep1 = s1.size(), keep2 = s2.size();
		long l1 = r1->read(name, comment, s1, qual);
		long l2 = 0;
		if (r2)
			l2 = r2->read(name2, comment2, s2, qual2);
		if (l1 < 0 || l2 < 0) {
			s1.resize(keep1);
			s2.resize(keep2);
			if (l1 < -1 || l2 < -1)
				perr = l1 == -2 || l2 == -2 ? "truncated quality string" : "stream error";
			more = false;
			break;
		}
		b.off[0].push_back(s1.size());
		if (r2)
			b.off[1].push_back(s2.size());
		if (keep_names)
			b.names.push_back(name);
		if (keep_records) {
			b.rname[0].push_back(name);
			b.rcomment[0].push_back(comment);
			b.rqual[0].push_back(qual);
			if (r2) {
				b.rname[1].push_back(name2);
				b.rcomment[1].push_back(comment2);
				b.rqual[1].push_back(qual2);
			}
		}
		++b.n;
	}
	return more;
}

/* A categorized-read output file: plain or gzip (".gz" postfix), as
 * Dynamicofstream chooses by the name (Common/Dynamicofstream.cpp:14-24). */
struct OutFile {
	FILE *f = nullptr;
	gzFile g = nullptr;
	bool open(const std::string &path)
	{
		if (path.size() >= 3 && path.compare(path.size() - 3, 3, ".gz") == 0)
			g = gzopen(path.c_str(), "wb");
		else
			f = fopen(path.c_str(), "wb");
		return f || g;
	}
	bool write(const std::string &t)
	{
		if (t.empty())
			return true;
		if (g)
			return gzwrite(g, t.data(), (unsigned)t.size()) == (int)t.size();
		return fwrite(t.data(), 1, t.size(), f) == t.size();
	}
	bool close()
	{
		bool ok = true;
		if (g)
			ok = gzclose(g) == Z_OK;
		if (f)
			ok = fclose(f) == 0;
		f = nullptr;
		g = nullptr;
		return ok;
	}
};

/* ">name comment\nseq\n" or "@name comment\nseq\n+\nqual\n", with the space
 * written even for an empty comment (BioBloomClassifier.h:144-209). */
void append_record(std::string &out, bool fastq, const std::string &name,
		const std::string &comment, const char *seq, size_t len, const std::string &qual)
{
	out += fastq ? '@' : '>';
	out += name;
	out += ' ';
	out += comment;
	out += '\n';
	out.append(seq, len);
	if (fastq) {
		out += "\n+\n";
		out += qual;
	}
	out += '\n';
}

int run_pipeline(bbt_ctx *ctx, const std::vector<std::string> &files1, const std::string *file2,
		const char *prefix, const char *read_status, const char *out_type = nullptr,
		const char *postfix = nullptr)
{
	const bool paired = file2 != nullptr;
	const bool print = out_type && out_type[0];
	const bool fastq_out = print && std::string(out_type) == "fq";
	const bool keep_records = print || ctx->to_stdout;
	/* output files: one per filter, then noMatch, then multiMatch
	 * (BioBloomClassifier.cpp:116-127, 319-337) */
	std::vector<OutFile> outs[2];
	if (print) {
		const std::string pre = prefix ? prefix : "", post = postfix ? postfix : "";
		std::vector<std::string> labels(ctx->ids);
		labels.push_back("noMatch");
		labels.push_back("multiMatch");
		for (int m = 0; m < (paired ? 2 : 1); ++m) {
			outs[m].resize(labels.size());
			for (size_t i = 0; i < labels.size(); ++i) {
				const std::string path = pre + "_" + labels[i] +
						(paired ? (m ? "_2." : "_1.") : ".") + out_type + post;
				if (!outs[m][i].open(path)) {
					for (int mm = 0; mm < 2; ++mm)
						for (OutFile &o : outs[mm])
							o.close();
					return fail(ctx, BBT_ERR_IO, "cannot write " + path);
				}
			}
		}
	}
	const uint64_t max_reads = std::min<uint64_t>(ctx->cap_reads, 1ull << 18);
	const uint64_t max_bases = std::min<uint64_t>(ctx->cap_bases, 64ull << 20);
	std::ofstream status;
	if (read_status) {
		status.open(read_status);
		if (!status)
			return fail(ctx, BBT_ERR_IO, std::string("cannot write ") + read_status);
	}
	HostBatch hb[2];
	std::vector<char> stage1[2], stage2[2];
	for (int i = 0; i < 2; ++i) {
		size_t cap = max_bases + (1 << 20);
		cudaError_t e = cudaMallocHost(&hb[i].seq[0], cap);
		if (e == cudaSuccess && paired)
			e = cudaMallocHost(&hb[i].seq[1], cap);
		if (e != cudaSuccess) {
			for (HostBatch &x : hb) {
				cudaFreeHost(x.seq[0]);
				cudaFreeHost(x.seq[1]);
			}
			return cuda_fail(ctx, e, "cudaMallocHost(batch)");
		}
		hb[i].cap = cap;
	}
	Pipe pipe;
	uint64_t total = 0;
	/* Reader thread: fills the two batches alternately.  A batch ends at
	 * max_reads / max_bases or at the end of a file; the final batch (maybe
	 * empty) has last set. */
	std::thread reader([&]() {
		size_t fi = 0;
		FastxReader *r1 = nullptr;
		FastxReader *r2 = nullptr;
		auto open_next = [&]() -> bool {
			delete r1;
			delete r2;
			r1 = r2 = nullptr;
			if (fi >= files1.size())
				return false;
			r1 = new FastxReader(files1[fi]);
			if (!r1->ok()) {
				pipe.err = "file " + files1[fi] + " cannot be opened";
				return false;
			}
			if (paired) {
				r2 = new FastxReader(*file2);
				if (!r2->ok()) {
					pipe.err = "file " + *file2 + " cannot be opened";
					return false;
				}
			}
			++fi;
			return true;
		};
		bool have = open_next();
		int which = 0;
		for (;;) {
			{
				std::unique_lock<std::mutex> lk(pipe.mu);
				pipe.cv.wait(lk, [&] { return pipe.filled[which] == 0 || pipe.stop; });
				if (pipe.stop)
					break;
			}
			HostBatch &b = hb[which];
			b.n = 0;
			if (have) {
				std::string perr;
				bool more = fill_batch(b, r1, r2, max_reads, max_bases, read_status != nullptr,
						keep_records, stage1[which], stage2[which], perr);
				if (!perr.empty())
					std::cerr << "warning: " << perr << "; reading of this file stopped there"
					          << std::endl;
				size_t need = std::max(stage1[which].size(), stage2[which].size());
				if (need > b.cap) {
					/* a record longer than the batch buffer: grow it */
					cudaFreeHost(b.seq[0]);
					cudaFreeHost(b.seq[1]);
					b.seq[0] = b.seq[1] = nullptr;
					b.cap = 0;
					bool okp = cudaMallocHost(&b.seq[0], need) == cudaSuccess &&
							(!paired || cudaMallocHost(&b.seq[1], need) == cudaSuccess);
					if (!okp) {
						pipe.err = "cannot allocate pinned memory for a long record";
						b.n = 0;
						have = false;
					} else {
						b.cap = need;
					}
				}
				if (b.n) {
					memcpy(b.seq[0], stage1[which].data(), stage1[which].size());
					if (paired)
						memcpy(b.seq[1], stage2[which].data(), stage2[which].size());
				}
				if (have && !more)
					have = paired ? false : open_next();
			}
			b.last = !have;
			{
				std::lock_guard<std::mutex> lk(pipe.mu);
				pipe.filled[which] = 1;
			}
			pipe.cv.notify_all();
			if (b.last)
				break;
			which ^= 1;
		}
		delete r1;
		delete r2;
	});
	int rc = BBT_OK;
	int which = 0;
	for (;;) {
		{
			std::unique_lock<std::mutex> lk(pipe.mu);
			pipe.cv.wait(lk, [&] { return pipe.filled[which] != 0; });
		}
		HostBatch &b = hb[which];
		const bool last = b.last;
		if (b.n) {
			b.cat.resize(b.n);
			bbt_batch bt;
			bt.seq = b.seq[0];
			bt.offsets = b.off[0].data();
			bt.seq2 = paired ? b.seq[1] : nullptr;
			bt.offsets2 = paired ? b.off[1].data() : nullptr;
			bt.n_reads = b.n;
			bt.location = BBT_HOST;
			bbt_result res;
			res.hits = nullptr;
			res.hits2 = nullptr;
			res.category = (read_status || keep_records) ? b.cat.data() : nullptr;
			res.location = BBT_HOST;
			rc = bbt_classify_batch(ctx, &bt, &res, nullptr);
			if (rc)
				break;
			if (keep_records) {
				/* categorized files, and stdout for the first filter's reads (-d)
				 * or everything else (-n), BioBloomClassifier.h:115-142, 211-247 */
				std::vector<std::string> text[2];
				if (print) {
					text[0].resize(ctx->nf + 2);
					text[1].resize(ctx->nf + 2);
				}
				std::string so;
				for (uint64_t i = 0; i < b.n; ++i) {
					const uint32_t c = b.cat[i];
					for (int m = 0; m < (paired ? 2 : 1); ++m) {
						const uint64_t o = b.off[m][i], e = b.off[m][i + 1];
						const char *sq = b.seq[m] + o;
						if (print)
							append_record(text[m][c], fastq_out, b.rname[m][i], b.rcomment[m][i],
									sq, e - o, b.rqual[m][i]);
						if (ctx->to_stdout && (ctx->inverse ? c != 0 : c == 0))
							append_record(so, true, b.rname[m][i], b.rcomment[m][i], sq, e - o,
									b.rqual[m][i]);
					}
				}
				for (int m = 0; m < (paired ? 2 : 1) && print; ++m)
					for (size_t c = 0; c < text[m].size(); ++c)
						if (!outs[m][c].write(text[m][c]))
							rc = fail(ctx, BBT_ERR_IO, "cannot write a categorized read file");
				if (!so.empty() && fwrite(so.data(), 1, so.size(), stdout) != so.size())
					rc = fail(ctx, BBT_ERR_IO, "cannot write to stdout");
				if (rc)
					break;
			}
			if (read_status) {
				for (uint64_t i = 0; i < b.n; ++i) {
					uint32_t c = b.cat[i];
					status << b.names[i] << '\t'
					       << (c < ctx->nf ? ctx->ids[c] : c == ctx->nf ? "noMatch" : "multiMatch")
					       << '\n';
				}
			}
			total += b.n;
		}
		{
			std::lock_guard<std::mutex> lk(pipe.mu);
			pipe.filled[which] = 0;
		}
		pipe.cv.notify_all();
		if (last)
			break;
		which ^= 1;
	}
	{
		std::lock_guard<std::mutex> lk(pipe.mu);
		pipe.stop = true;
	}
	pipe.cv.notify_all();
	reader.join();
	for (HostBatch &x : hb) {
		cudaFreeHost(x.seq[0]);
		cudaFreeHost(x.seq[1]);
	}
	bool closed = true;
	for (int m = 0; m < 2; ++m)
		for (OutFile &o : outs[m])
			closed = o.close() && closed;
	fflush(stdout);
	if (rc)
		return rc;
	if (!closed)
		return fail(ctx, BBT_ERR_IO, "cannot write a categorized read file");
	if (!pipe.err.empty())
		return fail(ctx, BBT_ERR_IO, pipe.err);
	std::cerr << "Total Reads: " << total << "\n";
	std::string sum_path = std::string(prefix ? prefix : "") + "_summary.tsv";
	std::cerr << "Writing file: " << sum_path << std::endl;
	std::vector<uint64_t> counts(2 * (ctx->nf + 2) + 2);
	uint64_t reads = 0;
	rc = bbt_summary(ctx, counts.data(), &reads);
	if (rc)
		return rc;
	std::ofstream out(sum_path);
	if (!out)
		return fail(ctx, BBT_ERR_IO, "cannot write " + sum_path);
	out << summary_text(ctx, counts, reads);
	return out ? BBT_OK : fail(ctx, BBT_ERR_IO, "cannot write " + sum_path);
}

} // namespace
} // namespace bbt

using namespace bbt;

extern "C" int bbt_filter_files(bbt_ctx *ctx, const char *const *files, int n_files,
		const char *prefix, const char *read_status)
{
	if (!ctx || !files || n_files <= 0)
		return fail(ctx, BBT_ERR_ARG, "bbt_filter_files: need at least one input file");
	std::vector<std::string> f;
	for (int i = 0; i < n_files; ++i)
		f.push_back(files[i]);
	std::cerr << "Filtering Start" << std::endl;
	return run_pipeline(ctx, f, nullptr, prefix, read_status);
}

extern "C" int bbt_filter_pair_files(bbt_ctx *ctx, const char *file1, const char *file2,
		const char *prefix, const char *read_status)
{
	if (!ctx || !file1 || !file2)
		return fail(ctx, BBT_ERR_ARG, "bbt_filter_pair_files: need two input files");
	std::vector<std::string> f(1, file1);
	std::string f2 = file2;
	std::cerr << "Filtering Start" << std::endl;
	return run_pipeline(ctx, f, &f2, prefix, read_status);
}

extern "C" int bbt_filter_files_print(bbt_ctx *ctx, const char *const *files, int n_files,
		const char *prefix, const char *out_type, const char *postfix, const char *read_status)
{
	if (!ctx || !files || n_files <= 0)
		return fail(ctx, BBT_ERR_ARG, "bbt_filter_files_print: need at least one input file");
	if (!out_type || (std::string(out_type) != "fa" && std::string(out_type) != "fq"))
		return fail(ctx, BBT_ERR_ARG, "bbt_filter_files_print: out_type is \"fa\" or \"fq\"");
	std::vector<std::string> f;
	for (int i = 0; i < n_files; ++i)
		f.push_back(files[i]);
	std::cerr << "Filtering Start" << std::endl;
	return run_pipeline(ctx, f, nullptr, prefix, read_status, out_type, postfix);
}

extern "C" int bbt_filter_pair_files_print(bbt_ctx *ctx, const char *file1, const char *file2,
		const char *prefix, const char *out_type, const char *postfix, const char *read_status)
{
	if (!ctx || !file1 || !file2)
		return fail(ctx, BBT_ERR_ARG, "bbt_filter_pair_files_print: need two input files");
	if (!out_type || (std::string(out_type) != "fa" && std::string(out_type) != "fq"))
		return fail(ctx, BBT_ERR_ARG, "bbt_filter_pair_files_print: out_type is \"fa\" or \"fq\"");
	std::vector<std::string> f(1, file1);
	std::string f2 = file2;
	std::cerr << "Filtering Start" << std::endl;
	return run_pipeline(ctx, f, &f2, prefix, read_status, out_type, postfix);
}
