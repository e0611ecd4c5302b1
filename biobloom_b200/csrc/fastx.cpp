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
#include <unordered_map>

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
	/* the bases 2-bit packed with validity bits (pinned), as the batch goes
	 * to the device when DUST masking is off; pk_bad: a mate has bases that
	 * are not ACGT (else its validity bits are not sent) */
	uint32_t *pkw[2] = {nullptr, nullptr}, *pkv[2] = {nullptr, nullptr};
	size_t pk_cap = 0;
	bool pk_bad[2] = {false, false};
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

/* A mate waiting for its partner in a single-file paired input. */
struct PendingMate {
	std::string comment, qual;
	std::vector<char> seq;
};

/* BioBloomClassifier::filterPair(file) / filterPairPrint(file, type)
 * (BioBloomClassifier.cpp:463-564, 571-729): the header is the read name
 * without its last two characters when it ends in '1' or '2' ("x/1" -> "x");
 * the first record of a header waits in `pending`, the next record with the
 * same header completes the pair (the waiting record is mate 1) and the
 * header is free again.  Records never paired are dropped.  Mates go to the
 * batch in the order their pairs complete. */
bool fill_batch_smart(HostBatch &b, FastxReader *r, uint64_t max_reads, uint64_t max_bases,
		bool keep_names, bool keep_records, std::vector<char> &s1, std::vector<char> &s2,
		std::unordered_map<std::string, PendingMate> &pending, std::string &perr)
{
	std::string name, comment, qual;
	std::vector<char> seq;
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
	while (b.n < max_reads && s1.size() < max_bases && s2.size() < max_bases) {
		seq.clear();
		long l = r->read(name, comment, seq, qual);
		if (l < 0) {
			if (l < -1)
				perr = l == -2 ? "truncated quality string" : "stream error";
			return false;
		}
		if (!name.empty() && (name.back() == '1' || name.back() == '2'))
			name.resize(name.size() >= 2 ? name.size() - 2 : 0);
		auto it = pending.find(name);
		if (it == pending.end()) {
			PendingMate &pm = pending[name];
			pm.comment = comment;
			pm.qual = qual;
			pm.seq = seq;
			continue;
		}
		PendingMate &m1 = it->second;
		s1.insert(s1.end(), m1.seq.begin(), m1.seq.end());
		s2.insert(s2.end(), seq.begin(), seq.end());
		b.off[0].push_back(s1.size());
		b.off[1].push_back(s2.size());
		if (keep_names)
			b.names.push_back(name);
		if (keep_records) {
			b.rname[0].push_back(name);
			b.rcomment[0].push_back(m1.comment);
			b.rqual[0].push_back(m1.qual);
			b.rname[1].push_back(name);
			b.rcomment[1].push_back(comment);
			b.rqual[1].push_back(qual);
		}
		pending.erase(it);
		++b.n;
	}
	return true;
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
 * written even for an empty comment (BioBloomClassifier.h:144-209); extra
 * (scores, each with its leading space) goes right after the comment. */
void append_record(std::string &out, bool fastq, const std::string &name,
		const std::string &comment, const char *seq, size_t len, const std::string &qual,
		const std::string &extra = std::string())
{
	out += fastq ? '@' : '>';
	out += name;
	out += ' ';
	out += comment;
	out += extra;
	out += '\n';
	out.append(seq, len);
	if (fastq) {
		out += "\n+\n";
		out += qual;
	}
	out += '\n';
}

/* A double as std::ostream prints it by default (precision 6, %g). */
void append_double(std::string &out, double v)
{
	char buf[64];
	snprintf(buf, sizeof buf, " %g", v);
	out += buf;
}

/* BESTHIT: the largest score of one read (evaluateReadBestHit,
 * BioBloomClassifier.cpp:1194-1218: maxScore starts at 0) and how many
 * filters reach it (none unless it is above 0). */
double best_of(const double *sc, uint32_t nf, uint32_t *count)
{
	double mx = 0;
	for (uint32_t f = 0; f < nf; ++f)
		if (mx < sc[f])
			mx = sc[f];
	uint32_t c = 0;
	if (mx > 0)
		for (uint32_t f = 0; f < nf; ++f)
			c += sc[f] == mx;
	*count = c;
	return mx;
}

/* What a categorized file's record carries after the comment
 * (printSingleToFile / printPairToFile, BioBloomClassifier.h:144-209,
 * 291-411): SCORES puts every filter's score on multiMatch records; BESTHIT
 * puts the read's best score on every record, except multiMatch records of
 * FASTA files and of pairs, which carry the score once per best filter. */
std::string file_extra(const bbt_ctx *ctx, uint32_t cat, bool fastq, bool paired,
		const double *sc)
{
	std::string x;
	const uint32_t multi = ctx->nf + 1;
	if (ctx->mode == BBT_MODE_SCORES && cat == multi) {
		for (uint32_t f = 0; f < ctx->nf; ++f)
			append_double(x, sc[f]);
	} else if (ctx->mode == BBT_MODE_BESTHIT) {
		uint32_t cnt = 0;
		const double mx = best_of(sc, ctx->nf, &cnt);
		if (cat == multi && (!fastq || paired)) {
			for (uint32_t i = 0; i < cnt; ++i)
				append_double(x, mx);
		} else {
			append_double(x, mx);
		}
	}
	return x;
}

/* The reads of one pipeline run: single-end files; pairs of files (files2[i]
 * holds the mates of files1[i]); or one file whose mates are matched by name. */
struct PipeInput {
	std::vector<std::string> files1, files2;
	bool smart = false;
};

int run_pipeline(bbt_ctx *ctx, const PipeInput &in, const char *prefix, const char *read_status,
		const char *out_type = nullptr, const char *postfix = nullptr)
{
	const std::vector<std::string> &files1 = in.files1;
	const bool paired = in.smart || !in.files2.empty();
	const bool print = out_type && out_type[0];
	const bool fastq_out = print && std::string(out_type) == "fq";
	const bool keep_records = print || ctx->to_stdout;
	/* BESTHIT and SCORES records carry evalScore values */
	const bool want_scores = keep_records &&
			(ctx->mode == BBT_MODE_BESTHIT || ctx->mode == BBT_MODE_SCORES);
	std::vector<double> scores[2];
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
	/* batches cross to the device 2-bit packed (a quarter of the bytes)
	 * unless DUST masking needs the ASCII bases there; the ASCII copy stays
	 * on the host for printing records */
	const bool pack = !ctx->dust;
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
		std::unordered_map<std::string, PendingMate> pending;
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
			if (!in.files2.empty()) {
				r2 = new FastxReader(in.files2[fi]);
				if (!r2->ok()) {
					pipe.err = "file " + in.files2[fi] + " cannot be opened";
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
				bool more = in.smart
						? fill_batch_smart(b, r1, max_reads, max_bases, read_status != nullptr,
								keep_records, stage1[which], stage2[which], pending, perr)
						: fill_batch(b, r1, r2, max_reads, max_bases, read_status != nullptr,
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
				if (b.n && pack && need > b.pk_cap) {
					for (int m = 0; m < 2; ++m) {
						cudaFreeHost(b.pkw[m]);
						cudaFreeHost(b.pkv[m]);
						b.pkw[m] = b.pkv[m] = nullptr;
					}
					b.pk_cap = 0;
					const size_t cap = std::max(need, b.cap);
					bool okp = true;
					for (int m = 0; okp && m < (paired ? 2 : 1); ++m)
						okp = cudaMallocHost(&b.pkw[m], (cap / 16 + 2) * sizeof(uint32_t)) ==
										cudaSuccess &&
								cudaMallocHost(&b.pkv[m], (cap / 32 + 2) * sizeof(uint32_t)) ==
										cudaSuccess;
					if (!okp) {
						pipe.err = "cannot allocate pinned memory for packed bases";
						b.n = 0;
						have = false;
					} else {
						b.pk_cap = cap;
					}
				}
				if (b.n && pack) {
					for (int m = 0; m < (paired ? 2 : 1); ++m) {
						const std::vector<char> &st = m ? stage2[which] : stage1[which];
						uint64_t bad = 0;
						bbt_pack_bases(st.data(), st.size(), b.pkw[m], b.pkv[m], &bad);
						b.pk_bad[m] = bad != 0;
					}
				}
				if (b.n && (!pack || keep_records)) {
					memcpy(b.seq[0], stage1[which].data(), stage1[which].size());
					if (paired)
						memcpy(b.seq[1], stage2[which].data(), stage2[which].size());
				}
				if (have && !more)
					have = in.smart ? false : open_next();
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
			bbt_batch bt = {};
			bt.seq = b.seq[0];
			bt.offsets = b.off[0].data();
			bt.seq2 = paired ? b.seq[1] : nullptr;
			bt.offsets2 = paired ? b.off[1].data() : nullptr;
			bt.n_reads = b.n;
			bt.location = BBT_HOST;
			if (pack) {
				bt.encoding = BBT_BASES_2BIT;
				bt.seq = (const char *)b.pkw[0];
				bt.valid = b.pk_bad[0] ? b.pkv[0] : nullptr;
				if (paired) {
					bt.seq2 = (const char *)b.pkw[1];
					bt.valid2 = b.pk_bad[1] ? b.pkv[1] : nullptr;
				}
			}
			bbt_result res;
			res.hits = nullptr;
			res.hits2 = nullptr;
			res.category = (read_status || keep_records) ? b.cat.data() : nullptr;
			res.location = BBT_HOST;
			if (want_scores) {
				for (int m = 0; m < (paired ? 2 : 1); ++m)
					scores[m].resize(b.n * ctx->nf);
				rc = bbt_classify_batch_scores(ctx, &bt, &res, scores[0].data(),
						paired ? scores[1].data() : nullptr, nullptr);
			} else {
				rc = bbt_classify_batch(ctx, &bt, &res, nullptr);
			}
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
				const std::string none;
				for (uint64_t i = 0; i < b.n; ++i) {
					const uint32_t c = b.cat[i];
					for (int m = 0; m < (paired ? 2 : 1); ++m) {
						const uint64_t o = b.off[m][i], e = b.off[m][i + 1];
						const char *sq = b.seq[m] + o;
						const double *sc = want_scores ? scores[m].data() + i * ctx->nf : nullptr;
						if (print)
							append_record(text[m][c], fastq_out, b.rname[m][i], b.rcomment[m][i],
									sq, e - o, b.rqual[m][i],
									sc ? file_extra(ctx, c, fastq_out, paired, sc) : none);
						if (ctx->to_stdout && (ctx->inverse ? c != 0 : c == 0)) {
							/* printSingle / printPair: BESTHIT adds the read's score */
							std::string x;
							if (sc && !ctx->inverse && ctx->mode == BBT_MODE_BESTHIT) {
								uint32_t cnt;
								append_double(x, best_of(sc, ctx->nf, &cnt));
							}
							append_record(so, true, b.rname[m][i], b.rcomment[m][i], sq, e - o,
									b.rqual[m][i], x);
						}
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
		for (int m = 0; m < 2; ++m) {
			cudaFreeHost(x.pkw[m]);
			cudaFreeHost(x.pkv[m]);
		}
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

static bool valid_out_type(const char *t)
{
	return t && (std::string(t) == "fa" || std::string(t) == "fq");
}

extern "C" int bbt_filter_files(bbt_ctx *ctx, const char *const *files, int n_files,
		const char *prefix, const char *read_status)
{
	if (!ctx || !files || n_files <= 0)
		return fail(ctx, BBT_ERR_ARG, "bbt_filter_files: need at least one input file");
	PipeInput in;
	for (int i = 0; i < n_files; ++i)
		in.files1.push_back(files[i]);
	std::cerr << "Filtering Start" << std::endl;
	return run_pipeline(ctx, in, prefix, read_status);
}

extern "C" int bbt_filter_pair_files(bbt_ctx *ctx, const char *file1, const char *file2,
		const char *prefix, const char *read_status)
{
	if (!ctx || !file1 || !file2)
		return fail(ctx, BBT_ERR_ARG, "bbt_filter_pair_files: need two input files");
	PipeInput in;
	in.files1.push_back(file1);
	in.files2.push_back(file2);
	std::cerr << "Filtering Start" << std::endl;
	return run_pipeline(ctx, in, prefix, read_status);
}

extern "C" int bbt_filter_files_print(bbt_ctx *ctx, const char *const *files, int n_files,
		const char *prefix, const char *out_type, const char *postfix, const char *read_status)
{
	if (!ctx || !files || n_files <= 0)
		return fail(ctx, BBT_ERR_ARG, "bbt_filter_files_print: need at least one input file");
	if (!valid_out_type(out_type))
		return fail(ctx, BBT_ERR_ARG, "bbt_filter_files_print: out_type is \"fa\" or \"fq\"");
	PipeInput in;
	for (int i = 0; i < n_files; ++i)
		in.files1.push_back(files[i]);
	std::cerr << "Filtering Start" << std::endl;
	return run_pipeline(ctx, in, prefix, read_status, out_type, postfix);
}

extern "C" int bbt_filter_pair_files_print(bbt_ctx *ctx, const char *file1, const char *file2,
		const char *prefix, const char *out_type, const char *postfix, const char *read_status)
{
	if (!ctx || !file1 || !file2)
		return fail(ctx, BBT_ERR_ARG, "bbt_filter_pair_files_print: need two input files");
	if (!valid_out_type(out_type))
		return fail(ctx, BBT_ERR_ARG,
				"bbt_filter_pair_files_print: out_type is \"fa\" or \"fq\"");
	PipeInput in;
	in.files1.push_back(file1);
	in.files2.push_back(file2);
	std::cerr << "Filtering Start" << std::endl;
	return run_pipeline(ctx, in, prefix, read_status, out_type, postfix);
}

extern "C" int bbt_filter_pair_file_lists(bbt_ctx *ctx, const char *const *files1,
		const char *const *files2, int n_pairs, const char *prefix, const char *read_status)
{
	if (!ctx || !files1 || !files2 || n_pairs <= 0)
		return fail(ctx, BBT_ERR_ARG, "bbt_filter_pair_file_lists: need at least one file pair");
	PipeInput in;
	for (int i = 0; i < n_pairs; ++i) {
		in.files1.push_back(files1[i] ? files1[i] : "");
		in.files2.push_back(files2[i] ? files2[i] : "");
	}
	std::cerr << "Filtering Start" << std::endl;
	return run_pipeline(ctx, in, prefix, read_status);
}

extern "C" int bbt_filter_smart_pairs(bbt_ctx *ctx, const char *file, const char *prefix,
		const char *read_status)
{
	if (!ctx || !file)
		return fail(ctx, BBT_ERR_ARG, "bbt_filter_smart_pairs: need an input file");
	PipeInput in;
	in.files1.push_back(file);
	in.smart = true;
	std::cerr << "Filtering Start" << std::endl;
	return run_pipeline(ctx, in, prefix, read_status);
}

extern "C" int bbt_filter_smart_pairs_print(bbt_ctx *ctx, const char *file, const char *prefix,
		const char *out_type, const char *postfix, const char *read_status)
{
	if (!ctx || !file)
		return fail(ctx, BBT_ERR_ARG, "bbt_filter_smart_pairs_print: need an input file");
	if (!valid_out_type(out_type))
		return fail(ctx, BBT_ERR_ARG,
				"bbt_filter_smart_pairs_print: out_type is \"fa\" or \"fq\"");
	PipeInput in;
	in.files1.push_back(file);
	in.smart = true;
	std::cerr << "Filtering Start" << std::endl;
	return run_pipeline(ctx, in, prefix, read_status, out_type, postfix);
}
