/*
 * mibf_pipeline.cpp -- the file pipeline of biobloommicategorizer
 * (bbt_mibf_filter_files / bbt_mibf_filter_pair_files).
 *
 * Replaces MIBFClassifier::filter / filterPair (MIBFClassifier.hpp:200-616):
 * a reader thread parses records into one of two batches while the other is
 * classified on the device; records are written in input order (the
 * reference's one-thread order), then "<prefix>_summary.tsv".  The read count
 * of the summary is the number of reads (pairs) read, which is what the
 * reference's threaded loops count (its one-thread single-end loop leaves the
 * count at 0, MIBFClassifier.hpp:217-226).
 */
#include <condition_variable>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <iostream>
#include <mutex>
#include <thread>

#include "fastx.hpp"
#include "mibf_ctx.hpp"

namespace bbt {
namespace {

struct MiBatch {
	std::vector<char> seq[2];
	/* the bases 2-bit packed with validity bits, as the batch goes to the
	 * device (the ASCII bases stay for the output records); bad: a mate has
	 * bases that are not ACGT (else its validity bits are not sent) */
	std::vector<uint32_t> pw[2], pv[2];
	bool bad[2] = {false, false};
	std::vector<uint64_t> off[2];
	std::vector<std::string> name[2], comment[2], qual[2];
	uint64_t n = 0;
	bool last = false;
};

struct MiPipe {
	std::mutex mu;
	std::condition_variable cv;
	int filled[2] = {0, 0};
	bool stop = false;
	std::string err;
};

constexpr uint64_t kBatchReads = 1ull << 16;
constexpr uint64_t kBatchBases = 32ull << 20;

/* Read up to one batch; returns false at the end of the input(s). */
bool fill(MiBatch &b, FastxReader *r1, FastxReader *r2, bool keep_qual, std::string &perr)
{
	std::string nm, cm, ql;
	for (int m = 0; m < 2; ++m) {
		b.seq[m].clear();
		b.off[m].assign(1, 0);
		b.name[m].clear();
		b.comment[m].clear();
		b.qual[m].clear();
	}
	b.n = 0;
	while (b.n < kBatchReads && b.seq[0].size() < kBatchBases && b.seq[1].size() < kBatchBases) {
		const size_t k1 = b.seq[0].size(), k2 = b.seq[1].size();
		long l1 = r1->read(nm, cm, b.seq[0], ql);
		if (l1 < 0) {
			b.seq[0].resize(k1);
			if (l1 < -1)
				perr = l1 == -2 ? "truncated quality string" : "stream error";
			return false;
		}
		b.name[0].push_back(nm);
		b.comment[0].push_back(cm);
		if (keep_qual)
			b.qual[0].push_back(ql);
		if (r2) {
			long l2 = r2->read(nm, cm, b.seq[1], ql);
			if (l2 < 0) {
				b.seq[0].resize(k1);
				b.seq[1].resize(k2);
				b.name[0].pop_back();
				b.comment[0].pop_back();
				if (keep_qual)
					b.qual[0].pop_back();
				if (l2 < -1)
					perr = l2 == -2 ? "truncated quality string" : "stream error";
				return false;
			}
			b.name[1].push_back(nm);
			b.comment[1].push_back(cm);
			if (keep_qual)
				b.qual[1].push_back(ql);
			b.off[1].push_back(b.seq[1].size());
		}
		b.off[0].push_back(b.seq[0].size());
		++b.n;
	}
	return true;
}

int run(bbt_mibf *ctx, const std::vector<std::string> &files, const std::string *file2,
		const char *prefix, int out_type, FILE *out)
{
	const bool paired = file2 != nullptr;
	const bool keep_qual = out_type == BBT_MIBF_OUT_FASTQ;
	MiBatch hb[2];
	MiPipe pipe;
	std::thread reader([&]() {
		size_t fi = 0;
		FastxReader *r1 = nullptr, *r2 = nullptr;
		auto open_next = [&]() -> bool {
			delete r1;
			delete r2;
			r1 = r2 = nullptr;
			if (fi >= files.size())
				return false;
			r1 = new FastxReader(files[fi]);
			if (!r1->ok()) {
				pipe.err = "file " + files[fi] + " cannot be opened";
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
			MiBatch &b = hb[which];
			b.n = 0;
			if (have) {
				std::string perr;
				bool more = fill(b, r1, r2, keep_qual, perr);
				for (int m = 0; b.n && m < (paired ? 2 : 1); ++m) {
					const uint64_t nb = b.seq[m].size();
					b.pw[m].resize(nb / 16 + 2);
					b.pv[m].resize(nb / 32 + 2);
					uint64_t nbad = 0;
					bbt_pack_bases(b.seq[m].data(), nb, b.pw[m].data(), b.pv[m].data(), &nbad);
					b.bad[m] = nbad != 0;
				}
				if (!perr.empty())
					std::cerr << "warning: " << perr << "; reading of this file stopped there"
					          << std::endl;
				if (!more)
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
	uint64_t total = 0;
	int which = 0;
	std::vector<bbt_mibf_hit> hits;
	std::vector<uint32_t> nh, sat;
	std::string text;
	const uint32_t nids = (uint32_t)ctx->names.size();
	for (;;) {
		{
			std::unique_lock<std::mutex> lk(pipe.mu);
			pipe.cv.wait(lk, [&] { return pipe.filled[which] != 0; });
		}
		MiBatch &b = hb[which];
		const bool last = b.last;
		if (b.n) {
			bbt_batch bt = {};
			bt.seq = (const char *)b.pw[0].data();
			bt.offsets = b.off[0].data();
			bt.seq2 = paired ? (const char *)b.pw[1].data() : nullptr;
			bt.offsets2 = paired ? b.off[1].data() : nullptr;
			bt.n_reads = b.n;
			bt.location = BBT_HOST;
			bt.encoding = BBT_BASES_2BIT;
			bt.valid = b.bad[0] ? b.pv[0].data() : nullptr;
			bt.valid2 = paired && b.bad[1] ? b.pv[1].data() : nullptr;
			uint32_t mh = std::min<uint32_t>(8, nids);
			for (;;) {
				hits.resize(b.n * mh);
				nh.resize(b.n);
				sat.resize(b.n);
				bbt_mibf_result res;
				res.hits = hits.data();
				res.max_hits = mh;
				res.n_hits = nh.data();
				res.sat_count = sat.data();
				res.location = BBT_HOST;
				rc = bbt_mibf_classify_batch(ctx, &bt, &res, nullptr);
				if (rc == BBT_ERR_OVERFLOW && mh < nids) {
					mh = nids; /* the summary was not counted; run the batch again */
					continue;
				}
				break;
			}
			if (rc)
				break;
			text.clear();
			for (uint64_t i = 0; i < b.n; ++i) {
				if (ctx->p.hit_only && nh[i] == 0)
					continue;
				const bbt_mibf_hit *hp = hits.data() + i * mh;
				for (int m = 0; m < (paired ? 2 : 1); ++m) {
					const uint64_t o = b.off[m][i], e = b.off[m][i + 1];
					std::string seq(b.seq[m].data() + o, e - o);
					mibf_format_record(text, ctx->names, out_type, b.name[m][i].c_str(),
							b.comment[m][i].c_str(), seq.c_str(),
							keep_qual ? b.qual[m][i].c_str() : nullptr, hp, nh[i], sat[i]);
				}
			}
			if (!text.empty() && fwrite(text.data(), 1, text.size(), out) != text.size()) {
				rc = mibf_fail(ctx, BBT_ERR_IO, "cannot write the read records");
				break;
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
	fflush(out);
	if (rc)
		return rc;
	if (!pipe.err.empty())
		return mibf_fail(ctx, BBT_ERR_IO, pipe.err);
	std::cerr << "Total Reads:" << total << std::endl;
	const std::string sum_path = std::string(prefix ? prefix : "") + "_summary.tsv";
	std::cerr << "Writing file: " << sum_path << std::endl;
	std::vector<uint64_t> counts(2 * (ctx->names.size() + 2) + 2);
	rc = bbt_mibf_summary(ctx, counts.data(), nullptr);
	if (rc)
		return rc;
	std::ofstream so(sum_path);
	if (!so)
		return mibf_fail(ctx, BBT_ERR_IO, "cannot write " + sum_path);
	so << mibf_summary_text(ctx->names, counts, total);
	return so ? BBT_OK : mibf_fail(ctx, BBT_ERR_IO, "cannot write " + sum_path);
}

} // namespace
} // namespace bbt

using namespace bbt;

extern "C" int bbt_mibf_filter_files(bbt_mibf *ctx, const char *const *files, int n_files,
		const char *prefix, int out_type, void *out)
{
	if (!ctx || !files || n_files <= 0)
		return mibf_fail(ctx, BBT_ERR_ARG, "bbt_mibf_filter_files: need at least one input file");
	std::vector<std::string> f;
	for (int i = 0; i < n_files; ++i)
		f.push_back(files[i]);
	std::cerr << "Filtering Start" << std::endl;
	return run(ctx, f, nullptr, prefix, out_type, out ? (FILE *)out : stdout);
}

extern "C" int bbt_mibf_filter_pair_files(bbt_mibf *ctx, const char *file1, const char *file2,
		const char *prefix, int out_type, void *out)
{
	if (!ctx || !file1 || !file2)
		return mibf_fail(ctx, BBT_ERR_ARG, "bbt_mibf_filter_pair_files: need two input files");
	std::vector<std::string> f(1, file1);
	std::string f2 = file2;
	return run(ctx, f, &f2, prefix, out_type, out ? (FILE *)out : stdout);
}
