/*
 * mibf_host.cpp -- host-side pieces of the miBF path: the file formats, the
 * significance thresholds (frame probabilities and minCount), the seed tables
 * of the kernels, and the record / summary text of biobloommicategorizer.
 */
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <sstream>

#include "mibf_ctx.hpp"

namespace bbt {

void set_global_error(const std::string &msg);

int mibf_fail(bbt_mibf *ctx, int code, const std::string &msg)
{
	if (ctx)
		ctx->err = msg;
	else
		set_global_error(msg);
	return code;
}

static std::string trim(const std::string &s)
{
	size_t a = s.find_first_not_of(" \t\r\n"), b = s.find_last_not_of(" \t\r\n");
	return a == std::string::npos ? std::string() : s.substr(a, b - a + 1);
}

std::string read_mibf_header(FILE *f, MibfHeader &h)
{
	char line[1 << 14];
	if (!fgets(line, sizeof line, f) || strcmp(line, "[BTLMIBloomFilter]\n") != 0)
		return "not a miBF file (no [BTLMIBloomFilter] header)";
	bool end = false, have_m = false, have_pop = false;
	while (fgets(line, sizeof line, f)) {
		if (!strcmp(line, "[HeaderEnd]\n")) {
			end = true;
			break;
		}
		std::string s(line);
		size_t eq = s.find('=');
		if (eq == std::string::npos)
			return "malformed header line: " + trim(s);
		std::string key = trim(s.substr(0, eq)), val = trim(s.substr(eq + 1));
		if (key == "BitVectorSize") {
			h.m = strtoull(val.c_str(), nullptr, 10);
			have_m = true;
		} else if (key == "HashNum") {
			h.h = (unsigned)strtoul(val.c_str(), nullptr, 10);
		} else if (key == "KmerSize") {
			h.k = (unsigned)strtoul(val.c_str(), nullptr, 10);
		} else if (key == "IDWidth") {
			h.id_width = (unsigned)strtoul(val.c_str(), nullptr, 10);
		} else if (key == "PopCount") {
			h.pop = strtoull(val.c_str(), nullptr, 10);
			have_pop = true;
		} else if (key == "Seeds") {
			std::stringstream in(val);
			std::string t;
			while (in >> t)
				h.seeds.push_back(t);
		}
	}
	if (!end)
		return "header has no [HeaderEnd]";
	if (!have_m || h.m == 0 || h.m % 64)
		return "BitVectorSize must be a positive multiple of 64";
	if (!have_pop)
		return "header has no PopCount";
	if (h.id_width != 16)
		return "only 16-bit IDs are supported";
	if (h.k == 0 || h.k > kMibfMaxK)
		return "KmerSize must be between 1 and 32";
	if (h.h == 0 || h.h > kMibfMaxSeeds)
		return "HashNum must be between 1 and 16";
	if (!h.seeds.empty()) {
		if (h.seeds.size() != h.h)
			return "the number of seeds differs from HashNum";
		for (const std::string &s : h.seeds) {
			if (s.size() != h.k)
				return "a seed's length differs from KmerSize";
			if (s.find_first_not_of("01") != std::string::npos)
				return "seeds are strings of '0' and '1'";
		}
	}
	return std::string();
}

int write_mibf_header(FILE *f, const MibfHeader &h)
{
	int r = fprintf(f, "[BTLMIBloomFilter]\nFormat = 1\nBitVectorSize = %llu\nHashNum = %u\n"
			"KmerSize = %u\nIDWidth = 16\nSeeds =", (unsigned long long)h.m, h.h, h.k);
	for (const std::string &s : h.seeds)
		r = r < 0 ? r : fprintf(f, " %s", s.c_str());
	r = r < 0 ? r : fprintf(f, "\nPopCount = %llu\n[HeaderEnd]\n", (unsigned long long)h.pop);
	return r < 0 ? -1 : 0;
}

std::string mibf_ids_path(const std::string &bf_path)
{
	return bf_path.substr(0, bf_path.size() >= 3 ? bf_path.size() - 3 : 0) + "_ids.txt";
}

std::string mibf_sdsl_path(const std::string &bf_path)
{
	return bf_path.substr(0, bf_path.size() >= 3 ? bf_path.size() - 3 : 0) + ".sdsl";
}

/* The loop of MIBFClassifier.hpp:67-76: a line counts only when the next
 * getline still leaves the stream good, so an unterminated last line is
 * dropped; each line gives its second whitespace-separated field. */
bool read_mibf_names(const std::string &path, std::vector<std::string> &names)
{
	std::ifstream in(path.c_str());
	if (!in.good())
		return false;
	names.assign(1, "repeat");
	std::string line;
	std::getline(in, line);
	while (in.good()) {
		std::stringstream conv(line);
		unsigned short id;
		std::string name;
		conv >> id;
		conv >> name;
		names.push_back(name);
		std::getline(in, line);
	}
	return true;
}

double mibf_frame_prob(double p, unsigned h, unsigned need)
{
	double acc = 0;
	for (unsigned j = need; j <= h; ++j) {
		double c = 1;
		for (unsigned t = 0; t < j; ++t)
			c = c * (double)(h - t) / (double)(t + 1);
		acc += c * pow(p, (double)j) * pow(1.0 - p, (double)(h - j));
	}
	return acc;
}

static double binom_pmf(double n, double p, double i)
{
	if (p <= 0.0)
		return i == 0 ? 1.0 : 0.0;
	if (p >= 1.0)
		return i == n ? 1.0 : 0.0;
	return exp(lgamma(n + 1) - lgamma(i + 1) - lgamma(n - i + 1) + i * log(p) +
			(n - i) * log1p(-p));
}

/* n * KL(x/n || p) for x/n > p: by the Chernoff bound the binomial pmf at x is
 * at most exp(-this). */
static double chernoff_exponent(double n, double p, double x)
{
	const double a = x / n;
	double d = a * log(a / p);
	if (a < 1.0)
		d += (1.0 - a) * log((1.0 - a) / (1.0 - p));
	return n * d;
}

/*
 * Smallest x with P(X > x) <= q, X ~ Binomial(n, p), the pmf summed from x = n
 * down in double precision.  Terms whose Chernoff bound is below e^-800 are
 * exactly 0.0 in double (exp underflows below about e^-745, and the computed
 * exponent is off by far less than 55), so the sum starts at the largest x
 * above n*p whose bound is not that small: the additions that change the sum,
 * and so the result, are exactly those of summing every term from x = n.
 */
unsigned binom_upper_quantile(unsigned n_, double p, double q)
{
	const double n = n_;
	double x = n, tail = 0.0;
	if (p > 0.0 && p < 1.0 && n > 64 && chernoff_exponent(n, p, n) > 800.0) {
		double lo = std::ceil(n * p) + 1.0, hi = n; /* bound(hi) > 800 */
		if (lo < hi && chernoff_exponent(n, p, lo) <= 800.0) {
			while (hi - lo > 1.0) {
				double mid = std::floor((lo + hi) / 2);
				if (chernoff_exponent(n, p, mid) > 800.0)
					hi = mid;
				else
					lo = mid;
			}
			x = std::min(n, hi + 2.0); /* every term above is exactly zero */
		}
	}
	while (x > 0) {
		double t = tail + binom_pmf(n, p, x);
		if (t > q)
			break;
		tail = t;
		x -= 1.0;
	}
	return (unsigned)x;
}

unsigned mibf_min_count(unsigned frame_count, double frame_prob, double score, unsigned num_ids)
{
	const double critical = score / double(num_ids - 1);
	const unsigned i = binom_upper_quantile(frame_count, frame_prob, critical);
	return i > 1 ? i : 1;
}

static inline uint64_t rol64(uint64_t v, unsigned s)
{
	s &= 63u;
	return s ? (v << s) | (v >> (64u - s)) : v;
}

std::vector<unsigned long long> mibf_seed_tables(const std::vector<std::string> &seeds,
		unsigned k)
{
	static const uint64_t fw[4] = {0x3c8bfbb395c60474ULL, 0x3193c18562a02b4cULL,
			0x20323ed082572324ULL, 0x295549f54be24456ULL};
	std::vector<std::string> eff = seeds;
	if (eff.empty())
		eff.push_back(std::string(k, '1')); /* k-mer mode: one seed of all care */
	std::vector<unsigned long long> t(eff.size() * 32 * 4 * 2, 0ull);
	for (size_t s = 0; s < eff.size(); ++s)
		for (unsigned j = 0; j < k && j < 32; ++j) {
			if (eff[s][j] != '1')
				continue;
			for (unsigned c = 0; c < 4; ++c) {
				unsigned long long *e = &t[((s * 32 + j) * 4 + c) * 2];
				e[0] = rol64(fw[c], k - 1 - j);
				e[1] = rol64(fw[3 - c], j);
			}
		}
	return t;
}

std::string mibf_summary_text(const std::vector<std::string> &names,
		const std::vector<uint64_t> &c, uint64_t reads)
{
	const size_t nf = names.size();
	const uint64_t *above = c.data();
	const uint64_t *unique = c.data() + (nf + 2);
	const uint64_t multi = c[2 * (nf + 2)];
	const uint64_t nomatch = c[2 * (nf + 2) + 1];
	const double rc = (double)reads;
	std::ostringstream o;
	o << "filter_id\thits\tmisses\tshared\trate_hit\trate_miss\trate_shared\n";
	for (size_t i = 0; i < nf; ++i) {
		o << names[i] << "\t" << above[i] << "\t" << reads - above[i] << "\t"
		  << (above[i] - unique[i]) << "\t" << double(above[i]) / rc << "\t"
		  << double(reads - above[i]) / rc << "\t" << double(above[i] - unique[i]) / rc << "\n";
	}
	o << "multiMatch\t" << multi << "\t" << reads - multi << "\t" << 0 << "\t"
	  << double(multi) / rc << "\t" << double(reads - multi) / rc << "\t" << 0.0 << "\n";
	o << "noMatch\t" << nomatch << "\t" << reads - nomatch << "\t" << 0 << "\t"
	  << double(nomatch) / rc << "\t" << double(reads - nomatch) / rc << "\t" << 0.0 << "\n";
	return o.str();
}

static void append_results(std::string &out, const std::vector<std::string> &names,
		const bbt_mibf_hit *hits, uint32_t n)
{
	out += '\t';
	char num[16];
	for (uint32_t i = 0; i < n; ++i) {
		if (i)
			out += ';';
		out += hits[i].id < names.size() ? names[hits[i].id] : std::string();
		const uint32_t v[6] = {hits[i].nonSatFrameCount, hits[i].solidCount, hits[i].count,
				hits[i].nonSatCount, hits[i].totalNonSatCount, hits[i].totalCount};
		for (uint32_t x : v) {
			snprintf(num, sizeof num, ",%u", x);
			out += num;
		}
	}
}

void mibf_format_record(std::string &out, const std::vector<std::string> &names, int out_type,
		const char *name, const char *comment, const char *seq, const char *qual,
		const bbt_mibf_hit *hits, uint32_t n_hits, uint32_t sat_count)
{
	const bool has_comment = comment && comment[0];
	auto best_name = [&]() -> std::string {
		return hits[0].id < names.size() ? names[hits[0].id] : std::string();
	};
	if (out_type == BBT_MIBF_OUT_FASTA || out_type == BBT_MIBF_OUT_FASTQ) {
		out += out_type == BBT_MIBF_OUT_FASTA ? '>' : '@';
		out += name;
		if (has_comment) {
			out += ' ';
			out += comment;
		}
		if (n_hits) {
			out += '\t';
			out += best_name();
			append_results(out, names, hits, n_hits);
		}
		out += '\n';
		out += seq ? seq : "";
		if (out_type == BBT_MIBF_OUT_FASTQ) {
			out += "\n+\n";
			out += qual ? qual : "";
		}
	} else {
		out += n_hits ? best_name() : std::string("*");
		out += '\t';
		out += name;
		if (has_comment) {
			out += ' ';
			out += comment;
		}
		out += '\t';
		out += std::to_string(sat_count);
		if (n_hits)
			append_results(out, names, hits, n_hits);
		else
			out += "\t*";
	}
	out += '\n';
}

} // namespace bbt

using namespace bbt;

/* The host half of loading: header, names, frame probabilities.  The ID array
 * is counted per ID on the way through (calcFrameProbs) and, when ids_out is
 * given, kept. */
int bbt::mibf_load_host(bbt_mibf *ctx, const char *bf_path, std::vector<uint16_t> *ids_out)
{
	const std::string path = bf_path ? bf_path : "";
	FILE *f = fopen(path.c_str(), "rb");
	if (!f)
		return mibf_fail(ctx, BBT_ERR_IO, "Error: " + path + " File cannot be opened");
	std::string msg = read_mibf_header(f, ctx->hd);
	if (!msg.empty()) {
		fclose(f);
		return mibf_fail(ctx, BBT_ERR_FORMAT, path + ": " + msg);
	}
	const std::string idp = mibf_ids_path(path);
	if (!read_mibf_names(idp, ctx->names)) {
		fclose(f);
		return mibf_fail(ctx, BBT_ERR_IO, "Error: " + idp +
				" File cannot be opened. A corresponding id file is needed.");
	}
	if (ctx->names.size() > kMibfMaxIds) {
		fclose(f);
		return mibf_fail(ctx, BBT_ERR_UNSUPPORTED, "more than " + std::to_string(kMibfMaxIds - 1) +
				" targets in " + idp + " (IDs are 15-bit)");
	}
	const unsigned nids = (unsigned)ctx->names.size();
	std::vector<uint64_t> owned(nids, 0);
	uint64_t sat = 0;
	if (ids_out)
		ids_out->resize(ctx->hd.pop);
	std::vector<uint16_t> chunk;
	const uint64_t step = 1ull << 24;
	for (uint64_t done = 0; done < ctx->hd.pop;) {
		const uint64_t n = std::min<uint64_t>(step, ctx->hd.pop - done);
		uint16_t *dst;
		if (ids_out) {
			dst = ids_out->data() + done;
		} else {
			chunk.resize(n);
			dst = chunk.data();
		}
		if (fread(dst, sizeof(uint16_t), n, f) != n) {
			fclose(f);
			return mibf_fail(ctx, BBT_ERR_FORMAT, path + ": fewer IDs than PopCount");
		}
		for (uint64_t i = 0; i < n; ++i) {
			const unsigned id = dst[i] & 0x7FFFu;
			if (id < nids)
				++owned[id];
			sat += (dst[i] & kMibfSat) != 0;
		}
		done += n;
	}
	fclose(f);
	const unsigned h = ctx->hd.h;
	ctx->allowed_miss = (ctx->p.frame_matches > h || ctx->hd.seeds.empty())
			? 0 : h - ctx->p.frame_matches;
	ctx->need = ctx->allowed_miss >= h ? 0 : h - ctx->allowed_miss;
	ctx->frame_prob.assign(nids, 0.0);
	for (unsigned id = 0; id < nids; ++id)
		ctx->frame_prob[id] = mibf_frame_prob((double)owned[id] / (double)ctx->hd.m, h, ctx->need);
	ctx->rate_saturated = ctx->hd.pop ? (double)sat / (double)ctx->hd.pop : 0.0;
	return BBT_OK;
}

extern "C" void bbt_mibf_default_params(bbt_mibf_params *p)
{
	if (!p)
		return;
	memset(p, 0, sizeof(*p));
	p->score = pow(10.0, -10.0);  /* BioBloomMICategorizer.cpp:132 */
	p->frame_matches = 1;         /* -a default */
	p->multi_thresh = 1.0;        /* -m default */
	p->streak = 3;                /* -r default */
}

extern "C" unsigned bbt_mibf_min_count(unsigned frame_count, double frame_prob, double score,
		unsigned num_ids)
{
	if (num_ids < 2)
		return 1;
	return mibf_min_count(frame_count, frame_prob, score, num_ids);
}

extern "C" int bbt_mibf_open_host(const char *bf_path, const bbt_mibf_params *params,
		bbt_mibf **out)
{
	if (!out)
		return mibf_fail(nullptr, BBT_ERR_ARG, "bbt_mibf_open_host: out is NULL");
	*out = nullptr;
	bbt_mibf *ctx = new bbt_mibf();
	if (params)
		ctx->p = *params;
	else
		bbt_mibf_default_params(&ctx->p);
	ctx->host_only = true;
	int rc = mibf_load_host(ctx, bf_path, nullptr);
	if (rc) {
		mibf_fail(nullptr, rc, ctx->err);
		delete ctx;
		return rc;
	}
	*out = ctx;
	return BBT_OK;
}

extern "C" int bbt_mibf_format_record(const bbt_mibf *ctx, int out_type, const char *name,
		const char *comment, const char *seq, const char *qual, const bbt_mibf_hit *hits,
		uint32_t n_hits, uint32_t sat_count, char *buf, size_t cap, size_t *len)
{
	if (!ctx || !name || (n_hits && !hits))
		return BBT_ERR_ARG;
	std::string s;
	mibf_format_record(s, ctx->names, out_type, name, comment, seq, qual, hits, n_hits,
			sat_count);
	if (len)
		*len = s.size();
	if (buf && cap) {
		size_t n = std::min(cap - 1, s.size());
		memcpy(buf, s.data(), n);
		buf[n] = 0;
	}
	return BBT_OK;
}

extern "C" const char *bbt_last_error(const bbt_ctx *ctx);

extern "C" const char *bbt_mibf_last_error(const bbt_mibf *ctx)
{
	return ctx ? ctx->err.c_str() : bbt_last_error(nullptr);
}

extern "C" unsigned bbt_mibf_num_ids(const bbt_mibf *ctx)
{
	return ctx ? (unsigned)ctx->names.size() : 0;
}

extern "C" const char *bbt_mibf_id_name(const bbt_mibf *ctx, unsigned id)
{
	return ctx && id < ctx->names.size() ? ctx->names[id].c_str() : nullptr;
}

extern "C" int bbt_mibf_info(const bbt_mibf *ctx, uint64_t *m, unsigned *h, unsigned *k,
		unsigned *n_seeds)
{
	if (!ctx)
		return BBT_ERR_ARG;
	if (m)
		*m = ctx->hd.m;
	if (h)
		*h = ctx->hd.h;
	if (k)
		*k = ctx->hd.k;
	if (n_seeds)
		*n_seeds = (unsigned)ctx->hd.seeds.size();
	return BBT_OK;
}

extern "C" int bbt_mibf_frame_probs(const bbt_mibf *ctx, double *probs, double *rate_saturated)
{
	if (!ctx)
		return BBT_ERR_ARG;
	if (probs)
		memcpy(probs, ctx->frame_prob.data(), ctx->frame_prob.size() * sizeof(double));
	if (rate_saturated)
		*rate_saturated = ctx->rate_saturated;
	return BBT_OK;
}
