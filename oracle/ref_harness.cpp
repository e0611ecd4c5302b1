/*
 * ref_harness.cpp -- drives the reference's own classification code
 * (compiled from the reference sources by oracle/Makefile into oracle/_ref).
 * TEST INFRASTRUCTURE ONLY.
 *
 *   ref_harness hits  SCORE STREAK FILTER.bf[,FILTER.bf...] READS [READS2]
 *       For every read (pair), prints one line "<name>\t<hits>" where hits is
 *       the comma-separated list of filter indices whose
 *       SeqEval::evalRead (Common/SeqEval.h:493-524) accepted the read
 *       (for pairs: "<hits1>|<hits2>").  Then prints "#SUMMARY" and the
 *       ResultsManager summary text (ResultsManager.hpp:191-237), computed
 *       by the reference's own ResultsManager.
 *   ref_harness scores METHOD STREAK FILTER.bf[,FILTER.bf...] READS
 *       For every read, prints "<name>\t<s0>,<s1>,..." where s_f is
 *       SeqEval::evalScore (Common/SeqEval.h:534-560) of the read against
 *       filter f under METHOD (simple, length, harmonic or binomial), as the
 *       16 hex digits of the double's bits.
 *   ref_harness dust T W READS
 *       For every read, prints "<name>\t<start>-<finish>,..." with the
 *       intervals the reference's sdust (Common/sdust.c) masks.
 *   ref_harness time  SCORE STREAK THREADS INCLUSIVE PREFIX FILTERS READS [READS2]
 *       (BBT_MODE = ordered / besthit / scores selects a filtering mode)
 *       Builds a BioBloomClassifier (BioBloomClassifier.cpp:21-28; filter
 *       load not timed), then times filter()/filterPair() and prints one JSON
 *       line with the wall time, reads and cores used.
 *
 * A score > 1 selects LENGTH scoring, as BioBloomCategorizer.cpp:423-430 does.
 * The environment variable BBT_DUST="T,W" turns on DUST masking (-D -T T -W W,
 * BioBloomCategorizer.cpp:323-337) for hits and scores.
 */
#include "BioBloomClassifier.h"
#include "ResultsManager.hpp"
#include "Common/Options.h"
#include "Common/SeqEval.h"
#include "Common/sdust.h"
#include <omp.h>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <sstream>
#include <string>
#include <vector>

using namespace std;

static vector<string> split_commas(const string &s)
{
	vector<string> out;
	string cur;
	stringstream in(s);
	while (getline(in, cur, ','))
		if (!cur.empty())
			out.push_back(cur);
	return out;
}

/* -s as BioBloomCategorizer.cpp:414-441 reads it; the scoring method (-S)
 * comes from the environment variable BBT_SCORING ("harmonic" or
 * "binomial"; unset = simple). */
static void set_score(double score)
{
	const char *m = getenv("BBT_SCORING");
	std::string method = m ? m : "";
	if (method == "binomial") {
		opt::scoringMethod = opt::BINOMIAL;
		opt::score = pow(10.0, -(score / 10.0));
		return;
	}
	if (method == "harmonic")
		opt::scoringMethod = opt::HARMONIC;
	opt::score = score;
	unsigned matchLen = (unsigned)score;
	if (matchLen > 1) {
		opt::score = (unsigned)matchLen;
		opt::scoringMethod = opt::LENGTH;
	}
}

static void set_dust()
{
	const char *d = getenv("BBT_DUST");
	if (!d || !*d)
		return;
	opt::dust = true;
	unsigned T = 20, W = 64;
	if (sscanf(d, "%u,%u", &T, &W) >= 1) {
		opt::dustT = T;
		opt::dustWindow = W;
	}
}

static string join(const vector<unsigned> &v)
{
	string s;
	for (size_t i = 0; i < v.size(); ++i) {
		if (i)
			s += ",";
		s += to_string(v[i]);
	}
	return s;
}

static int mode_hits(int argc, char **argv)
{
	if (argc < 6) {
		fprintf(stderr, "usage: ref_harness hits SCORE STREAK FILTERS READS [READS2]\n");
		return 2;
	}
	set_score(atof(argv[2]));
	set_dust();
	opt::streakThreshold = (unsigned)atoi(argv[3]);
	vector<string> paths = split_commas(argv[4]);
	vector<BloomFilter *> filters;
	vector<string> ids;
	for (size_t i = 0; i < paths.size(); ++i) {
		filters.push_back(new BloomFilter(paths[i]));
		BloomFilterInfo info(paths[i].substr(0, paths[i].size() - 2) + "txt");
		ids.push_back(info.getFilterID());
	}
	bool paired = argc > 6;
	ResultsManager<unsigned> res(ids, false);
	gzFile fp1 = gzopen(argv[5], "r");
	gzFile fp2 = paired ? gzopen(argv[6], "r") : Z_NULL;
	if (fp1 == Z_NULL || (paired && fp2 == Z_NULL)) {
		fprintf(stderr, "cannot open reads\n");
		return 1;
	}
	kseq_t *k1 = kseq_init(fp1);
	kseq_t *k2 = paired ? kseq_init(fp2) : NULL;
	/* records first, then SeqEval::evalRead over them on all threads (each
	 * call reads only its filter and its sequence), output in file order */
	vector<string> names, seqs1, seqs2;
	for (;;) {
		int l1 = kseq_read(k1);
		int l2 = paired ? kseq_read(k2) : 0;
		if (l1 < 0 || l2 < 0)
			break;
		names.push_back(k1->name.s);
		seqs1.push_back(string(k1->seq.s, l1));
		if (paired)
			seqs2.push_back(string(k2->seq.s, l2));
	}
	const size_t total = names.size();
	vector<vector<unsigned> > hits1(total), hits2(paired ? total : 0);
#pragma omp parallel for schedule(dynamic, 256)
	for (long i = 0; i < (long)total; ++i) {
		for (unsigned f = 0; f < filters.size(); ++f) {
			if (SeqEval::evalRead(seqs1[i], *filters[f], opt::score))
				hits1[i].push_back(f);
			if (paired && SeqEval::evalRead(seqs2[i], *filters[f], opt::score))
				hits2[i].push_back(f);
		}
	}
	for (size_t i = 0; i < total; ++i) {
		if (paired) {
			res.updateSummaryData(hits1[i], hits2[i]);
			printf("%s\t%s|%s\n", names[i].c_str(), join(hits1[i]).c_str(),
					join(hits2[i]).c_str());
		} else {
			res.updateSummaryData(hits1[i]);
			printf("%s\t%s\n", names[i].c_str(), join(hits1[i]).c_str());
		}
	}
	printf("#SUMMARY\n%s", res.getResultsSummary(total).c_str());
	kseq_destroy(k1);
	gzclose(fp1);
	if (paired) {
		kseq_destroy(k2);
		gzclose(fp2);
	}
	return 0;
}

static int mode_scores(int argc, char **argv)
{
	if (argc < 6) {
		fprintf(stderr, "usage: ref_harness scores METHOD STREAK FILTERS READS\n");
		return 2;
	}
	string method = argv[2];
	if (method == "length")
		opt::scoringMethod = opt::LENGTH;
	else if (method == "harmonic")
		opt::scoringMethod = opt::HARMONIC;
	else if (method == "binomial")
		opt::scoringMethod = opt::BINOMIAL;
	else
		opt::scoringMethod = opt::SIMPLE;
	set_dust();
	opt::streakThreshold = (unsigned)atoi(argv[3]);
	vector<string> paths = split_commas(argv[4]);
	vector<BloomFilter *> filters;
	for (size_t i = 0; i < paths.size(); ++i)
		filters.push_back(new BloomFilter(paths[i]));
	gzFile fp = gzopen(argv[5], "r");
	if (fp == Z_NULL) {
		fprintf(stderr, "cannot open reads\n");
		return 1;
	}
	kseq_t *k = kseq_init(fp);
	for (int l; (l = kseq_read(k)) >= 0;) {
		string seq(k->seq.s, l);
		printf("%s\t", k->name.s);
		for (unsigned f = 0; f < filters.size(); ++f) {
			double v = SeqEval::evalScore(seq, *filters[f]);
			unsigned long long bits;
			memcpy(&bits, &v, sizeof bits);
			printf("%s%016llx", f ? "," : "", bits);
		}
		printf("\n");
	}
	kseq_destroy(k);
	gzclose(fp);
	return 0;
}

static int mode_dust(int argc, char **argv)
{
	if (argc < 5) {
		fprintf(stderr, "usage: ref_harness dust T W READS\n");
		return 2;
	}
	int T = atoi(argv[2]), W = atoi(argv[3]);
	gzFile fp = gzopen(argv[4], "r");
	if (fp == Z_NULL) {
		fprintf(stderr, "cannot open reads\n");
		return 1;
	}
	kseq_t *k = kseq_init(fp);
	for (int l; (l = kseq_read(k)) >= 0;) {
		int n = 0;
		uint64_t *iv = sdust(0, (const uint8_t *)k->seq.s, l, T, W, &n);
		printf("%s\t", k->name.s);
		for (int i = 0; i < n; ++i)
			printf("%s%u-%u", i ? "," : "", (unsigned)(iv[i] >> 32), (unsigned)iv[i]);
		printf("\n");
		free(iv);
	}
	kseq_destroy(k);
	gzclose(fp);
	return 0;
}

static size_t count_records(const char *path)
{
	gzFile fp = gzopen(path, "r");
	if (fp == Z_NULL)
		return 0;
	kseq_t *k = kseq_init(fp);
	size_t n = 0;
	while (kseq_read(k) >= 0)
		++n;
	kseq_destroy(k);
	gzclose(fp);
	return n;
}

static int mode_time(int argc, char **argv)
{
	if (argc < 9) {
		fprintf(stderr, "usage: ref_harness time SCORE STREAK THREADS INCLUSIVE PREFIX FILTERS READS [READS2]\n");
		return 2;
	}
	set_score(atof(argv[2]));
	set_dust();
	opt::streakThreshold = (unsigned)atoi(argv[3]);
	int threads = atoi(argv[4]);
	if (threads > 0)
		omp_set_num_threads(threads);
	opt::threads = (unsigned)(threads > 0 ? threads : omp_get_max_threads());
	bool inclusive = atoi(argv[5]) != 0;
	opt::outputPrefix = argv[6];
	vector<string> paths = split_commas(argv[7]);
	bool paired = argc > 9;
	size_t reads = count_records(argv[8]);
	BioBloomClassifier bbc(paths, opt::score, opt::outputPrefix, opt::filePostfix);
	if (inclusive)
		bbc.setInclusive();
	/* BBT_MODE: the filtering mode (-c, -b, -w; BioBloomCategorizer.cpp:
	 * 276-318, 460-464) */
	const char *md = getenv("BBT_MODE");
	const string mode = md ? md : "";
	if (mode == "ordered")
		bbc.setOrderedFilter();
	else if (mode == "besthit")
		opt::mode = opt::BESTHIT;
	else if (mode == "scores")
		opt::mode = opt::SCORES;
	double t0 = omp_get_wtime();
	if (paired)
		bbc.filterPair(argv[8], argv[9]);
	else
		bbc.filter(vector<string>(1, argv[8]));
	double t1 = omp_get_wtime();
	printf("{\"seconds\": %.6f, \"records\": %zu, \"paired\": %d, \"threads\": %u}\n",
			t1 - t0, reads, paired ? 1 : 0, opt::threads);
	return 0;
}

int main(int argc, char **argv)
{
	if (argc < 2) {
		fprintf(stderr, "usage: ref_harness hits|time ...\n");
		return 2;
	}
	string mode = argv[1];
	if (mode == "hits")
		return mode_hits(argc, argv);
	if (mode == "time")
		return mode_time(argc, argv);
	if (mode == "scores")
		return mode_scores(argc, argv);
	if (mode == "dust")
		return mode_dust(argc, argv);
	fprintf(stderr, "unknown mode %s\n", argv[1]);
	return 2;
}
