/*
 * cli_micategorizer.cpp -- biobloommicategorizer on the B200 path.
 *
 * Same flags, defaults, checks and outputs as the reference CLI
 * (BioBloomCategorizer/BioBloomMICategorizer.cpp:78-341): one record per read
 * (pair) on stdout (TSV, or FASTA / FASTQ with --fa / --fq) and
 * "<prefix>_summary.tsv".  -t and -I are accepted and ignored (the work runs
 * on the GPU); --debug, -d and -n (which the reference leaves unused or
 * debug-only) are refused.  --device selects the GPU.
 */
#include <getopt.h>
#include <sys/stat.h>

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <iostream>
#include <sstream>
#include <string>
#include <vector>

#include "bbt_mibf.h"

using namespace std;

static void usage_exit()
{
	cerr << "Usage: biobloommicategorizer [OPTION]... -f [FILTER] [FILE]...\n"
	        "Usage: biobloommicategorizer [OPTION]... -f [FILTER1] -e [FILE1.fq] [FILE2.fq]\n"
	        "The input format may be FASTA, FASTQ, and compressed with gz. Output will be to\n"
	        "stdout with a summary file outputted to a prefix.\n"
	        "  -p, --prefix=N         Output prefix to use. Otherwise will output to current\n"
	        "                         directory.\n"
	        "  -f, --filter=N         Path of miBF '.bf' file\n"
	        "  -e, --paired_mode      Uses paired-end information.\n"
	        "  -s, --min_FPR=N        Minimum -10*log(FPR) threshold for a match. [100.0]\n"
	        "  -t, --threads=N        Accepted for compatibility (work runs on the GPU).\n"
	        "  -i, --hitOnly          Return only results that hit the filter.\n"
	        "      --fa               Output categorized reads in Fasta output.\n"
	        "      --fq               Output categorized reads in Fastq output.\n"
	        "      --version          Display version information.\n"
	        "  -h, --help             Display this dialog.\n"
	        "  -v, --verbose          Display verbose output\n"
	        "  -I, --interval         Accepted for compatibility.\n"
	        "      --device=N         CUDA device ordinal. [0]\n"
	        "Advanced options:\n"
	        "  -a, --frameMatches=N   Min number seed matches needed in a frame to match [1]\n"
	        "                         Ignored if k-mers used when indexing.\n"
	        "  -m, --multi=N          Multi Match threshold. [1.0]\n"
	        "  -r, --streak=N         Number of additional hits needed to skip classification. [3]\n"
	        "                         Checked against -c but has no effect on the results here:\n"
	        "                         every frame of a read is evaluated.\n"
	        "  -c, --minNoSat=N       Minimum count of non saturated matches. Increasing this value\n"
	        "                         will filter out repetitive or low quality sequences.[0]\n"
	        "  -b, --bestHitAgree     Filters out all matches where best hit is ambiguous because\n"
	        "                         match count metrics do not agree.\n";
	exit(EXIT_SUCCESS);
}

static bool fexists(const string &p)
{
	ifstream f(p.c_str());
	return f.good();
}

template <typename T>
static void parse_or_die(const char *arg, T &v, char opt)
{
	stringstream conv(arg);
	if (!(conv >> v)) {
		cerr << "Error - Invalid parameter! " << opt << ": " << arg << endl;
		exit(EXIT_FAILURE);
	}
}

int main(int argc, char **argv)
{
	bbt_mibf_params p;
	bbt_mibf_default_params(&p);
	int fastq = 0, fasta = 0, tsv = 0, version = 0, debug = 0, verbose = 0;
	bool paired = false, die = false;
	string filter, prefix, refused;
	enum { OPT_DEVICE = 1000 };
	static struct option long_options[] = {
		{"prefix", required_argument, NULL, 'p'},
		{"filter", required_argument, NULL, 'f'},
		{"paired", no_argument, NULL, 'e'},
		{"min_FPR", required_argument, NULL, 's'},
		{"help", no_argument, NULL, 'h'},
		{"interval", required_argument, NULL, 'I'},
		{"threads", required_argument, NULL, 't'},
		{"frameMatches", required_argument, NULL, 'a'},
		{"fq", no_argument, &fastq, 1},
		{"fa", no_argument, &fasta, 1},
		{"tsv", no_argument, &tsv, 1},
		{"hitOnly", no_argument, NULL, 'i'},
		{"version", no_argument, &version, 1},
		{"multi", required_argument, NULL, 'm'},
		{"streak", required_argument, NULL, 'r'},
		{"minNoSat", required_argument, NULL, 'c'},
		{"bestHitAgree", no_argument, NULL, 'b'},
		{"stdout", no_argument, NULL, 'd'},
		{"inverse", no_argument, NULL, 'n'},
		{"debug", no_argument, &debug, 1},
		{"verbose", no_argument, NULL, 'v'},
		{"device", required_argument, NULL, OPT_DEVICE},
		{NULL, 0, NULL, 0}};
	int c, idx = 0;
	while ((c = getopt_long(argc, argv, "p:f:es:hI:t:f:m:r:dnvc:a:bi", long_options, &idx)) !=
			-1) {
		switch (c) {
		case 's': {
			stringstream conv(optarg);
			double raw = 0;
			conv >> raw;
			p.score = pow(10.0, -(raw / 10.0));
			break;
		}
		case 'f': filter = optarg; break;
		case 'p': prefix = optarg; break;
		case 'h': usage_exit(); break;
		case 'I': {
			/* the report interval has no use here, but is parsed as the
			 * reference does, which returns 0 on a bad value
			 * (BioBloomMICategorizer.cpp:187-194) */
			unsigned interval = 0;
			stringstream conv(optarg);
			if (!(conv >> interval)) {
				cerr << "Error - Invalid parameters! I: " << optarg << endl;
				return 0;
			}
			break;
		}
		case 't': {
			/* host threads: parsed and checked as the reference does; the
			 * device does the classification */
			unsigned threads = 0;
			parse_or_die(optarg, threads, 't');
			break;
		}
		case 'e': paired = true; break;
		case 'a': parse_or_die(optarg, p.frame_matches, 'a'); break;
		case 'b': p.best_hit_agree = 1; break;
		case 'v': ++verbose; break;
		case 'r':
			parse_or_die(optarg, p.streak, 'r');
			/* The reference hands -r to MIBFQuerySupport
			 * (MIBFClassifier.hpp:222-225), whose early-exit rule lives
			 * in the btl_bloomfilter submodule, absent from the
			 * reference tree; this implementation evaluates every frame. */
			cerr << "Warning: -r has no effect: every frame of a read is evaluated" << endl;
			break;
		case 'c': parse_or_die(optarg, p.min_nonsat, 'c'); break;
		case 'm': parse_or_die(optarg, p.multi_thresh, 'm'); break;
		case 'd': refused += " -d"; break;
		case 'n': refused += " -n"; break;
		case 'i': p.hit_only = 1; break;
		case OPT_DEVICE: p.device = atoi(optarg); break;
		case '?': die = true; break;
		default: break;
		}
	}
	if (version) {
		cerr << "biobloommicategorizer (bbt-b200) 2.3.4-compatible" << endl;
		exit(EXIT_SUCCESS);
	}
	vector<string> files;
	while (optind < argc)
		files.push_back(argv[optind++]);
	if (paired && files.size() != 2) {
		cerr << "Usage of paired end mode:\n"
		     << "BioBloomCategorizer [OPTION]... -f \"[FILTER1]...\" [FILEPAIR1] [FILEPAIR2]\n"
		     << endl;
		exit(1);
	}
	if (p.streak < p.min_nonsat) {
		cerr << "-r should be greater or equalt to -c" << endl;
		exit(1);
	}
	if (files.empty()) {
		cerr << "Error: Need Input File" << endl;
		die = true;
	}
	if (filter.empty()) {
		cerr << "Error: Need Filter File (-f)" << endl;
		die = true;
	}
	if (die) {
		cerr << "Try '--help' for more information.\n";
		exit(EXIT_FAILURE);
	}
	if (debug)
		refused += " --debug";
	if (!refused.empty()) {
		cerr << "Error: option(s)" << refused << " are not supported by this implementation" << endl;
		exit(EXIT_FAILURE);
	}
	if (prefix.find('/') != string::npos) {
		struct stat sb;
		string dir = prefix.substr(0, prefix.find_last_of('/'));
		if (stat(dir.c_str(), &sb) == 0) {
			if (!S_ISDIR(sb.st_mode)) {
				cerr << "Error: Output folder - file exists with this name. " << dir << endl;
				exit(1);
			}
		} else {
			cerr << "Error: Output folder does not exist. " << dir << endl;
			exit(1);
		}
	}
	int out_type = BBT_MIBF_OUT_TSV;
	if (fasta && fastq) {
		cerr << "Error: fasta (--fa) and fastq (--fq) outputs types cannot be both set" << endl;
		exit(1);
	} else if (fastq) {
		out_type = BBT_MIBF_OUT_FASTQ;
	} else if (fasta) {
		out_type = BBT_MIBF_OUT_FASTA;
	}
	if (!fexists(filter)) {
		cerr << "Error: " + filter + " File cannot be opened" << endl;
		exit(1);
	}
	bbt_mibf *ctx = nullptr;
	if (bbt_mibf_open(filter.c_str(), &p, &ctx) != BBT_OK) {
		cerr << bbt_mibf_last_error(nullptr) << endl;
		exit(1);
	}
	int rc;
	if (paired) {
		rc = bbt_mibf_filter_pair_files(ctx, files[0].c_str(), files[1].c_str(), prefix.c_str(),
				out_type, stdout);
	} else {
		vector<const char *> fp;
		for (const string &f : files)
			fp.push_back(f.c_str());
		rc = bbt_mibf_filter_files(ctx, fp.data(), (int)fp.size(), prefix.c_str(), out_type,
				stdout);
	}
	if (rc != BBT_OK) {
		cerr << "Error: " << bbt_mibf_last_error(ctx) << endl;
		bbt_mibf_close(ctx);
		exit(1);
	}
	bbt_mibf_close(ctx);
	return 0;
}
