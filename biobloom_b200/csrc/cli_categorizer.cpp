/*
 * cli_categorizer.cpp -- biobloomcategorizer on the B200 path.
 *
 * Same flags as the reference CLI (BioBloomCategorizer/BioBloomCategorizer.cpp:
 * 171-205); the option checks (:355-385, 398-442), the score conversion
 * (integer > 1 selects LENGTH scoring, binomial -s as a Phred-scaled FPR,
 * :414-441), the filter existence check (:444-452) and the dispatch over
 * paired / smart-paired / file-list / single-end inputs (:458-532) follow it.
 * Output: "<prefix>_summary.tsv" and, with --read_status FILE, one
 * "<read>\t<category>" line per read (pair).  --fa / --fq (with -g) write the
 * reads of each category to their own files, -d / -n print the first filter's
 * reads (or all others) to stdout; -c, -b and -w select the ordered, best-hit
 * and with-scores modes, -D (with -T, -W) SDUST low-complexity masking.
 */
#include <getopt.h>
#include <sys/stat.h>

#include <cmath>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iostream>
#include <sstream>
#include <string>
#include <vector>

#include "bbt.h"

using namespace std;

static void usage_exit(int code)
{
	cerr << "Usage: biobloomcategorizer [OPTION]... -f \"[FILTER1]...\" [FILE]...\n"
	        "biobloomcategorizer [OPTION]... -e -f \"[FILTER1]...\" [FILE1.fq] [FILE2.fq]\n"
	        "Categorize Sequences. The input format may be FASTA, FASTQ, and compressed gz.\n"
	        "\n"
	        "  -p, --prefix=N         Output prefix to use. Otherwise will output to current\n"
	        "                         directory.\n"
	        "  -f, --filter_files=N   List of filter files to use. Required option.\n"
	        "  -e, --paired_mode      Uses paired-end information.\n"
	        "  -i, --inclusive        If one paired read matches, both reads will be included\n"
	        "                         in the filter.\n"
	        "  -s, --score=N          Score threshold for matching: a floating point score\n"
	        "                         between 0 and 1, or a positive integer minimum match\n"
	        "                         length in bases. [0.15]\n"
	        "  -t, --threads=N        Accepted for compatibility (work runs on the GPU).\n"
	        "  -g, --gz_output        Outputs all output files in compressed gzip.\n"
	        "      --fa               Output categorized reads in Fasta files.\n"
	        "      --fq               Output categorized reads in Fastq files.\n"
	        "  -d, --stdout_filter    Outputs all matching reads to stdout for the first\n"
	        "                         filter listed by -f.\n"
	        "  -n, --inverse          Inverts the output of -d (everything but first filter).\n"
	        "  -l, --file_list=N      A file of list of file pairs to run in parallel.\n"
	        "  -c, --ordered          Use ordered filtering. Order of filters matters\n"
	        "                         (filters listed first have higher priority).\n"
	        "  -b, --best_hit         Places reads into the filter with the best score\n"
	        "                         (no minimum threshold).\n"
	        "  -w, --with_score       Output multimatches with scores in the order of filter.\n"
	        "  -S, --score_type=N     harmonic or binomial scoring.\n"
	        "  -r, --streak=N         Hits tiling in second pass needed to jump several tiles\n"
	        "                         upon a miss. [3]\n"
	        "  -D, --dust             Filter using dust.\n"
	        "  -T, --T_dust           T parameter for dust. [20]\n"
	        "  -W, --window_dust      Window size for dust. [64]\n"
	        "  -I, --interval         Accepted for compatibility.\n"
	        "      --read_status=F    Write one '<read>\\t<category>' line per read to F.\n"
	        "      --device=N         CUDA device ordinal. [0]\n"
	        "      --devices=LIST     Comma-separated CUDA device ordinals: the filters are\n"
	        "                         loaded on each and the reads split across them.\n"
	        "  -v, --version          Display version information.\n"
	        "  -h, --help             Display this dialog.\n";
	exit(code);
}

static vector<string> split_ws(const string &s)
{
	vector<string> out;
	stringstream in(s);
	string t;
	while (in >> t)
		out.push_back(t);
	return out;
}

static bool fexists(const string &p)
{
	ifstream f(p.c_str());
	return f.good();
}

int main(int argc, char **argv)
{
	bbt_params p;
	bbt_default_params(&p);
	string filters, prefix, read_status, postfix;
	double binomial_score = 100; /* -s for binomial scoring, BioBloomCategorizer.cpp:168 */
	bool paired = false, die = false, to_stdout = false, inverse = false, collab = false;
	int mode = BBT_MODE_STD;
	string file_list;
	bool dust = false;
	unsigned dust_T = 20, dust_W = 64; /* Common/Options.cpp:36-38 */
	int fastq = 0, fasta = 0, verbose = 0;
	int device = 0;
	vector<int> devices;
	enum { OPT_READ_STATUS = 1000, OPT_DEVICE, OPT_DEVICES };
	static struct option long_options[] = {
		{"prefix", required_argument, NULL, 'p'},
		{"filter_files", required_argument, NULL, 'f'},
		{"paired_mode", no_argument, NULL, 'e'},
		{"inclusive", no_argument, NULL, 'i'},
		{"score", required_argument, NULL, 's'},
		{"help", no_argument, NULL, 'h'},
		{"interval", required_argument, NULL, 'I'},
		{"threads", required_argument, NULL, 't'},
		{"gz_output", no_argument, NULL, 'g'},
		{"fq", no_argument, &fastq, 1},
		{"fa", no_argument, &fasta, 1},
		{"file_list", required_argument, NULL, 'l'},
		{"version", no_argument, NULL, 'v'},
		{"multi", required_argument, NULL, 'm'},
		{"streak", required_argument, NULL, 'r'},
		{"min_hit_only", no_argument, NULL, 'o'},
		{"ordered", no_argument, NULL, 'c'},
		{"stdout_filter", no_argument, NULL, 'd'},
		{"inverse", no_argument, NULL, 'n'},
		{"best_hit", no_argument, NULL, 'b'},
		{"with_score", no_argument, NULL, 'w'},
		{"score_type", required_argument, NULL, 'S'},
		{"verbose", no_argument, &verbose, 1},
		{"dust", no_argument, NULL, 'D'},
		{"T_dust", required_argument, NULL, 'T'},
		{"window_dust", required_argument, NULL, 'W'},
		{"read_status", required_argument, NULL, OPT_READ_STATUS},
		{"device", required_argument, NULL, OPT_DEVICE},
		{"devices", required_argument, NULL, OPT_DEVICES},
		{NULL, 0, NULL, 0}};
	int c, idx = 0;
	while ((c = getopt_long(argc, argv, "f:p:hegl:vs:r:t:cdiwI:nm:S:bDT:W:", long_options,
			&idx)) != -1) {
		switch (c) {
		case 's': {
			stringstream conv(optarg);
			conv >> p.score;
			binomial_score = p.score;
			break;
		}
		case 'S':
			if (strcmp(optarg, "harmonic") == 0) {
				p.scoring = BBT_SCORE_HARMONIC;
			} else if (strcmp(optarg, "binomial") == 0) {
				p.scoring = BBT_SCORE_BINOMIAL;
			} else {
				cerr << "scoring method not recognized. Valid strings: harmonic or binomial"
				     << endl;
				die = true;
			}
			break;
		case 'f': filters = optarg; break;
		case 'p': prefix = optarg; break;
		case 'h': usage_exit(EXIT_SUCCESS); break;
		case 'e': paired = true; break;
		case 'i': p.inclusive = 1; break;
		case 'I': {
			/* the report interval has no use here, but is parsed as the
			 * reference does, which returns 0 on a bad value
			 * (BioBloomCategorizer.cpp:227-234) */
			unsigned interval = 0;
			stringstream conv(optarg);
			if (!(conv >> interval)) {
				cerr << "Error - Invalid parameters! I: " << optarg << endl;
				return 0;
			}
			break;
		}
		case 't': {
			/* host threads: parsed and checked as the reference does
			 * (BioBloomCategorizer.cpp:243-250); the device classifies */
			unsigned threads = 0;
			stringstream conv(optarg);
			if (!(conv >> threads)) {
				cerr << "Error - Invalid parameter! t: " << optarg << endl;
				exit(EXIT_FAILURE);
			}
			break;
		}
		case 'm': break;
		case 'r': {
			stringstream conv(optarg);
			if (!(conv >> p.streak_threshold)) {
				cerr << "Error - Invalid parameter! r: " << optarg << endl;
				exit(EXIT_FAILURE);
			}
			break;
		}
		case 'v':
			cerr << "biobloomcategorizer (bbt-b200) 2.3.4-compatible\n" << endl;
			exit(EXIT_SUCCESS);
		case 'g': postfix = ".gz"; break;
		case 'd': to_stdout = true; break;
		case 'n': inverse = true; break;
		case 'l': {
			stringstream conv(optarg);
			if (!(conv >> file_list)) {
				cerr << "Error - Invalid set of bloom filter parameters! l: " << optarg << endl;
				return 0;
			}
			break;
		}
		case 'c': collab = true; break;
		case 'w':
			if (mode == BBT_MODE_STD) {
				mode = BBT_MODE_SCORES;
			} else {
				cerr << "Filter scoring modes cannot be mixed with score mode" << endl;
				die = true;
			}
			break;
		case 'b':
			if (mode == BBT_MODE_STD) {
				mode = BBT_MODE_BESTHIT;
			} else {
				cerr << "Filter scoring modes cannot be mixed with best hit mode" << endl;
				die = true;
			}
			break;
		case 'D': dust = true; break;
		case 'T': {
			stringstream conv(optarg);
			conv >> dust_T;
			break;
		}
		case 'W': {
			stringstream conv(optarg);
			conv >> dust_W;
			break;
		}
		case 'o': break; /* --min_hit_only: accepted and ignored, as upstream */
		case OPT_READ_STATUS: read_status = optarg; break;
		case OPT_DEVICE: device = atoi(optarg); break;
		case OPT_DEVICES: {
			stringstream ss(optarg);
			string tok;
			while (getline(ss, tok, ','))
				if (!tok.empty())
					devices.push_back(atoi(tok.c_str()));
			break;
		}
		case '?': die = true; break;
		default: break;
		}
	}
	vector<string> files;
	while (optind < argc)
		files.push_back(argv[optind++]);
	vector<string> paths = split_ws(filters);
	bool smart = false;
	if (paired) {
		if (files.size() == 1) {
			smart = true;
		} else if (files.size() != 2 && file_list.empty()) {
			cerr << "Usage of paired end mode:\n"
			        "BioBloomCategorizer [OPTION]... -f \"[FILTER1]...\" [FILEPAIR1] [FILEPAIR2]\n"
			        "or BioBloomCategorizer [OPTION]... -f \"[FILTER1]...\" [SMARTPAIR]\n"
			     << endl;
			die = true;
		}
	}
	if (!file_list.empty() && !files.empty()) {
		cerr << "--file_list (-l) cannot be used with read files in specified in arguments"
		     << endl;
		die = true;
	}
	if (files.empty() && file_list.empty()) {
		cerr << "Error: Need Input File" << endl;
		die = true;
	}
	if (paths.empty()) {
		cerr << "Error: Need Filter File (-f)" << endl;
		die = true;
	}
	if (die) {
		cerr << "Try '--help' for more information.\n";
		exit(EXIT_FAILURE);
	}
	/* the output folder, then the output type, in the reference's order
	 * (BioBloomCategorizer.cpp:50-63,390-405) */
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
	string out_type;
	if (fasta && fastq) {
		cerr << "Error: fasta (--fa) and fastq (--fq) outputs types cannot be both set" << endl;
		exit(1);
	} else if (fastq) {
		out_type = "fq";
	} else if (fasta) {
		out_type = "fa";
	}
	if (paired && !file_list.empty() && !out_type.empty()) {
		/* the reference dereferences the empty input-file list here */
		cerr << "Error: --file_list (-l) with paired-end mode does not write read files" << endl;
		exit(EXIT_FAILURE);
	}
	if (mode == BBT_MODE_SCORES && out_type.empty()) {
		cerr << "Error: -w option cannot be used without output method" << endl;
		exit(EXIT_FAILURE);
	}
	if (mode == BBT_MODE_BESTHIT) {
		cerr << "Best Hit mode (no minimum threshold)" << endl;
	} else if (p.scoring == BBT_SCORE_BINOMIAL) {
		/* BioBloomCategorizer.cpp:418-421 */
		p.score = pow(10.0, -(binomial_score / 10.0));
		cerr << "FPR of a match: " << p.score << endl;
	} else {
		unsigned match_len = (unsigned)p.score;
		if (match_len > 1) {
			p.score = match_len;
			p.scoring = BBT_SCORE_LENGTH;
			cerr << "Min match length threshold: " << match_len << " bp" << endl;
		} else {
			cerr << "Min score threshold: " << p.score << endl;
		}
		if (p.score < 0) {
			cerr << "Error - s must be a positive integer or a floating point between 0 and 1."
			     << endl;
			exit(EXIT_FAILURE);
		}
	}
	for (const string &f : paths) {
		if (!fexists(f)) {
			cerr << "Error: " + f + " File cannot be opened" << endl;
			exit(EXIT_FAILURE);
		}
	}
	p.device = device;
	vector<const char *> cp;
	for (const string &f : paths)
		cp.push_back(f.c_str());
	cerr << "Starting to Load Filters." << endl;
	bbt_ctx *ctx = nullptr;
	const int orc = devices.empty()
			? bbt_open(cp.data(), (int)cp.size(), &p, &ctx)
			: bbt_open_devices(cp.data(), (int)cp.size(), &p, devices.data(),
					(int)devices.size(), &ctx);
	if (orc != BBT_OK) {
		cerr << "Error: " << bbt_last_error(nullptr) << endl;
		exit(1);
	}
	for (int i = 0; i < bbt_num_filters(ctx); ++i)
		cerr << "Loaded Filter: " << bbt_filter_id(ctx, i) << endl;
	cerr << "Filter Loading Complete." << endl;
	if (collab) {
		/* BioBloomClassifier::setOrderedFilter (BioBloomClassifier.h:67-75) */
		if (mode == BBT_MODE_BESTHIT) {
			cerr << "Best Hit mode and Ordered mode detected. Not yet supported." << endl;
			bbt_close(ctx);
			exit(1);
		}
		mode = BBT_MODE_ORDERED;
	}
	bbt_set_mode(ctx, mode);
	if (dust && bbt_set_dust(ctx, 1, dust_T, dust_W) != BBT_OK) {
		cerr << "Error: " << bbt_last_error(ctx) << endl;
		bbt_close(ctx);
		exit(1);
	}
	int rc = BBT_OK;
	const char *rs = read_status.empty() ? nullptr : read_status.c_str();
	if (to_stdout)
		bbt_set_stdout(ctx, 1, inverse ? 1 : 0);
	/* the list file: whitespace-separated first (and second) file per line */
	vector<string> list1, list2;
	if (!file_list.empty()) {
		ifstream lf(file_list.c_str());
		if (!lf.is_open() && paired) {
			cout << "Unable to open file";
			bbt_close(ctx);
			return 0;
		}
		string line;
		while (getline(lf, line)) {
			stringstream ss(line);
			string a, b;
			ss >> a;
			ss >> b;
			list1.push_back(a);
			list2.push_back(b);
		}
		cerr << "Using file list" << endl;
	}
	auto cstrs = [](const vector<string> &v) {
		vector<const char *> out;
		for (const string &f : v)
			out.push_back(f.c_str());
		return out;
	};
	if (paired) {
		if (!out_type.empty()) {
			rc = smart ? bbt_filter_smart_pairs_print(ctx, files[0].c_str(), prefix.c_str(),
						out_type.c_str(), postfix.c_str(), rs)
			           : bbt_filter_pair_files_print(ctx, files[0].c_str(), files[1].c_str(),
						prefix.c_str(), out_type.c_str(), postfix.c_str(), rs);
		} else if (smart) {
			rc = bbt_filter_smart_pairs(ctx, files[0].c_str(), prefix.c_str(), rs);
		} else if (!file_list.empty()) {
			vector<const char *> a = cstrs(list1), b = cstrs(list2);
			if (a.empty()) {
				cerr << "Error: the file list holds no files" << endl;
				rc = BBT_ERR_ARG;
			} else {
				rc = bbt_filter_pair_file_lists(ctx, a.data(), b.data(), (int)a.size(),
						prefix.c_str(), rs);
			}
		} else {
			rc = bbt_filter_pair_files(ctx, files[0].c_str(), files[1].c_str(), prefix.c_str(), rs);
		}
	} else {
		const vector<string> &in = file_list.empty() ? files : list1;
		vector<const char *> fp = cstrs(in);
		if (fp.empty()) {
			cerr << "Error: the file list holds no files" << endl;
			rc = BBT_ERR_ARG;
		} else {
			rc = out_type.empty()
					? bbt_filter_files(ctx, fp.data(), (int)fp.size(), prefix.c_str(), rs)
					: bbt_filter_files_print(ctx, fp.data(), (int)fp.size(), prefix.c_str(),
							out_type.c_str(), postfix.c_str(), rs);
		}
	}
	if (rc != BBT_OK) {
		cerr << "Error: " << bbt_last_error(ctx) << endl;
		bbt_close(ctx);
		exit(1);
	}
	bbt_close(ctx);
	return 0;
}
