/*
 * mibf_ctx.hpp -- the multi-index Bloom filter context behind bbt_mibf.h, and
 * the host-side pieces shared by the device code, the file pipeline and the
 * maker.
 */
#ifndef BBT_MIBF_CTX_HPP
#define BBT_MIBF_CTX_HPP

#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>
#include <string>
#include <vector>

#include "bbt_mibf.h"

namespace bbt {

constexpr unsigned kMibfMaxSeeds = 16;
constexpr unsigned kMibfMaxK = 32;
/* IDs (target names + the empty ID 0): up to kMibfSmemIds the query kernel
 * tallies a read in shared memory, above it in per-warp tables in global
 * memory; IDs are 15-bit (the top bit of a slot is the saturation flag), as
 * in the reference (BioBloomMaker/MIBFGen.hpp:112-118). */
constexpr unsigned kMibfSmemIds = 1024;
constexpr unsigned kMibfMaxIds = 32768;
/* resident blocks per SM of the query kernel with global tally tables (each
 * warp owns a 24 * num_ids byte table) */
constexpr int kMibfBigBlocksPerSm = 2;
constexpr uint16_t kMibfSat = 0x8000u;

/* Header of a "<p>.bf" miBF file. */
struct MibfHeader {
	uint64_t m = 0;
	unsigned h = 0;
	unsigned k = 0;
	unsigned id_width = 16;
	uint64_t pop = 0;
	std::vector<std::string> seeds;
};

/* Parse the text header of an open "<p>.bf"; leaves the stream at the IDs.
 * Returns an empty string or an error message. */
std::string read_mibf_header(FILE *f, MibfHeader &h);
int write_mibf_header(FILE *f, const MibfHeader &h);

/* "<p>_ids.txt" of "<p>.bf" (MIBFClassifier.hpp:52-53). */
std::string mibf_ids_path(const std::string &bf_path);
/* "<p>.sdsl" of "<p>.bf". */
std::string mibf_sdsl_path(const std::string &bf_path);

/* m_fullIDs: "repeat", then the second field of each ID-file line, in order
 * (MIBFClassifier.hpp:64-77). */
bool read_mibf_names(const std::string &path, std::vector<std::string> &names);

/* P(at least need of h values hit an ID) for per-value probability p. */
double mibf_frame_prob(double p, unsigned h, unsigned need);
/* Binomial(n, p): smallest x with P(X > x) <= q, from the top of the tail. */
unsigned binom_upper_quantile(unsigned n, double p, double q);
unsigned mibf_min_count(unsigned frame_count, double frame_prob, double score, unsigned num_ids);

/* Per-value seed tables of the query and build kernels: for seed s, position
 * j < k and base code c, {rol(seed(c), k-1-j), rol(seed_rc(c), j)} when j is a
 * care position of s, else {0, 0}; 32 positions per seed. */
std::vector<unsigned long long> mibf_seed_tables(const std::vector<std::string> &seeds,
		unsigned k);

/* summary.tsv text over `names` (ResultsManager::getResultsSummary). */
std::string mibf_summary_text(const std::vector<std::string> &names,
		const std::vector<uint64_t> &counts, uint64_t reads);

/* One output record (formatOutStr, MIBFClassifier.hpp:675-736). */
void mibf_format_record(std::string &out, const std::vector<std::string> &names, int out_type,
		const char *name, const char *comment, const char *seq, const char *qual,
		const bbt_mibf_hit *hits, uint32_t n_hits, uint32_t sat_count);

} // namespace bbt

struct bbt_mibf {
	std::string err;
	bbt_mibf_params p;
	bbt::MibfHeader hd;
	std::vector<std::string> names;      /* m_fullIDs */
	std::vector<double> frame_prob;      /* m_perFrameProb */
	double rate_saturated = 0;
	unsigned allowed_miss = 0, need = 0;
	bool host_only = false;
	/* device state */
	int dev = 0;
	int num_sms = 0;
	cudaStream_t stream = nullptr, h2d = nullptr, d2h = nullptr;
	uint4 *d_blocks = nullptr;            /* 32-byte rank blocks */
	unsigned long long *d_super = nullptr; /* rank at each superblock start */
	uint16_t *d_ids = nullptr;
	uint16_t *d_dense = nullptr;          /* dense ID map (one entry per bit), or null */
	unsigned long long *d_tables = nullptr;
	unsigned long long *d_counts = nullptr;
	unsigned long long *d_work = nullptr;
	unsigned int *d_flags = nullptr;       /* [0] result overflow */
	unsigned long long *d_stat = nullptr;  /* frames, probes, hits of the last batch */
	unsigned long long *d_gtally = nullptr; /* more than kMibfSmemIds IDs: per-warp tallies */
	uint64_t gtally_warps = 0;
	/* minCount rows, frame count -> num_ids entries; host copy and device copy */
	std::mutex mc_mu;
	std::vector<uint32_t> h_minc;
	std::vector<uint8_t> minc_have;
	uint32_t *d_minc = nullptr;
	uint32_t minc_rows = 0;               /* rows allocated on the device */
	/* host-batch results on the device */
	bbt_mibf_hit *d_hits = nullptr;
	uint32_t *d_nhits = nullptr, *d_sat = nullptr;
	uint64_t res_cap_reads = 0;
	uint32_t res_cap_hits = 0;
	unsigned int *d_fcmax = nullptr;
	/* host-batch pipeline: two chunk slots, each with its chunk's bases and
	 * rebased offsets on the device and the offsets in pinned memory */
	uint8_t *c_seq[2][2] = {{nullptr, nullptr}, {nullptr, nullptr}};
	uint32_t *c_valid[2][2] = {{nullptr, nullptr}, {nullptr, nullptr}}; /* packed batches */
	uint64_t *c_off[2][2] = {{nullptr, nullptr}, {nullptr, nullptr}};
	uint64_t *h_coff[2][2] = {{nullptr, nullptr}, {nullptr, nullptr}};
	uint64_t c_bases_cap = 0, c_reads_cap = 0;
	cudaEvent_t c_copied[2] = {nullptr, nullptr}, c_computed[2] = {nullptr, nullptr};
	uint64_t reads_seen = 0;
	cudaEvent_t ev0 = nullptr, ev1 = nullptr;
	double last_kernel_ms = 0;
	/* bucketed query (dense layout, mibf.cu): settings, then the scratch of
	 * one call (frame offsets, offset samples, packed bases, frame validity
	 * bits, resolved entries, the request pool, per-(bucket, block) counts
	 * and first slots, per-block totals, scan scratch) */
	int bk_mode = 0;                      /* 0 off, 1 on, 2 large batches on large maps */
	uint32_t bk_bshift = 23;              /* bucket of 2^23 entries (16 MB) */
	uint64_t bk_max_frames = 1ull << 30;  /* frames per sub-batch */
	uint64_t *d_bk_fo = nullptr, *h_bk_samples = nullptr, *d_bk_samples = nullptr;
	uint64_t bk_fo_cap = 0, bk_samples_cap = 0;
	uint32_t *d_bk_codes[2] = {nullptr, nullptr}, *d_bk_cvalid[2] = {nullptr, nullptr};
	uint64_t bk_codes_cap[2] = {0, 0}, bk_cvalid_cap[2] = {0, 0};
	uint32_t *d_bk_valid = nullptr;
	uint16_t *d_bk_e = nullptr;
	uint32_t *d_bk_off = nullptr;
	uint16_t *d_bk_slot = nullptr, *d_bk_res = nullptr;
	uint32_t *d_bk_cnt = nullptr, *d_bk_loc = nullptr, *d_bk_btot = nullptr;
	uint64_t bk_valid_cap = 0, bk_e_cap = 0, bk_off_cap = 0, bk_slot_cap = 0, bk_res_cap = 0;
	uint64_t bk_cnt_cap = 0, bk_loc_cap = 0, bk_btot_cap = 0;
	void *d_bk_tmp = nullptr;
	size_t bk_tmp_cap = 0;
};

namespace bbt {
int mibf_fail(bbt_mibf *ctx, int code, const std::string &msg);

/* Per-stream scratch for concurrent miBF classification (serving engine). */
struct MibfScratch {
	unsigned long long *work = nullptr;
	unsigned long long *counts = nullptr; /* a batch's summary counters */
	unsigned long long *stat = nullptr;
	unsigned int *flags = nullptr;
	unsigned long long *gtally = nullptr;  /* per-warp tally tables (many IDs) */
	uint64_t gtally_warps = 0;
};
int mibf_scratch_init(bbt_mibf *ctx, MibfScratch &sc);
void mibf_scratch_free(MibfScratch &sc);
/* Allocate minCount rows for frame counts below `rows` up front, so that later
 * requests only fill rows and never move the table under running kernels. */
int mibf_reserve_rows(bbt_mibf *ctx, uint32_t rows);
/* Make the minCount rows of these reads (host offsets) present on the device
 * (computed and copied under the context's lock, complete when it returns). */
int mibf_rows_for(bbt_mibf *ctx, const uint64_t *off, const uint64_t *off2, uint64_t n);
/* Classify n reads (pairs) on the device on stream s with this scratch; the
 * batch's summary is committed unless a read overflowed max_hits, which sets
 * sc.flags[0] (read it after the stream completes). */
int mibf_classify_slot(bbt_mibf *ctx, uint64_t n, const uint8_t *seq, const uint64_t *off,
		const uint8_t *seq2, const uint64_t *off2, bbt_mibf_hit *hits, uint32_t max_hits,
		uint32_t *n_hits, uint32_t *sat, cudaStream_t s, MibfScratch &sc);
/* load the header, IDs file names, ID array (host) and frame probabilities */
int mibf_load_host(bbt_mibf *ctx, const char *bf_path, std::vector<uint16_t> *ids_out);
}

#endif
