/*
 * ctx.hpp -- the classification context behind the C ABI (bbt_ctx).
 */
#ifndef BBT_CTX_HPP
#define BBT_CTX_HPP

#include <cuda_runtime.h>

#include <mutex>
#include <string>
#include <vector>

#include "bbt.h"
#include "classify.cuh"
#include "dust.cuh"

namespace bbt {

/* One staging slot for host batches (inputs in, results out). */
struct Slot {
	uint8_t *d_seq[2] = {nullptr, nullptr};   /* ASCII bytes or 2-bit code words */
	uint32_t *d_valid[2] = {nullptr, nullptr}; /* 2-bit batches: validity bits */
	uint64_t *d_off[2] = {nullptr, nullptr};
	uint64_t *d_hits[2] = {nullptr, nullptr};
	uint32_t *d_cat = nullptr;
	double *d_scores[2] = {nullptr, nullptr}; /* BESTHIT / SCORES: reads x filters */
	uint64_t scores_cap = 0;                  /* reads d_scores holds */
	/* Results bound for pageable host memory go through this pinned buffer
	 * (a device-to-host copy into pageable memory would block the host until
	 * the slot's kernels finish, and so stop the next slot's input copy from
	 * overlapping them); `pending` lists the host copies to make once `done`
	 * has been reached. */
	struct HostCopy {
		void *dst;
		size_t off;
		size_t bytes;
	};
	unsigned char *h_stage = nullptr;
	size_t stage_cap = 0;
	std::vector<HostCopy> pending;
	cudaEvent_t copied = nullptr;   /* inputs are on the device */
	cudaEvent_t computed = nullptr; /* kernels done */
	cudaEvent_t done = nullptr;     /* results are back on the host */
	bool used = false;
};

void set_global_error(const std::string &msg);

} // namespace bbt

struct bbt_ctx {
	std::string err;
	bbt_params p;
	int dev = 0;
	int num_sms = 0;
	cudaStream_t stream = nullptr;  /* kernels */
	cudaStream_t h2d = nullptr;     /* host -> device copies */
	cudaStream_t d2h = nullptr;     /* device -> host copies */
	std::vector<std::string> ids;
	std::vector<bbt::FilterDev> hf;
	std::vector<uint32_t *> d_words;
	bbt::FilterDev *d_filters = nullptr;
	uint32_t nf = 0, words = 0, kmax = 0;
	unsigned long long *d_counts = nullptr; /* 2*(nf+2)+2 summary counters */
	unsigned long long *d_work = nullptr;   /* persistent-kernel read counter */
	unsigned long long *d_stat = nullptr;   /* probes, frames */
	uint64_t reads_seen = 0;
	bbt::Slot slot[2];
	uint64_t cap_bases = 0, cap_reads = 0;
	uint64_t *d_tmp_hits[2] = {nullptr, nullptr};
	uint64_t tmp_hits_cap = 0;
	/* filtering mode (BBT_MODE_*): ORDERED, BESTHIT and SCORES */
	int mode = BBT_MODE_STD;
	double *d_fpr = nullptr;         /* each filter's FPR on the device (BINOMIAL scores) */
	double *d_tmp_scores[2] = {nullptr, nullptr}; /* BESTHIT scores nobody asked for */
	uint64_t tmp_scores_cap = 0;                  /* elements per mate array */
	/* -D: SDUST masking before classification (dust.cu) */
	bool dust = false;
	int dust_T = 20, dust_W = 64;
	uint32_t *d_dust[2] = {nullptr, nullptr};  /* per-mate masked-base bits */
	uint64_t dust_words_cap[2] = {0, 0};
	uint64_t *d_dust_redo = nullptr;
	uint64_t dust_redo_cap = 0;
	unsigned long long *d_dust_cnt = nullptr;  /* reads queued for pass 2, reads failed */
	void *d_dust_scratch = nullptr;
	uint64_t dust_per_thread = 0;
	uint32_t dust_threads2 = 0;
	/* two-pass filter-major scratch: padded frame offsets, per-block sums,
	 * per-frame canonical hashes and validity words of one sub-batch */
	uint64_t *d_tp_local = nullptr;
	uint64_t tp_local_cap = 0;
	unsigned long long *d_tp_sums = nullptr;
	unsigned long long *h_tp_sums = nullptr; /* pinned copy */
	uint64_t tp_sums_cap = 0;
	uint64_t *d_tp_h0 = nullptr;
	uint32_t *d_tp_vmask = nullptr;
	uint64_t tp_frames_cap = 0;
	bool same_k = true;
	/* BINOMIAL scoring: each filter's FPR and the accept thresholds
	 * calcMinCount(frames, fpr, score) by filter and frame count */
	std::vector<double> fpr;
	std::mutex bt_mu;
	std::vector<uint32_t> h_bthres;  /* nf x bt_rows */
	std::vector<uint8_t> bt_have;    /* by read length */
	uint32_t *d_bthres = nullptr;
	uint64_t bt_rows = 0;
	unsigned int *d_lenset = nullptr;
	bool capturing = false;          /* a CUDA graph is being captured */
	/* -d / -n: print reads of the first filter (or all others) to stdout */
	bool to_stdout = false, inverse = false;
	/* long-first read order of the persistent kernel (0 = index order) */
	uint64_t long_bases = 0;
	uint64_t *d_order = nullptr;
	uint64_t order_cap = 0;
	unsigned long long *d_order_cnt = nullptr;
	/* bucketed probe path (bucketed.cu): frame offsets of a batch's reads and
	 * their host samples, per-read state, the batch's bases as 2-bit codes
	 * (ASCII batches), validity / hit / requesting bits and canonical hashes
	 * of a sub-batch's frames, the request pool, per-(bucket, block) counts
	 * and first slots, scan scratch; and the path's settings */
	uint64_t *d_bk_fo = nullptr;
	uint8_t *d_bk_state = nullptr;
	uint64_t bk_reads_cap = 0;
	uint64_t *h_bk_samples = nullptr;      /* pinned */
	uint64_t *d_bk_samples = nullptr;
	uint64_t bk_samples_cap = 0;
	uint32_t *d_bk_codes[2] = {nullptr, nullptr};
	uint32_t *d_bk_cvalid[2] = {nullptr, nullptr};
	uint64_t bk_codes_cap[2] = {0, 0}, bk_cvalid_cap[2] = {0, 0};
	uint32_t *d_bk_vbits = nullptr, *d_bk_hbits = nullptr, *d_bk_abits = nullptr;
	uint64_t *d_bk_canon = nullptr;
	uint32_t *d_bk_off = nullptr;
	uint16_t *d_bk_fid = nullptr;
	uint8_t *d_bk_res = nullptr;
	uint32_t *d_bk_btot = nullptr;
	uint64_t bk_frames_cap = 0;
	uint32_t bk_pool_levels = 0;          /* tests per frame the pool holds */
	uint32_t *d_bk_cnt = nullptr, *d_bk_loc = nullptr;
	uint64_t bk_cnt_cap = 0;
	void *d_bk_tmp = nullptr;
	size_t bk_tmp_cap = 0;
	uint64_t bk_max_frames = 1ull << 30; /* frames per sub-batch */
	uint32_t bk_bshift = 27;             /* bucket of 2^27 bits (16 MB) */
	uint32_t bk_phase_split = 4;         /* phase boundary in sixteenths (16: one phase) */
	uint32_t bk_phase_min = 64;          /* the first phase covers min(F, 64) frames or more */
	uint32_t bk_levels = 1;              /* hash levels per round */
	int steps = BBT_STEPS_DECISION;      /* bbt_set_steps */
	/* bbt_open_devices: the same filters opened on the other devices; host
	 * batches are split across this context and these */
	std::vector<bbt_ctx *> peers;
	cudaEvent_t ev_start = nullptr, ev_stop = nullptr;
	cudaEvent_t ev_k0 = nullptr, ev_k1 = nullptr; /* around the last classify kernel */
	bbt::LaunchConfig lc;
	bbt_stats last = {0, 0, 0, 0, 0.0, 0.0, 0};
};

namespace bbt {
int fail(bbt_ctx *ctx, int code, const std::string &msg);

/* Per-stream scratch for classification calls that run concurrently on
 * several streams of one context (the serving engine): each stream needs its
 * own work counter and read-order buffer. */
struct BfScratch {
	unsigned long long *work = nullptr;
	unsigned long long *order_cnt = nullptr;
	uint64_t *order = nullptr;
	uint64_t order_cap = 0;
};
int bf_scratch_init(bbt_ctx *ctx, BfScratch &sc, uint64_t max_reads);
/* BINOMIAL: allocate threshold rows for reads up to max_len bases up front
 * (the serving engine, so that the table never moves under running kernels),
 * and fill the rows of these reads (host offsets). */
int bf_reserve_rows(bbt_ctx *ctx, uint64_t max_len);
int bf_rows_for(bbt_ctx *ctx, const uint64_t *off, const uint64_t *off2, uint64_t n);
void bf_scratch_free(BfScratch &sc);
/* Classify n reads (n pairs when seq2) resident on the device, offsets
 * relative to seq / seq2, into hits (hits2) and category on stream s, adding to
 * the summary counters; no host synchronization.  Plain or persistent kernel
 * (the tuned filter-major order is replaced by the persistent one). */
int bf_classify_slot(bbt_ctx *ctx, const uint8_t *seq, const uint64_t *off, const uint8_t *seq2,
		const uint64_t *off2, uint64_t n, uint64_t *hits, uint64_t *hits2, uint32_t *category,
		cudaStream_t s, BfScratch &sc);
int cuda_fail(bbt_ctx *ctx, cudaError_t e, const char *what);
std::string summary_text(const bbt_ctx *ctx, const std::vector<uint64_t> &counts, uint64_t reads);
}

#endif
