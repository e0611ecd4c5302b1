/*
 * api.cu -- the C ABI of libbbt.so (declared in include/bbt.h): contexts,
 * filter upload, batch classification with host staging, summary counters.
 */
#include <cuda_runtime.h>

#include <cub/device/device_scan.cuh>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <sstream>
#include <string>
#include <thread>
#include <vector>

#include "bbt.h"
#include "bucketed.cuh"
#include "classify.cuh"
#include "ctx.hpp"
#include "formats.hpp"
#include "twopass.cuh"

namespace bbt {

static std::mutex g_err_mu;
static std::string g_err;

void set_global_error(const std::string &msg)
{
	std::lock_guard<std::mutex> lk(g_err_mu);
	g_err = msg;
}

int fail(bbt_ctx *ctx, int code, const std::string &msg)
{
	if (ctx)
		ctx->err = msg;
	else
		set_global_error(msg);
	return code;
}

int cuda_fail(bbt_ctx *ctx, cudaError_t e, const char *what)
{
	std::string m = std::string(what) + ": " + cudaGetErrorString(e);
	return fail(ctx, e == cudaErrorMemoryAllocation ? BBT_ERR_NOMEM : BBT_ERR_CUDA, m);
}

/* ResultsManager::getResultsSummary (ResultsManager.hpp:191-237): the same
 * rows and the default ostream number format. */
std::string summary_text(const bbt_ctx *ctx, const std::vector<uint64_t> &c, uint64_t reads)
{
	const uint32_t nf = ctx->nf;
	const uint64_t *above = c.data();
	const uint64_t *unique = c.data() + (nf + 2);
	const uint64_t multi = c[2 * (nf + 2)];
	const uint64_t nomatch = c[2 * (nf + 2) + 1];
	const double rc = (double)reads;
	std::ostringstream o;
	o << "filter_id\thits\tmisses\tshared\trate_hit\trate_miss\trate_shared\n";
	for (uint32_t i = 0; i < nf; ++i) {
		o << ctx->ids[i] << "\t" << above[i] << "\t" << reads - above[i] << "\t"
		  << (above[i] - unique[i]) << "\t" << double(above[i]) / rc << "\t"
		  << double(reads - above[i]) / rc << "\t" << double(above[i] - unique[i]) / rc << "\n";
	}
	o << "multiMatch\t" << multi << "\t" << reads - multi << "\t" << 0 << "\t"
	  << double(multi) / rc << "\t" << double(reads - multi) / rc << "\t" << 0.0 << "\n";
	o << "noMatch\t" << nomatch << "\t" << reads - nomatch << "\t" << 0 << "\t"
	  << double(nomatch) / rc << "\t" << double(reads - nomatch) / rc << "\t" << 0.0 << "\n";
	return o.str();
}

} // namespace bbt

using namespace bbt;

#define CUDA_TRY(ctx, call)                                                                \
	do {                                                                                   \
		cudaError_t e_ = (call);                                                           \
		if (e_ != cudaSuccess)                                                             \
			return cuda_fail((ctx), e_, #call);                                            \
	} while (0)

extern "C" void bbt_default_params(bbt_params *p)
{
	if (!p)
		return;
	memset(p, 0, sizeof(*p));
	p->score = 0.15;           /* BioBloomCategorizer/Options.cpp:15 */
	p->streak_threshold = 3;   /* Common/Options.cpp:9 */
	p->scoring = BBT_SCORE_SIMPLE;
	p->path = BBT_PATH_AUTO;
}

extern "C" const char *bbt_last_error(const bbt_ctx *ctx)
{
	if (ctx)
		return ctx->err.c_str();
	static thread_local std::string copy;
	std::lock_guard<std::mutex> lk(g_err_mu);
	copy = g_err;
	return copy.c_str();
}

static void free_slot(Slot &s)
{
	for (int m = 0; m < 2; ++m) {
		cudaFree(s.d_seq[m]);
		cudaFree(s.d_valid[m]);
		s.d_valid[m] = nullptr;
		cudaFree(s.d_off[m]);
		cudaFree(s.d_hits[m]);
		cudaFree(s.d_scores[m]);
		s.d_seq[m] = nullptr;
		s.d_off[m] = nullptr;
		s.d_hits[m] = nullptr;
		s.d_scores[m] = nullptr;
	}
	s.scores_cap = 0;
	cudaFree(s.d_cat);
	s.d_cat = nullptr;
	cudaFreeHost(s.h_stage);
	s.h_stage = nullptr;
	s.stage_cap = 0;
	s.pending.clear();
}

/* Host memory that the GPU can copy into without staging (pinned or
 * registered). */
static bool host_pinned(const void *p)
{
	cudaPointerAttributes at;
	if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
		cudaGetLastError();
		return false;
	}
	return at.type == cudaMemoryTypeHost;
}

/* The staged results of a slot whose copies are done, to their destinations. */
static void flush_slot(Slot &s)
{
	for (const Slot::HostCopy &c : s.pending)
		memcpy(c.dst, s.h_stage + c.off, c.bytes);
	s.pending.clear();
}

extern "C" int bbt_close(bbt_ctx *ctx)
{
	if (!ctx)
		return BBT_OK;
	for (bbt_ctx *peer : ctx->peers)
		bbt_close(peer);
	ctx->peers.clear();
	cudaSetDevice(ctx->dev);
	if (ctx->stream)
		cudaStreamSynchronize(ctx->stream);
	if (ctx->h2d)
		cudaStreamSynchronize(ctx->h2d);
	if (ctx->d2h)
		cudaStreamSynchronize(ctx->d2h);
	for (uint32_t *w : ctx->d_words)
		cudaFree(w);
	cudaFree(ctx->d_filters);
	cudaFree(ctx->d_fpr);
	cudaFree(ctx->d_tmp_scores[0]);
	cudaFree(ctx->d_tmp_scores[1]);
	cudaFree(ctx->d_dust[0]);
	cudaFree(ctx->d_dust[1]);
	cudaFree(ctx->d_dust_redo);
	cudaFree(ctx->d_dust_cnt);
	cudaFree(ctx->d_dust_scratch);
	cudaFree(ctx->d_counts);
	cudaFree(ctx->d_work);
	cudaFree(ctx->d_order);
	cudaFree(ctx->d_order_cnt);
	cudaFree(ctx->d_bthres);
	cudaFree(ctx->d_lenset);
	cudaFree(ctx->d_stat);
	cudaFree(ctx->d_tmp_hits[0]);
	cudaFree(ctx->d_tmp_hits[1]);
	cudaFree(ctx->d_tp_local);
	cudaFree(ctx->d_tp_sums);
	cudaFreeHost(ctx->h_tp_sums);
	cudaFree(ctx->d_bk_fo);
	cudaFree(ctx->d_bk_state);
	cudaFreeHost(ctx->h_bk_samples);
	cudaFree(ctx->d_bk_samples);
	for (int i = 0; i < 2; ++i) {
		cudaFree(ctx->d_bk_codes[i]);
		cudaFree(ctx->d_bk_cvalid[i]);
	}
	cudaFree(ctx->d_bk_vbits);
	cudaFree(ctx->d_bk_hbits);
	cudaFree(ctx->d_bk_abits);
	cudaFree(ctx->d_bk_canon);
	cudaFree(ctx->d_bk_off);
	cudaFree(ctx->d_bk_fid);
	cudaFree(ctx->d_bk_res);
	cudaFree(ctx->d_bk_btot);
	cudaFree(ctx->d_bk_cnt);
	cudaFree(ctx->d_bk_loc);
	cudaFree(ctx->d_bk_tmp);
	cudaFree(ctx->d_tp_h0);
	cudaFree(ctx->d_tp_vmask);
	for (Slot &s : ctx->slot) {
		free_slot(s);
		if (s.copied)
			cudaEventDestroy(s.copied);
		if (s.computed)
			cudaEventDestroy(s.computed);
		if (s.done)
			cudaEventDestroy(s.done);
	}
	if (ctx->ev_start)
		cudaEventDestroy(ctx->ev_start);
	if (ctx->ev_stop)
		cudaEventDestroy(ctx->ev_stop);
	if (ctx->ev_k0)
		cudaEventDestroy(ctx->ev_k0);
	if (ctx->ev_k1)
		cudaEventDestroy(ctx->ev_k1);
	if (ctx->stream)
		cudaStreamDestroy(ctx->stream);
	if (ctx->h2d)
		cudaStreamDestroy(ctx->h2d);
	if (ctx->d2h)
		cudaStreamDestroy(ctx->d2h);
	delete ctx;
	return BBT_OK;
}

/* Read one .bf payload and copy it to the device in pinned chunks. */
static int upload_filter(bbt_ctx *ctx, const std::string &path, BfHeader &hd, uint32_t **d_out,
		uint64_t *pop_out)
{
	uint64_t pop = 0;
	FILE *f = fopen(path.c_str(), "rb");
	if (!f)
		return fail(ctx, BBT_ERR_IO, "file " + path + " cannot be opened");
	const char *msg = read_bf_header(f, hd);
	if (msg) {
		fclose(f);
		return fail(ctx, BBT_ERR_FORMAT, path + ": " + msg);
	}
	const uint64_t bytes = hd.m / 8;
	uint32_t *d = nullptr;
	cudaError_t e = cudaMalloc(&d, bytes);
	if (e != cudaSuccess) {
		fclose(f);
		return cuda_fail(ctx, e, "cudaMalloc(filter)");
	}
	const size_t chunk = 64ull << 20;
	void *pinned = nullptr;
	e = cudaMallocHost(&pinned, std::min<uint64_t>(chunk, bytes) * 2);
	if (e != cudaSuccess) {
		fclose(f);
		cudaFree(d);
		return cuda_fail(ctx, e, "cudaMallocHost(filter staging)");
	}
	uint64_t done = 0;
	int which = 0;
	cudaEvent_t ev[2];
	cudaEventCreateWithFlags(&ev[0], cudaEventDisableTiming);
	cudaEventCreateWithFlags(&ev[1], cudaEventDisableTiming);
	bool ev_used[2] = {false, false};
	int rc = BBT_OK;
	while (done < bytes) {
		size_t n = (size_t)std::min<uint64_t>(chunk, bytes - done);
		char *buf = (char *)pinned + which * std::min<uint64_t>(chunk, bytes);
		if (ev_used[which])
			cudaEventSynchronize(ev[which]);
		if (fread(buf, 1, n, f) != n) {
			rc = fail(ctx, BBT_ERR_FORMAT, path + ": filter payload is shorter than its header says");
			break;
		}
		for (size_t i = 0; i + 8 <= n; i += 8) {
			uint64_t w;
			memcpy(&w, buf + i, 8);
			pop += (uint64_t)__builtin_popcountll(w);
		}
		e = cudaMemcpyAsync((char *)d + done, buf, n, cudaMemcpyHostToDevice, ctx->h2d);
		if (e != cudaSuccess) {
			rc = cuda_fail(ctx, e, "cudaMemcpyAsync(filter)");
			break;
		}
		cudaEventRecord(ev[which], ctx->h2d);
		ev_used[which] = true;
		done += n;
		which ^= 1;
	}
	cudaStreamSynchronize(ctx->h2d);
	cudaEventDestroy(ev[0]);
	cudaEventDestroy(ev[1]);
	cudaFreeHost(pinned);
	fclose(f);
	if (rc != BBT_OK) {
		cudaFree(d);
		return rc;
	}
	*d_out = d;
	if (pop_out)
		*pop_out = pop;
	return BBT_OK;
}

/* Host-only checks of one filter's files before any device work: the .txt
 * sidecar opens and names the filter, the .bf header parses and the payload
 * holds the m / 8 bytes the header promises.  The reference exits on the same
 * conditions (BloomFilterInfo / BloomFilter constructors). */
static int check_filter_files(const std::string &path)
{
	std::map<std::string, std::string> kv;
	const std::string info = info_path_for(path);
	if (!read_ini(info, kv))
		return fail(nullptr, BBT_ERR_IO, "file " + info + " cannot be opened");
	if (kv.find("user_input_options.filter_id") == kv.end())
		return fail(nullptr, BBT_ERR_FORMAT, info + ": no user_input_options.filter_id");
	FILE *f = fopen(path.c_str(), "rb");
	if (!f)
		return fail(nullptr, BBT_ERR_IO, "file " + path + " cannot be opened");
	BfHeader hd;
	const char *msg = read_bf_header(f, hd);
	if (msg) {
		fclose(f);
		return fail(nullptr, BBT_ERR_FORMAT, path + ": " + msg);
	}
	const long at = ftell(f);
	const bool sized = at >= 0 && fseek(f, 0, SEEK_END) == 0;
	const long end = sized ? ftell(f) : -1;
	fclose(f);
	if (!sized || end < at || (uint64_t)(end - at) < hd.m / 8)
		return fail(nullptr, BBT_ERR_FORMAT, path + ": filter payload is shorter than its "
				"header says (" + std::to_string(hd.m / 8) + " bytes)");
	return BBT_OK;
}

static int alloc_slot(bbt_ctx *ctx, Slot &s, uint64_t bases, uint64_t reads)
{
	free_slot(s);
	for (int m = 0; m < 2; ++m) {
		CUDA_TRY(ctx, cudaMalloc(&s.d_seq[m], std::max<uint64_t>(bases, 16)));
		/* a 2-bit batch's validity bits: one bit per base plus alignment */
		CUDA_TRY(ctx, cudaMalloc(&s.d_valid[m], bases / 8 + 16));
		CUDA_TRY(ctx, cudaMalloc(&s.d_off[m], (reads + 1) * sizeof(uint64_t)));
		CUDA_TRY(ctx, cudaMalloc(&s.d_hits[m], reads * ctx->words * sizeof(uint64_t)));
	}
	CUDA_TRY(ctx, cudaMalloc(&s.d_cat, reads * sizeof(uint32_t)));
	return BBT_OK;
}

/* Filters far above L2, where sorting probes by address pays for its passes:
 * the largest above 256 MB. */
static bool bucketing_pays(const bbt_ctx *ctx)
{
	for (const FilterDev &f : ctx->hf)
		if (f.m / 8 > (256ull << 20))
			return true;
	return false;
}

/* The tuned path: with two or more filters of one k that each fit in L2,
 * probe them one at a time out of L2 (two-pass filter-major); otherwise the
 * persistent read-major kernel. */
static int auto_path(const bbt_ctx *ctx)
{
	if (ctx->nf < 2 || !ctx->same_k)
		return BBT_PATH_PERSISTENT;
	int l2 = 0;
	cudaDeviceGetAttribute(&l2, cudaDevAttrL2CacheSize, ctx->dev);
	for (const FilterDev &f : ctx->hf)
		if (f.m / 8 > (uint64_t)l2 * 3 / 4)
			return BBT_PATH_PERSISTENT;
	return BBT_PATH_FILTER_MAJOR;
}

static LaunchConfig pick_config(const bbt_ctx *ctx)
{
	LaunchConfig lc;
	lc.path = ctx->p.path == BBT_PATH_AUTO ? auto_path(ctx) : ctx->p.path;
	lc.warps_per_block = ctx->p.warps_per_block ? (int)ctx->p.warps_per_block : 8;
	lc.seg = ctx->p.frames_per_lane == 8 ? 8 : 4;
	lc.num_sms = ctx->num_sms;
	lc.count = 0;
	lc.steps = ctx->steps;
	return lc;
}

extern "C" int bbt_open(const char *const *bf_paths, int n_filters, const bbt_params *params,
		bbt_ctx **out)
{
	if (!out || !bf_paths || n_filters <= 0)
		return fail(nullptr, BBT_ERR_ARG, "bbt_open: need at least one filter path and an out pointer");
	*out = nullptr;
	bbt_ctx *ctx = new bbt_ctx();
	if (params)
		ctx->p = *params;
	else
		bbt_default_params(&ctx->p);
	if (!(ctx->p.score < 4294967296.0) && ctx->p.scoring != BBT_SCORE_BINOMIAL) {
		bbt_close(ctx);
		return fail(nullptr, BBT_ERR_ARG, "score must be below 2^32");
	}
	if (ctx->p.score > 1 && (ctx->p.scoring == BBT_SCORE_SIMPLE ||
			ctx->p.scoring == BBT_SCORE_HARMONIC) && (unsigned)ctx->p.score > 1) {
		/* BioBloomCategorizer.cpp:423-430: an integer score > 1 is a
		 * minimum match length */
		ctx->p.score = (double)(unsigned)ctx->p.score;
		ctx->p.scoring = BBT_SCORE_LENGTH;
	}
	if (ctx->p.scoring == BBT_SCORE_SIMPLE && (ctx->p.score < 0 || ctx->p.score > 1)) {
		std::string m = "score must be in [0, 1] or an integer > 1";
		bbt_close(ctx);
		return fail(nullptr, BBT_ERR_ARG, m);
	}
	if ((ctx->p.scoring == BBT_SCORE_HARMONIC && (ctx->p.score < 0 || ctx->p.score > 1)) ||
			(ctx->p.scoring == BBT_SCORE_BINOMIAL && !(ctx->p.score > 0 && ctx->p.score <= 1)) ||
			ctx->p.scoring < BBT_SCORE_SIMPLE || ctx->p.scoring > BBT_SCORE_BINOMIAL) {
		std::string m = "harmonic scores are in [0, 1]; binomial scores are a minimum FPR in "
				"(0, 1]; the scoring method is BBT_SCORE_*";
		bbt_close(ctx);
		return fail(nullptr, BBT_ERR_ARG, m);
	}
	for (int i = 0; i < n_filters; ++i) {
		if (!bf_paths[i]) {
			bbt_close(ctx);
			return fail(nullptr, BBT_ERR_ARG, "null filter path");
		}
		int rc0 = check_filter_files(bf_paths[i]);
		if (rc0 != BBT_OK) {
			std::string m = bbt_last_error(nullptr);
			bbt_close(ctx);
			return fail(nullptr, rc0, m);
		}
	}
	int ndev = 0;
	cudaError_t e = cudaGetDeviceCount(&ndev);
	if (e != cudaSuccess || ndev == 0) {
		bbt_close(ctx);
		return fail(nullptr, BBT_ERR_NODEVICE,
				std::string("no CUDA device: ") + (e != cudaSuccess ? cudaGetErrorString(e) : "0 devices"));
	}
	if (ctx->p.device < 0 || ctx->p.device >= ndev) {
		bbt_close(ctx);
		return fail(nullptr, BBT_ERR_ARG, "device ordinal out of range");
	}
	ctx->dev = ctx->p.device;
	int rc = BBT_OK;
#define OPEN_TRY(call)                                              \
	do {                                                            \
		cudaError_t e_ = (call);                                    \
		if (e_ != cudaSuccess) {                                    \
			rc = cuda_fail(ctx, e_, #call);                         \
			goto fail_out;                                          \
		}                                                           \
	} while (0)
	OPEN_TRY(cudaSetDevice(ctx->dev));
	OPEN_TRY(cudaDeviceGetAttribute(&ctx->num_sms, cudaDevAttrMultiProcessorCount, ctx->dev));
	/* Bloom probes are isolated 4-byte reads at random addresses: fetching
	 * more than the 32-byte sector per L2 miss only moves bytes nobody reads.
	 * The limit belongs to this process's context and ends with it. */
	OPEN_TRY(cudaDeviceSetLimit(cudaLimitMaxL2FetchGranularity,
			ctx->p.l2_fetch_bytes ? ctx->p.l2_fetch_bytes : 32));
	OPEN_TRY(cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking));
	OPEN_TRY(cudaStreamCreateWithFlags(&ctx->h2d, cudaStreamNonBlocking));
	OPEN_TRY(cudaStreamCreateWithFlags(&ctx->d2h, cudaStreamNonBlocking));
	OPEN_TRY(cudaEventCreate(&ctx->ev_start));
	OPEN_TRY(cudaEventCreate(&ctx->ev_stop));
	OPEN_TRY(cudaEventCreate(&ctx->ev_k0));
	OPEN_TRY(cudaEventCreate(&ctx->ev_k1));
	for (Slot &s : ctx->slot) {
		OPEN_TRY(cudaEventCreateWithFlags(&s.copied, cudaEventDisableTiming));
		OPEN_TRY(cudaEventCreateWithFlags(&s.computed, cudaEventDisableTiming));
		OPEN_TRY(cudaEventCreateWithFlags(&s.done, cudaEventDisableTiming));
	}
	for (int i = 0; i < n_filters; ++i) {
		if (!bf_paths[i]) {
			rc = fail(ctx, BBT_ERR_ARG, "null filter path");
			goto fail_out;
		}
		std::string path = bf_paths[i];
		std::map<std::string, std::string> kv;
		std::string info = info_path_for(path);
		if (!read_ini(info, kv)) {
			rc = fail(ctx, BBT_ERR_IO, "file " + info + " cannot be opened");
			goto fail_out;
		}
		auto it = kv.find("user_input_options.filter_id");
		if (it == kv.end()) {
			rc = fail(ctx, BBT_ERR_FORMAT, info + ": no user_input_options.filter_id");
			goto fail_out;
		}
		ctx->ids.push_back(it->second);
		BfHeader hd;
		uint32_t *d = nullptr;
		uint64_t pop = 0;
		rc = upload_filter(ctx, path, hd, &d, &pop);
		if (rc != BBT_OK)
			goto fail_out;
		ctx->d_words.push_back(d);
		ctx->hf.push_back(make_filter_dev(d, hd.m, hd.h, hd.k));
		/* BloomFilter::getFPRPrecompute as restated: (set bits / m) ^ h */
		ctx->fpr.push_back(pow((double)pop / (double)hd.m, (double)hd.h));
		ctx->kmax = std::max(ctx->kmax, hd.k);
	}
	ctx->nf = (uint32_t)n_filters;
	for (const FilterDev &fd : ctx->hf)
		ctx->same_k = ctx->same_k && fd.k == ctx->hf[0].k;
	ctx->words = (ctx->nf + 63) / 64;
	OPEN_TRY(cudaMalloc(&ctx->d_filters, sizeof(FilterDev) * ctx->nf));
	OPEN_TRY(cudaMemcpy(ctx->d_filters, ctx->hf.data(), sizeof(FilterDev) * ctx->nf,
			cudaMemcpyHostToDevice));
	OPEN_TRY(cudaMalloc(&ctx->d_fpr, sizeof(double) * ctx->nf));
	OPEN_TRY(cudaMemcpy(ctx->d_fpr, ctx->fpr.data(), sizeof(double) * ctx->nf,
			cudaMemcpyHostToDevice));
	OPEN_TRY(cudaMalloc(&ctx->d_counts, sizeof(unsigned long long) * (2 * (ctx->nf + 2) + 2)));
	OPEN_TRY(cudaMemset(ctx->d_counts, 0, sizeof(unsigned long long) * (2 * (ctx->nf + 2) + 2)));
	OPEN_TRY(cudaMalloc(&ctx->d_work, sizeof(unsigned long long)));
	OPEN_TRY(cudaMalloc(&ctx->d_order_cnt, 2 * sizeof(unsigned long long)));
	OPEN_TRY(cudaMalloc(&ctx->d_stat, 3 * sizeof(unsigned long long)));
	OPEN_TRY(cudaMemset(ctx->d_stat, 0, 3 * sizeof(unsigned long long)));
	ctx->cap_reads = ctx->p.max_batch_reads ? ctx->p.max_batch_reads : (1ull << 20);
	ctx->cap_bases = ctx->p.max_batch_bases ? ctx->p.max_batch_bases : (256ull << 20);
	for (Slot &s : ctx->slot) {
		rc = alloc_slot(ctx, s, ctx->cap_bases, ctx->cap_reads);
		if (rc != BBT_OK)
			goto fail_out;
	}
	ctx->lc = pick_config(ctx);
	*out = ctx;
	return BBT_OK;
fail_out : {
	std::string m = ctx->err;
	bbt_close(ctx);
	return fail(nullptr, rc, m);
}
#undef OPEN_TRY
}

extern "C" int bbt_open_devices(const char *const *bf_paths, int n_filters,
		const bbt_params *params, const int *devices, int n_devices, bbt_ctx **out)
{
	if (!out || !devices || n_devices < 1)
		return fail(nullptr, BBT_ERR_ARG, "bbt_open_devices: need at least one device and an "
				"out pointer");
	*out = nullptr;
	bbt_params p;
	if (params)
		p = *params;
	else
		bbt_default_params(&p);
	bbt_ctx *first = nullptr;
	p.device = devices[0];
	int rc = bbt_open(bf_paths, n_filters, &p, &first);
	if (rc)
		return rc;
	for (int i = 1; i < n_devices; ++i) {
		bbt_ctx *peer = nullptr;
		p.device = devices[i];
		rc = bbt_open(bf_paths, n_filters, &p, &peer);
		if (rc) {
			std::string m = bbt_last_error(nullptr);
			bbt_close(first);
			return fail(nullptr, rc, "device " + std::to_string(devices[i]) + ": " + m);
		}
		first->peers.push_back(peer);
	}
	*out = first;
	return BBT_OK;
}

extern "C" int bbt_num_filters(const bbt_ctx *ctx)
{
	return ctx ? (int)ctx->nf : BBT_ERR_ARG;
}

extern "C" const char *bbt_filter_id(const bbt_ctx *ctx, int i)
{
	if (!ctx || i < 0 || (uint32_t)i >= ctx->nf)
		return nullptr;
	return ctx->ids[i].c_str();
}

/* ---- BINOMIAL thresholds: calcMinCount(frames, fpr of filter, score) ---- */

namespace bbt {
unsigned binom_upper_quantile(unsigned n, double p, double q);
}

/* Rows for read lengths below `rows` (callers hold bt_mu). */
static int bt_grow(bbt_ctx *ctx, uint64_t rows)
{
	if (rows <= ctx->bt_rows)
		return BBT_OK;
	rows = std::max<uint64_t>(rows, std::max<uint64_t>(2 * ctx->bt_rows, 1024));
	std::vector<uint32_t> h((size_t)ctx->nf * rows, 0);
	for (uint32_t f = 0; f < ctx->nf && ctx->bt_rows; ++f)
		memcpy(&h[(size_t)f * rows], &ctx->h_bthres[(size_t)f * ctx->bt_rows], ctx->bt_rows * 4);
	uint32_t *d = nullptr;
	CUDA_TRY(ctx, cudaDeviceSynchronize()); /* no kernel may still read the old table */
	CUDA_TRY(ctx, cudaMalloc(&d, h.size() * 4));
	CUDA_TRY(ctx, cudaMemcpy(d, h.data(), h.size() * 4, cudaMemcpyHostToDevice));
	cudaFree(ctx->d_bthres);
	ctx->d_bthres = d;
	ctx->h_bthres.swap(h);
	ctx->bt_have.resize(rows, 0);
	ctx->bt_rows = rows;
	return BBT_OK;
}

/* Make the rows of these read lengths present on the device. */
static int ensure_bthres(bbt_ctx *ctx, const std::vector<uint64_t> &lens)
{
	if (ctx->p.scoring != BBT_SCORE_BINOMIAL || lens.empty())
		return BBT_OK;
	std::lock_guard<std::mutex> lk(ctx->bt_mu);
	int rc = bt_grow(ctx, lens.back() + 1);
	if (rc)
		return rc;
	std::vector<uint64_t> missing;
	for (uint64_t L : lens)
		if (!ctx->bt_have[L])
			missing.push_back(L);
	if (missing.empty())
		return BBT_OK;
	const long long nm = (long long)missing.size() * ctx->nf;
#pragma omp parallel for schedule(dynamic, 8)
	for (long long t = 0; t < nm; ++t) {
		const uint64_t L = missing[t / ctx->nf];
		const uint32_t f = (uint32_t)(t % ctx->nf);
		const unsigned k = ctx->hf[f].k;
		if (L < k)
			continue;
		const uint64_t fc = L - k + 1;
		const unsigned i = binom_upper_quantile((unsigned)fc, ctx->fpr[f], ctx->p.score);
		ctx->h_bthres[(size_t)f * ctx->bt_rows + fc] = i > 1 ? i : 1;
	}
	for (uint64_t L : missing)
		ctx->bt_have[L] = 1;
	/* rows L - k + 1 of each filter, for the lengths just computed */
	for (uint32_t f = 0; f < ctx->nf; ++f) {
		const unsigned k = ctx->hf[f].k;
		for (uint64_t L : missing) {
			if (L < k)
				continue;
			const size_t at = (size_t)f * ctx->bt_rows + (L - k + 1);
			CUDA_TRY(ctx, cudaMemcpy(ctx->d_bthres + at, &ctx->h_bthres[at], 4,
					cudaMemcpyHostToDevice));
		}
	}
	return BBT_OK;
}

static std::vector<uint64_t> host_lengths(const uint64_t *off, const uint64_t *off2, uint64_t n)
{
	std::vector<uint64_t> lens;
	std::vector<uint8_t> seen;
	for (int m = 0; m < (off2 ? 2 : 1); ++m) {
		const uint64_t *o = m ? off2 : off;
		for (uint64_t i = 0; i < n; ++i) {
			const uint64_t L = o[i + 1] - o[i];
			if (L >= seen.size())
				seen.resize(L + 1, 0);
			if (!seen[L]) {
				seen[L] = 1;
				lens.push_back(L);
			}
		}
	}
	std::sort(lens.begin(), lens.end());
	return lens;
}

static int device_lengths(bbt_ctx *ctx, const bbt_batch *b, cudaStream_t s,
		std::vector<uint64_t> &lens)
{
	if (!ctx->d_lenset)
		CUDA_TRY(ctx, cudaMalloc(&ctx->d_lenset, (1 + 2048) * 4));
	CUDA_TRY(ctx, cudaMemsetAsync(ctx->d_lenset, 0, (1 + 2048) * 4, s));
	CUDA_TRY(ctx, launch_length_set(b->offsets, b->seq2 ? b->offsets2 : nullptr, b->n_reads,
			b->seq2 ? 2 : 1, ctx->d_lenset, ctx->num_sms, s));
	std::vector<unsigned int> h(1 + 2048);
	CUDA_TRY(ctx, cudaMemcpyAsync(h.data(), ctx->d_lenset, h.size() * 4, cudaMemcpyDeviceToHost,
			s));
	CUDA_TRY(ctx, cudaStreamSynchronize(s));
	for (uint64_t L = 0; L < 65536 && L <= h[0]; ++L)
		if ((h[1 + (L >> 5)] >> (L & 31)) & 1u)
			lens.push_back(L);
	for (uint64_t L = 65536; L <= h[0]; ++L) /* rare: every longer length up to the maximum */
		lens.push_back(L);
	return BBT_OK;
}

int bbt::bf_reserve_rows(bbt_ctx *ctx, uint64_t max_len)
{
	if (ctx->p.scoring != BBT_SCORE_BINOMIAL)
		return BBT_OK;
	std::lock_guard<std::mutex> lk(ctx->bt_mu);
	return bt_grow(ctx, max_len + 1);
}

int bbt::bf_rows_for(bbt_ctx *ctx, const uint64_t *off, const uint64_t *off2, uint64_t n)
{
	if (ctx->p.scoring != BBT_SCORE_BINOMIAL)
		return BBT_OK;
	std::vector<uint64_t> lens = host_lengths(off, off2, n);
	if (!lens.empty() && lens.back() >= ctx->bt_rows)
		return fail(ctx, BBT_ERR_ARG, "a read is longer than the binomial threshold rows "
				"reserved for serving");
	return ensure_bthres(ctx, lens);
}

static ClassifyArgs base_args(const bbt_ctx *ctx)
{
	ClassifyArgs a;
	memset(&a, 0, sizeof a);
	a.filters = ctx->d_filters;
	a.nf = ctx->nf;
	a.words = ctx->words;
	a.score = ctx->p.score;
	a.one_minus = 1.0 - ctx->p.score;
	a.streak_thr = ctx->p.streak_threshold;
	a.scoring = ctx->p.scoring;
	a.min_len = (unsigned)std::round(ctx->p.score);
	a.kmax = ctx->kmax;
	a.bthres = ctx->d_bthres;
	a.bthres_rows = ctx->bt_rows;
	a.work = ctx->d_work;
	if (ctx->lc.count) {
		a.probes = ctx->d_stat;
		a.frames = ctx->d_stat + 1;
		a.alg_probes = ctx->d_stat + 2;
	}
	return a;
}

/* Grow a device buffer to hold at least n elements (contents not kept). */
template <typename T>
static int grow(bbt_ctx *ctx, T **buf, uint64_t &cap, uint64_t n)
{
	if (n <= cap)
		return BBT_OK;
	cudaFree(*buf);
	*buf = nullptr;
	cap = 0;
	CUDA_TRY(ctx, cudaMalloc(buf, std::max<uint64_t>(n, 1) * sizeof(T)));
	cap = n;
	return BBT_OK;
}

/* Two-pass filter-major classification of one batch (all filters share k):
 * scan of padded frame counts, a host read of the per-block totals to cut the
 * batch into sub-batches whose frames fit the scratch, then hash pass and
 * filter pass per sub-batch. */
static int run_two_pass(bbt_ctx *ctx, ClassifyArgs &a, cudaStream_t s,
		const ScoreArgs *sa = nullptr, bool classify = true)
{
	const uint64_t total = a.n * a.mates;
	const uint64_t B = two_pass_block_reads();
	const uint64_t nb = (total + B - 1) / B;
	const unsigned k = ctx->hf[0].k;
	int rc = grow(ctx, &ctx->d_tp_local, ctx->tp_local_cap, total);
	if (rc)
		return rc;
	if (nb + 1 > ctx->tp_sums_cap) {
		cudaFree(ctx->d_tp_sums);
		cudaFreeHost(ctx->h_tp_sums);
		ctx->d_tp_sums = nullptr;
		ctx->h_tp_sums = nullptr;
		ctx->tp_sums_cap = 0;
		CUDA_TRY(ctx, cudaMalloc(&ctx->d_tp_sums, (nb + 1) * sizeof(unsigned long long)));
		CUDA_TRY(ctx, cudaMallocHost(&ctx->h_tp_sums, (nb + 1) * sizeof(unsigned long long)));
		ctx->tp_sums_cap = nb + 1;
	}
	CUDA_TRY(ctx, two_pass_scan(a, k, ctx->d_tp_local, ctx->d_tp_sums, s));
	CUDA_TRY(ctx, cudaMemcpyAsync(ctx->h_tp_sums, ctx->d_tp_sums,
			(nb + 1) * sizeof(unsigned long long), cudaMemcpyDeviceToHost, s));
	CUDA_TRY(ctx, cudaStreamSynchronize(s));
	const unsigned long long *sums = ctx->h_tp_sums;
	/* frame slots per sub-batch (8 bytes of hash each) */
	const uint64_t budget = ctx->p.max_batch_bases ? std::max<uint64_t>(ctx->p.max_batch_bases, 32)
	                                               : (512ull << 20);
	std::vector<uint64_t> cuts(1, 0);
	uint64_t most = 0;
	while (cuts.back() < nb) {
		const uint64_t b0 = cuts.back();
		uint64_t b1 = b0 + 1;
		while (b1 < nb && sums[b1 + 1] - sums[b0] <= budget)
			++b1;
		most = std::max<uint64_t>(most, sums[b1] - sums[b0]);
		cuts.push_back(b1);
	}
	if (most > ctx->tp_frames_cap) {
		cudaFree(ctx->d_tp_h0);
		cudaFree(ctx->d_tp_vmask);
		ctx->d_tp_h0 = nullptr;
		ctx->d_tp_vmask = nullptr;
		ctx->tp_frames_cap = 0;
		CUDA_TRY(ctx, cudaMalloc(&ctx->d_tp_h0, most * sizeof(uint64_t)));
		CUDA_TRY(ctx, cudaMalloc(&ctx->d_tp_vmask, (most / 32 + 1) * sizeof(uint32_t)));
		ctx->tp_frames_cap = most;
	}
	/* scans, then per sub-batch the hash pass and the filter and / or score pass */
	ctx->last.kernels += 2 + (cuts.size() - 1) * (1 + (classify ? 1 : 0) + (sa ? 1 : 0));
	for (size_t c = 0; c + 1 < cuts.size(); ++c) {
		TwoPassArgs p;
		p.t0 = cuts[c] * B;
		p.t1 = std::min(total, cuts[c + 1] * B);
		p.r_first = 0;
		p.local = ctx->d_tp_local;
		p.sums = ctx->d_tp_sums;
		p.s0 = sums[cuts[c]];
		p.k = k;
		p.h0 = ctx->d_tp_h0;
		p.vmask = ctx->d_tp_vmask;
		p.work = ctx->d_work;
		CUDA_TRY(ctx, two_pass_sub_batch(a, p, ctx->lc, s, sa, classify));
	}
	return BBT_OK;
}

/* Scratch of the bucketed path for sub-batches of up to `frames` frames and
 * nbkt buckets x nblk blocks of counts. */
static int bk_reserve(bbt_ctx *ctx, uint64_t frames, uint64_t cnt_entries)
{
	if (frames > ctx->bk_frames_cap || ctx->bk_levels > ctx->bk_pool_levels) {
		cudaFree(ctx->d_bk_vbits);
		cudaFree(ctx->d_bk_hbits);
		cudaFree(ctx->d_bk_abits);
		cudaFree(ctx->d_bk_canon);
		cudaFree(ctx->d_bk_off);
		cudaFree(ctx->d_bk_fid);
		cudaFree(ctx->d_bk_res);
		cudaFree(ctx->d_bk_btot);
		ctx->d_bk_vbits = ctx->d_bk_hbits = ctx->d_bk_abits = ctx->d_bk_off = nullptr;
		ctx->d_bk_btot = nullptr;
		ctx->d_bk_canon = nullptr;
		ctx->d_bk_fid = nullptr;
		ctx->d_bk_res = nullptr;
		ctx->bk_frames_cap = 0;
		/* whole window blocks, plus spare words for reads across the end */
		const uint64_t f = (frames + kBkWinFrames - 1) / kBkWinFrames * kBkWinFrames;
		CUDA_TRY(ctx, cudaMalloc(&ctx->d_bk_vbits, (f / 32 + 2) * sizeof(uint32_t)));
		CUDA_TRY(ctx, cudaMalloc(&ctx->d_bk_hbits, (f / 32 + 2) * sizeof(uint32_t)));
		CUDA_TRY(ctx, cudaMalloc(&ctx->d_bk_abits, (f / 32 + 2) * sizeof(uint32_t)));
		CUDA_TRY(ctx, cudaMalloc(&ctx->d_bk_canon, f * sizeof(uint64_t)));
		/* a round requests up to bk_levels tests per frame */
		const uint64_t pool = f * std::max<uint32_t>(ctx->bk_levels, 1);
		CUDA_TRY(ctx, cudaMalloc(&ctx->d_bk_off, pool * sizeof(uint32_t)));
		CUDA_TRY(ctx, cudaMalloc(&ctx->d_bk_fid, pool * sizeof(uint16_t)));
		CUDA_TRY(ctx, cudaMalloc(&ctx->d_bk_res, pool));
		CUDA_TRY(ctx, cudaMalloc(&ctx->d_bk_btot, (f / kBkWinFrames) * sizeof(uint32_t)));
		ctx->bk_frames_cap = f;
		ctx->bk_pool_levels = std::max<uint32_t>(ctx->bk_levels, 1);
	}
	if (cnt_entries > ctx->bk_cnt_cap) {
		cudaFree(ctx->d_bk_cnt);
		cudaFree(ctx->d_bk_loc);
		ctx->d_bk_cnt = ctx->d_bk_loc = nullptr;
		ctx->bk_cnt_cap = 0;
		CUDA_TRY(ctx, cudaMalloc(&ctx->d_bk_cnt, cnt_entries * sizeof(uint32_t)));
		CUDA_TRY(ctx, cudaMalloc(&ctx->d_bk_loc, cnt_entries * sizeof(uint32_t)));
		ctx->bk_cnt_cap = cnt_entries;
	}
	return BBT_OK;
}

static int bk_tmp(bbt_ctx *ctx, size_t bytes)
{
	if (bytes <= ctx->bk_tmp_cap)
		return BBT_OK;
	cudaFree(ctx->d_bk_tmp);
	ctx->d_bk_tmp = nullptr;
	ctx->bk_tmp_cap = 0;
	CUDA_TRY(ctx, cudaMalloc(&ctx->d_bk_tmp, bytes));
	ctx->bk_tmp_cap = bytes;
	return BBT_OK;
}

/* Staging slots of host batches on the bucketed path. */
constexpr uint64_t kBkSlotBases = 2ull << 30;
constexpr uint64_t kBkSlotReads = 8ull << 20;

struct BkCut {
	uint64_t r0, r1;  /* reads of the sub-batch */
	uint64_t f0, f1;  /* their frames */
};

/* Sub-batches of consecutive reads with at most `most` frames each, from the
 * frame offsets fo (device) of `total` reads: samples of fo every 4096 reads
 * come to the host (one short wait), and a sample interval above the limit is
 * read in full.  Reads with more than `most` frames on their own go to
 * `oversize`. */
static int bk_plan(bbt_ctx *ctx, const ClassifyArgs &a, const uint64_t *fo, uint64_t total,
		uint64_t most, cudaStream_t s, std::vector<BkCut> &cuts, std::vector<uint64_t> &oversize,
		uint64_t mate_end[2])
{
	const uint64_t S = 4096;
	const uint64_t ns = total / S + 1;
	if (ns + 3 > ctx->bk_samples_cap) {
		cudaFreeHost(ctx->h_bk_samples);
		cudaFree(ctx->d_bk_samples);
		ctx->h_bk_samples = nullptr;
		ctx->d_bk_samples = nullptr;
		ctx->bk_samples_cap = 0;
		CUDA_TRY(ctx, cudaMallocHost(&ctx->h_bk_samples, (ns + 3) * sizeof(uint64_t)));
		CUDA_TRY(ctx, cudaMalloc(&ctx->d_bk_samples, (ns + 3) * sizeof(uint64_t)));
		ctx->bk_samples_cap = ns + 3;
	}
	uint64_t *h = ctx->h_bk_samples;
	/* fo[0], fo[S], fo[2S], ..., then fo[total], then the end offset of each
	 * mate array: gathered on the device, one copy */
	CUDA_TRY(ctx, launch_bk_samples(fo, total, S, ctx->d_bk_samples, ns, ctx->num_sms, s));
	CUDA_TRY(ctx, launch_bk_samples(fo + total, 0, 0, ctx->d_bk_samples + ns, 1, ctx->num_sms,
			s));
	for (uint32_t m = 0; m < a.mates; ++m)
		CUDA_TRY(ctx, launch_bk_samples(a.off[m] + a.n, 0, 0, ctx->d_bk_samples + ns + 1 + m, 1,
				ctx->num_sms, s));
	CUDA_TRY(ctx, cudaMemcpyAsync(h, ctx->d_bk_samples, (ns + 1 + a.mates) * sizeof(uint64_t),
			cudaMemcpyDeviceToHost, s));
	CUDA_TRY(ctx, cudaStreamSynchronize(s));
	for (uint32_t m = 0; m < 2; ++m)
		mate_end[m] = m < a.mates ? h[ns + 1 + m] : 0;
	std::vector<uint64_t> pt(ns + 1), fv(ns + 1);
	for (uint64_t j = 0; j < ns; ++j) {
		pt[j] = j * S;
		fv[j] = h[j];
	}
	pt[ns] = total;
	fv[ns] = h[ns];
	cuts.clear();
	oversize.clear();
	uint64_t j = 0;
	std::vector<uint64_t> fine;
	while (pt[j] < total) {
		uint64_t jj = j;
		while (jj + 1 <= ns && fv[jj + 1] - fv[j] <= most)
			++jj;
		if (jj > j) {
			if (fv[jj] > fv[j])
				cuts.push_back({pt[j], pt[jj], fv[j], fv[jj]});
			j = jj;
			continue;
		}
		/* the next sample interval alone is above the limit: cut it per read */
		const uint64_t a0 = pt[j], a1 = pt[j + 1];
		fine.resize(a1 - a0 + 1);
		CUDA_TRY(ctx, cudaMemcpy(fine.data(), fo + a0, fine.size() * sizeof(uint64_t),
				cudaMemcpyDeviceToHost));
		uint64_t r = a0;
		while (r < a1) {
			uint64_t e = r;
			while (e + 1 <= a1 && fine[e + 1 - a0] - fine[r - a0] <= most)
				++e;
			if (e == r) {
				oversize.push_back(r);
				e = r + 1;
			} else if (fine[e - a0] > fine[r - a0]) {
				cuts.push_back({r, e, fine[r - a0], fine[e - a0]});
			}
			r = e;
		}
		j = j + 1;
	}
	return BBT_OK;
}

/* The bucketed probe path over one batch (STD / ORDERED modes, every scoring
 * method): per filter, sub-batches of reads, each resolved in phases and
 * rounds (bucketed.cu).  Hit words are built bit by bit: zeroed first. */
static int run_bucketed(bbt_ctx *ctx, ClassifyArgs &a, cudaStream_t s)
{
	const uint64_t total = a.n * a.mates;
	const size_t hb = a.n * ctx->words * sizeof(uint64_t);
	CUDA_TRY(ctx, cudaMemsetAsync(a.hits[0], 0, hb, s));
	if (a.mates == 2)
		CUDA_TRY(ctx, cudaMemsetAsync(a.hits[1], 0, hb, s));
	if (total == 0)
		return BBT_OK;
	if (total + 1 > ctx->bk_reads_cap) {
		cudaFree(ctx->d_bk_fo);
		cudaFree(ctx->d_bk_state);
		ctx->d_bk_fo = nullptr;
		ctx->d_bk_state = nullptr;
		ctx->bk_reads_cap = 0;
		CUDA_TRY(ctx, cudaMalloc(&ctx->d_bk_fo, (total + 1) * sizeof(uint64_t)));
		CUDA_TRY(ctx, cudaMalloc(&ctx->d_bk_state, total + 1));
		ctx->bk_reads_cap = total + 1;
	}
	const uint64_t most = std::max<uint64_t>(ctx->bk_max_frames, kBkWinFrames);
	size_t scan_bytes = 0;
	CUDA_TRY(ctx, cub::DeviceScan::InclusiveSum(nullptr, scan_bytes, ctx->d_bk_fo + 1,
			ctx->d_bk_fo + 1, total, s));
	int rc = bk_tmp(ctx, scan_bytes);
	if (rc)
		return rc;
	const uint32_t levels = std::max<uint32_t>(ctx->bk_levels, 1);
	std::vector<BkCut> cuts;
	std::vector<uint64_t> oversize;
	PackedBases pk[2];
	memset(pk, 0, sizeof pk);
	bool have_pk = false;
	unsigned cur_k = 0;
	for (uint32_t f = 0; f < ctx->nf; ++f) {
		const FilterDev &F = ctx->hf[f];
		if (F.k != cur_k) {
			cur_k = F.k;
			CUDA_TRY(ctx, cudaMemsetAsync(ctx->d_bk_fo, 0, sizeof(uint64_t), s));
			CUDA_TRY(ctx, launch_bk_frame_counts(a, cur_k, ctx->d_bk_fo + 1, ctx->num_sms, s));
			CUDA_TRY(ctx, cub::DeviceScan::InclusiveSum(ctx->d_bk_tmp, scan_bytes,
					ctx->d_bk_fo + 1, ctx->d_bk_fo + 1, total, s));
			uint64_t mate_end[2];
			rc = bk_plan(ctx, a, ctx->d_bk_fo, total, most, s, cuts, oversize, mate_end);
			if (rc)
				return rc;
			ctx->last.kernels += 2 + a.mates;
			/* the bases as 2-bit codes: packed batches as they are, ASCII
			 * batches packed once per call */
			for (uint32_t m = 0; !have_pk && m < a.mates; ++m) {
				const uint64_t len = mate_end[m] - a.off_base[m];
				if (a.packed) {
					pk[m].words = reinterpret_cast<const uint32_t *>(a.seq[m]);
					pk[m].nwords = (len + 15) / 16;
					pk[m].valid = a.valid[m];
					pk[m].nvalid = a.valid[m] ? (len + 31) / 32 : 0;
					continue;
				}
				rc = grow(ctx, &ctx->d_bk_codes[m], ctx->bk_codes_cap[m], 2 * (len / 32 + 2));
				if (!rc)
					rc = grow(ctx, &ctx->d_bk_cvalid[m], ctx->bk_cvalid_cap[m], len / 32 + 2);
				if (rc)
					return rc;
				CUDA_TRY(ctx, launch_bk_pack(a.seq[m], len, ctx->d_bk_codes[m],
						ctx->d_bk_cvalid[m], ctx->num_sms, s));
				pk[m].words = ctx->d_bk_codes[m];
				pk[m].nwords = 2 * (len / 32 + 2);
				pk[m].valid = ctx->d_bk_cvalid[m];
				pk[m].nvalid = len / 32 + 2;
				ctx->last.kernels += 1;
			}
			have_pk = true;
		}
		CUDA_TRY(ctx, cudaMemsetAsync(ctx->d_bk_state, 0, total, s));
		for (uint64_t r : oversize) /* the direct kernel's, below */
			CUDA_TRY(ctx, cudaMemsetAsync(ctx->d_bk_state + r, 1, 1, s));
		unsigned bshift = std::max<unsigned>(ctx->bk_bshift, 12);
		while (((F.m + (1ull << bshift) - 1) >> bshift) > 2048)
			++bshift;
		const uint32_t nbkt = (uint32_t)((F.m + (1ull << bshift) - 1) >> bshift);
		const uint32_t split = std::min<uint32_t>(ctx->bk_phase_split, kBkPhaseDen);
		std::vector<std::pair<uint32_t, uint32_t> > phases;
		if (split > 0 && split < kBkPhaseDen)
			phases = {{0, split}, {split, kBkPhaseDen}};
		else
			phases = {{0, kBkPhaseDen}};
		/* rounds of up to `levels` hash levels each */
		std::vector<std::pair<uint32_t, uint32_t> > rounds;
		for (uint32_t l = 0; l < F.h;) {
			const uint32_t nl = std::min<uint32_t>(levels, F.h - l);
			rounds.push_back({l, nl});
			l += nl;
		}
		for (const BkCut &c : cuts) {
			const uint64_t T = c.f1 - c.f0;
			const uint32_t nblk = (uint32_t)((T + kBkWinFrames - 1) / kBkWinFrames);
			rc = bk_reserve(ctx, T, (uint64_t)nbkt * nblk);
			if (rc)
				return rc;
			const uint64_t words = (T + 31) / 32 + 2;
			CUDA_TRY(ctx, cudaMemsetAsync(ctx->d_bk_vbits, 0, words * sizeof(uint32_t), s));
			CUDA_TRY(ctx, cudaMemsetAsync(ctx->d_bk_hbits, 0, words * sizeof(uint32_t), s));
			BucketArgs b;
			memset(&b, 0, sizeof b);
			b.a = a;
			b.pk[0] = pk[0];
			b.pk[1] = pk[1];
			b.f = F;
			b.fbit = f;
			b.r0 = c.r0;
			b.nr = c.r1 - c.r0;
			b.fo = ctx->d_bk_fo;
			b.fo0 = c.f0;
			b.T = T;
			b.nblk = nblk;
			b.vbits = ctx->d_bk_vbits;
			b.hbits = ctx->d_bk_hbits;
			b.abits = ctx->d_bk_abits;
			b.canon = ctx->d_bk_canon;
			b.state = ctx->d_bk_state;
			b.ph_min = ctx->bk_phase_min;
			b.nbkt = nbkt;
			b.bshift = bshift;
			b.cnt = ctx->d_bk_cnt;
			b.loc = ctx->d_bk_loc;
			b.cap = (uint64_t)kBkWinFrames * ctx->bk_pool_levels;
			b.req_off = ctx->d_bk_off;
			b.req_fid = ctx->d_bk_fid;
			b.res = ctx->d_bk_res;
			b.btot = ctx->d_bk_btot;
			b.issued = a.probes;
			b.next = ctx->d_work;
			for (const auto &ph : phases) {
				b.ph_lo = ph.first;
				b.ph_hi = ph.second;
				for (size_t ri = 0; ri < rounds.size(); ++ri) {
					b.level = rounds[ri].first;
					b.nlevels = rounds[ri].second;
					if (ri == 0)
						CUDA_TRY(ctx, launch_bk_hash(b, s));
					else
						CUDA_TRY(ctx, launch_bk_emit(b, s));
					CUDA_TRY(ctx, launch_bk_resolve(b, ctx->num_sms, s));
				}
				CUDA_TRY(ctx, launch_bk_apply(b, s));
				CUDA_TRY(ctx, launch_bk_walk(b, ctx->num_sms, s));
				ctx->last.kernels += 2 * (uint32_t)rounds.size() + 2;
			}
		}
	}
	/* reads too long for any sub-batch: the persistent kernel, every filter */
	for (uint64_t r : oversize) {
		const uint32_t mate = r >= a.n ? 1u : 0u;
		const uint64_t i = r - (mate ? a.n : 0);
		ClassifyArgs one = a;
		one.seq[0] = one.seq[1] = a.seq[mate];
		one.valid[0] = one.valid[1] = a.valid[mate];
		one.off[0] = one.off[1] = a.off[mate] + i;
		one.off_base[0] = one.off_base[1] = a.off_base[mate];
		one.dust[0] = one.dust[1] = a.dust[mate];
		one.hits[0] = a.hits[mate] + i * ctx->words;
		one.hits[1] = nullptr;
		one.n = 1;
		one.mates = 1;
		one.order = nullptr;
		LaunchConfig lc = ctx->lc;
		lc.path = BBT_PATH_PERSISTENT;
		CUDA_TRY(ctx, cudaMemsetAsync(ctx->d_work, 0, sizeof(unsigned long long), s));
		CUDA_TRY(ctx, launch_classify(one, lc, s));
		ctx->last.kernels += 1;
	}
	return BBT_OK;
}

/* -D: the SDUST masks of a batch's reads (dust.cu) into ctx->d_dust, set in
 * a.dust.  mate_bases: bases of each mate array counted from its off_base. */
static int run_dust(bbt_ctx *ctx, ClassifyArgs &a, const uint64_t *mate_bases, cudaStream_t s)
{
	DustArgs d;
	memset(&d, 0, sizeof d);
	for (uint32_t m = 0; m < a.mates; ++m) {
		const uint64_t words = mate_bases[m] / 32 + 2;
		int rc = grow(ctx, &ctx->d_dust[m], ctx->dust_words_cap[m], words);
		if (rc)
			return rc;
		CUDA_TRY(ctx, cudaMemsetAsync(ctx->d_dust[m], 0, words * sizeof(uint32_t), s));
		d.seq[m] = a.seq[m];
		d.off[m] = a.off[m];
		d.off_base[m] = a.off_base[m];
		d.mask[m] = ctx->d_dust[m];
	}
	int rc = grow(ctx, &ctx->d_dust_redo, ctx->dust_redo_cap, a.n * a.mates);
	if (rc)
		return rc;
	CUDA_TRY(ctx, cudaMemsetAsync(ctx->d_dust_cnt, 0, sizeof(unsigned long long), s));
	d.n = a.n;
	d.mates = a.mates;
	d.T = ctx->dust_T;
	d.W = ctx->dust_W;
	d.redo = ctx->d_dust_redo;
	d.redo_count = ctx->d_dust_cnt;
	d.failed = ctx->d_dust_cnt + 1;
	d.scratch = ctx->d_dust_scratch;
	d.scratch_per_thread = ctx->dust_per_thread;
	CUDA_TRY(ctx, launch_dust_pass1(d, ctx->num_sms, s));
	CUDA_TRY(ctx, launch_dust_pass2(d, ctx->dust_threads2, s));
	a.dust[0] = ctx->d_dust[0];
	a.dust[1] = a.mates == 2 ? ctx->d_dust[1] : nullptr;
	ctx->last.kernels += 2;
	return BBT_OK;
}

/* -D: after the stream has finished a call's batches, fail the call if a
 * read's masking did not fit pass 2's scratch. */
static int dust_check(bbt_ctx *ctx)
{
	unsigned long long failed = 0;
	CUDA_TRY(ctx, cudaMemcpy(&failed, ctx->d_dust_cnt + 1, sizeof failed, cudaMemcpyDeviceToHost));
	if (failed)
		return fail(ctx, BBT_ERR_UNSUPPORTED,
				"DUST: " + std::to_string(failed) + " read(s) held more pending low-complexity "
				"intervals than the masking kernel's scratch");
	return BBT_OK;
}

/* classify + summarize one staged or device-resident batch on stream s;
 * scores (optional, per mate array): evalScore of every filter */
static int run_kernels(bbt_ctx *ctx, ClassifyArgs &a, uint32_t *d_cat, cudaStream_t s,
		double *const *scores = nullptr, const uint64_t *mate_bases = nullptr)
{
	ctx->last.kernels = 2; /* classification (counted below for two-pass) + summary */
	if (ctx->dust) {
		if (!mate_bases)
			return fail(ctx, BBT_ERR_UNSUPPORTED, "DUST masking needs the batch's base counts");
		int rc = run_dust(ctx, a, mate_bases, s);
		if (rc)
			return rc;
	}
	ScoreArgs sa;
	sa.scores[0] = scores ? scores[0] : nullptr;
	sa.scores[1] = scores && a.mates == 2 ? scores[1] : nullptr;
	sa.fpr = ctx->d_fpr;
	sa.besthit = 0;
	bool want_scores = sa.scores[0] || sa.scores[1];
	const bool two_pass = ctx->lc.path == BBT_PATH_FILTER_MAJOR && ctx->same_k;
	CUDA_TRY(ctx, cudaEventRecord(ctx->ev_k0, s));
	if (two_pass && (ctx->mode == BBT_MODE_BESTHIT || want_scores)) {
		/* filter-major score pass (and filter pass for the hits unless
		 * BESTHIT, whose hits come from the scores) */
		ScoreArgs ps = sa;
		if (ctx->mode == BBT_MODE_BESTHIT && !want_scores) {
			const uint64_t need = a.n * ctx->nf;
			if (need > ctx->tmp_scores_cap) {
				cudaFree(ctx->d_tmp_scores[0]);
				cudaFree(ctx->d_tmp_scores[1]);
				ctx->d_tmp_scores[0] = ctx->d_tmp_scores[1] = nullptr;
				ctx->tmp_scores_cap = 0;
				CUDA_TRY(ctx, cudaMalloc(&ctx->d_tmp_scores[0], need * sizeof(double)));
				CUDA_TRY(ctx, cudaMalloc(&ctx->d_tmp_scores[1], need * sizeof(double)));
				ctx->tmp_scores_cap = need;
			}
			ps.scores[0] = ctx->d_tmp_scores[0];
			ps.scores[1] = a.mates == 2 ? ctx->d_tmp_scores[1] : nullptr;
		}
		const bool classify = ctx->mode != BBT_MODE_BESTHIT;
		if (classify) {
			const size_t hb = a.n * ctx->words * sizeof(uint64_t);
			CUDA_TRY(ctx, cudaMemsetAsync(a.hits[0], 0, hb, s));
			if (a.mates == 2)
				CUDA_TRY(ctx, cudaMemsetAsync(a.hits[1], 0, hb, s));
		}
		ctx->last.kernels -= 1; /* the passes count themselves */
		int rc = run_two_pass(ctx, a, s, &ps, classify);
		if (rc)
			return rc;
		if (!classify) {
			CUDA_TRY(ctx, launch_best_hits(a, ps.scores, ctx->num_sms, s));
			ctx->last.kernels += 1;
		}
		want_scores = false; /* done */
	} else if (ctx->mode == BBT_MODE_BESTHIT) {
		/* the hit words are the filters of the largest score */
		sa.besthit = 1;
		CUDA_TRY(ctx, launch_scores(a, sa, ctx->lc, s));
	} else if (ctx->lc.path == BBT_PATH_BUCKETED && !want_scores) {
		ctx->last.kernels -= 1; /* the passes count themselves */
		int rc = run_bucketed(ctx, a, s);
		if (rc)
			return rc;
	} else if (two_pass) {
		/* accepted (filter, read) items OR their bit into zeroed words */
		const size_t hb = a.n * ctx->words * sizeof(uint64_t);
		CUDA_TRY(ctx, cudaMemsetAsync(a.hits[0], 0, hb, s));
		if (a.mates == 2)
			CUDA_TRY(ctx, cudaMemsetAsync(a.hits[1], 0, hb, s));
		ctx->last.kernels -= 1; /* the passes count themselves */
		int rc = run_two_pass(ctx, a, s);
		if (rc)
			return rc;
	} else {
		LaunchConfig lc = ctx->lc;
		if (lc.path == BBT_PATH_FILTER_MAJOR)
			lc.path = BBT_PATH_PERSISTENT; /* filters of different k */
		if (lc.path != BBT_PATH_PLAIN)
			CUDA_TRY(ctx, cudaMemsetAsync(ctx->d_work, 0, sizeof(unsigned long long), s));
		if (lc.path != BBT_PATH_PLAIN && ctx->long_bases) {
			int rc = grow(ctx, &ctx->d_order, ctx->order_cap, a.n * a.mates);
			if (rc)
				return rc;
			CUDA_TRY(ctx, cudaMemsetAsync(ctx->d_order_cnt, 0, 2 * sizeof(unsigned long long), s));
			CUDA_TRY(ctx, launch_long_first(a, ctx->long_bases, ctx->d_order, ctx->d_order_cnt,
					ctx->num_sms, s));
			a.order = ctx->d_order;
			ctx->last.kernels += 1;
		}
		CUDA_TRY(ctx, launch_classify(a, lc, s));
	}
	if (want_scores && ctx->mode != BBT_MODE_BESTHIT) {
		CUDA_TRY(ctx, launch_scores(a, sa, ctx->lc, s));
		ctx->last.kernels += 1;
	}
	CUDA_TRY(ctx, cudaEventRecord(ctx->ev_k1, s));
	CUDA_TRY(ctx, launch_summarize(a.hits[0], a.mates == 2 ? a.hits[1] : nullptr, a.n, ctx->nf,
			ctx->words, ctx->p.inclusive, ctx->mode == BBT_MODE_ORDERED, d_cat, ctx->d_counts,
			ctx->num_sms, s));
	return BBT_OK;
}

static int ensure_tmp_hits(bbt_ctx *ctx, uint64_t n)
{
	if (n <= ctx->tmp_hits_cap)
		return BBT_OK;
	cudaFree(ctx->d_tmp_hits[0]);
	cudaFree(ctx->d_tmp_hits[1]);
	ctx->d_tmp_hits[0] = ctx->d_tmp_hits[1] = nullptr;
	ctx->tmp_hits_cap = 0;
	CUDA_TRY(ctx, cudaMalloc(&ctx->d_tmp_hits[0], n * ctx->words * sizeof(uint64_t)));
	CUDA_TRY(ctx, cudaMalloc(&ctx->d_tmp_hits[1], n * ctx->words * sizeof(uint64_t)));
	ctx->tmp_hits_cap = n;
	return BBT_OK;
}

static int classify_device(bbt_ctx *ctx, const bbt_batch *b, bbt_result *r, cudaStream_t s,
		double *const *scores = nullptr)
{
	const bool paired = b->seq2 != nullptr;
	if (ctx->p.scoring == BBT_SCORE_BINOMIAL && ctx->mode != BBT_MODE_BESTHIT &&
			!ctx->capturing) {
		/* the thresholds of the batch's read lengths (a short host wait) */
		std::vector<uint64_t> lens;
		int rc = device_lengths(ctx, b, s, lens);
		if (!rc)
			rc = ensure_bthres(ctx, lens);
		if (rc)
			return rc;
	}
	ClassifyArgs a = base_args(ctx);
	a.seq[0] = (const uint8_t *)b->seq;
	a.off[0] = b->offsets;
	a.seq[1] = (const uint8_t *)(paired ? b->seq2 : b->seq);
	a.off[1] = paired ? b->offsets2 : b->offsets;
	a.packed = b->encoding == BBT_BASES_2BIT;
	if (a.packed && ctx->dust)
		return fail(ctx, BBT_ERR_UNSUPPORTED, "DUST masking reads ASCII bases; pass the batch "
				"as BBT_BASES_ASCII");
	a.valid[0] = a.packed ? b->valid : nullptr;
	a.valid[1] = a.packed ? (paired ? b->valid2 : b->valid) : nullptr;
	a.n = b->n_reads;
	a.mates = paired ? 2 : 1;
	if (!r->hits || (paired && !r->hits2)) {
		int rc = ensure_tmp_hits(ctx, b->n_reads);
		if (rc)
			return rc;
	}
	a.hits[0] = r->hits ? r->hits : ctx->d_tmp_hits[0];
	a.hits[1] = paired ? (r->hits2 ? r->hits2 : ctx->d_tmp_hits[1]) : nullptr;
	uint64_t mate_bases[2] = {0, 0};
	if (ctx->dust) {
		if (ctx->capturing)
			return fail(ctx, BBT_ERR_UNSUPPORTED, "DUST masking cannot be captured in a graph");
		/* the mask arrays are sized by the batch's bases (a short host wait) */
		for (uint32_t m = 0; m < a.mates; ++m) {
			uint64_t ends[2];
			CUDA_TRY(ctx, cudaMemcpyAsync(&ends[0], a.off[m], sizeof(uint64_t),
					cudaMemcpyDeviceToHost, s));
			CUDA_TRY(ctx, cudaMemcpyAsync(&ends[1], a.off[m] + b->n_reads, sizeof(uint64_t),
					cudaMemcpyDeviceToHost, s));
			CUDA_TRY(ctx, cudaStreamSynchronize(s));
			a.off_base[m] = ends[0];
			mate_bases[m] = ends[1] - ends[0];
			a.seq[m] += ends[0]; /* bases indexed from offsets[0] */
		}
		CUDA_TRY(ctx, cudaMemsetAsync(ctx->d_dust_cnt + 1, 0, sizeof(unsigned long long), s));
	}
	CUDA_TRY(ctx, cudaEventRecord(ctx->ev_start, s));
	int rc = run_kernels(ctx, a, r->category, s, scores, mate_bases);
	if (rc)
		return rc;
	CUDA_TRY(ctx, cudaEventRecord(ctx->ev_stop, s));
	if (ctx->dust) {
		CUDA_TRY(ctx, cudaStreamSynchronize(s));
		rc = dust_check(ctx);
		if (rc)
			return rc;
	}
	ctx->reads_seen += b->n_reads;
	ctx->last.reads = b->n_reads * a.mates;
	return BBT_OK;
}

/* Host batches: split into sub-batches that fit the staging slots; copies in
 * (h2d stream), kernels (ctx->stream) and copies out (d2h stream) of
 * consecutive sub-batches overlap, two slots deep. */
static int classify_host(bbt_ctx *ctx, const bbt_batch *b, bbt_result *r,
		double *const *scores = nullptr)
{
	const bool paired = b->seq2 != nullptr;
	const uint64_t n = b->n_reads;
	const bool packed = b->encoding == BBT_BASES_2BIT;
	const bool want_scores = scores && (scores[0] || (paired && scores[1]));
	if (ctx->lc.path == BBT_PATH_BUCKETED && !ctx->p.max_batch_bases &&
			!ctx->p.max_batch_reads && ctx->cap_bases < kBkSlotBases && n > ctx->cap_reads) {
		/* the bucketed path sweeps the filter once per round of a slot load:
		 * large loads keep those sweeps few */
		for (Slot &sl : ctx->slot)
			if (sl.used)
				CUDA_TRY(ctx, cudaEventSynchronize(sl.done));
		CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
		ctx->cap_bases = kBkSlotBases;
		ctx->cap_reads = kBkSlotReads;
		for (Slot &sl : ctx->slot) {
			flush_slot(sl);
			sl.used = false;
			int rc = alloc_slot(ctx, sl, ctx->cap_bases, ctx->cap_reads);
			if (rc)
				return rc;
		}
	}
	if (want_scores) {
		/* per-slot score arrays of cap_reads reads */
		for (Slot &sl : ctx->slot) {
			if (sl.scores_cap >= ctx->cap_reads)
				continue;
			for (int m = 0; m < 2; ++m) {
				cudaFree(sl.d_scores[m]);
				sl.d_scores[m] = nullptr;
			}
			sl.scores_cap = 0;
			for (int m = 0; m < 2; ++m)
				CUDA_TRY(ctx, cudaMalloc(&sl.d_scores[m],
						ctx->cap_reads * ctx->nf * sizeof(double)));
			sl.scores_cap = ctx->cap_reads;
		}
	}
	if (ctx->p.scoring == BBT_SCORE_BINOMIAL && ctx->mode != BBT_MODE_BESTHIT) {
		int rc = ensure_bthres(ctx, host_lengths(b->offsets, paired ? b->offsets2 : nullptr, n));
		if (rc)
			return rc;
	}
	/* staged copies left by a call that failed part way belong to that call */
	for (Slot &sl : ctx->slot) {
		if (sl.used)
			CUDA_TRY(ctx, cudaEventSynchronize(sl.done));
		sl.pending.clear();
		sl.used = false;
	}
	uint64_t i0 = 0;
	int which = 0;
	/* at least about eight slot loads per call (of 64k reads or more), so
	 * that a batch that fits one slot still overlaps its copies with its
	 * kernels */
	const uint64_t step = std::min<uint64_t>(ctx->cap_reads,
			std::max<uint64_t>(1ull << 16, (n + 7) / 8));
	const bool out_pinned[5] = {r->hits && host_pinned(r->hits),
			paired && r->hits2 && host_pinned(r->hits2),
			r->category && host_pinned(r->category),
			want_scores && scores[0] && host_pinned(scores[0]),
			want_scores && paired && scores[1] && host_pinned(scores[1])};
	if (ctx->dust)
		CUDA_TRY(ctx, cudaMemsetAsync(ctx->d_dust_cnt + 1, 0, sizeof(unsigned long long),
				ctx->stream));
	CUDA_TRY(ctx, cudaEventRecord(ctx->ev_start, ctx->stream));
	while (i0 < n) {
		/* largest i1 with bases and reads inside the slot capacity */
		uint64_t i1 = std::min(n, i0 + step);
		auto bases = [&](uint64_t lo, uint64_t hi) {
			uint64_t x = b->offsets[hi] - b->offsets[lo];
			if (paired)
				x = std::max(x, b->offsets2[hi] - b->offsets2[lo]);
			return x;
		};
		if (bases(i0, i1) > ctx->cap_bases) {
			uint64_t lo = i0 + 1, hi = i1;
			while (lo < hi) {
				uint64_t mid = (lo + hi + 1) / 2;
				if (bases(i0, mid) <= ctx->cap_bases)
					lo = mid;
				else
					hi = mid - 1;
			}
			i1 = lo;
			if (bases(i0, i1) > ctx->cap_bases) {
				/* one read longer than the staging area: grow both slots */
				for (Slot &s : ctx->slot) {
					if (s.used)
						CUDA_TRY(ctx, cudaEventSynchronize(s.done));
					flush_slot(s);
					s.used = false;
				}
				uint64_t need = bases(i0, i1);
				for (Slot &s : ctx->slot) {
					int rc = alloc_slot(ctx, s, need, ctx->cap_reads);
					if (rc)
						return rc;
				}
				ctx->cap_bases = need;
			}
		}
		Slot &s = ctx->slot[which];
		if (s.used)
			CUDA_TRY(ctx, cudaEventSynchronize(s.done));
		flush_slot(s);
		const uint64_t cnt = i1 - i0;
		ClassifyArgs a = base_args(ctx);
		a.n = cnt;
		a.mates = paired ? 2 : 1;
		uint64_t mate_bases[2] = {0, 0};
		a.packed = packed;
		for (int m = 0; m < (paired ? 2 : 1); ++m) {
			const char *seq = m ? b->seq2 : b->seq;
			const uint64_t *off = m ? b->offsets2 : b->offsets;
			const uint64_t lo = off[i0], hi = off[i1];
			mate_bases[m] = hi - lo;
			if (packed) {
				/* whole words from a 32-base boundary, so that code words and
				 * validity words share the slot's base index */
				const uint64_t lo_a = lo & ~31ull;
				const uint32_t *valid = m ? b->valid2 : b->valid;
				if (hi > lo) {
					const uint64_t w0 = lo_a / 16, w1 = (hi + 15) / 16;
					CUDA_TRY(ctx, cudaMemcpyAsync(s.d_seq[m],
							reinterpret_cast<const uint32_t *>(seq) + w0, (w1 - w0) * 4,
							cudaMemcpyHostToDevice, ctx->h2d));
					if (valid) {
						const uint64_t v0 = lo_a / 32, v1 = (hi + 31) / 32;
						CUDA_TRY(ctx, cudaMemcpyAsync(s.d_valid[m], valid + v0, (v1 - v0) * 4,
								cudaMemcpyHostToDevice, ctx->h2d));
					}
				}
				a.valid[m] = valid ? s.d_valid[m] : nullptr;
				a.off_base[m] = lo_a;
			} else {
				if (hi > lo)
					CUDA_TRY(ctx, cudaMemcpyAsync(s.d_seq[m], seq + lo, hi - lo,
							cudaMemcpyHostToDevice, ctx->h2d));
				a.off_base[m] = lo;
			}
			CUDA_TRY(ctx, cudaMemcpyAsync(s.d_off[m], off + i0, (cnt + 1) * sizeof(uint64_t),
					cudaMemcpyHostToDevice, ctx->h2d));
			a.seq[m] = s.d_seq[m];
			a.off[m] = s.d_off[m];
			a.hits[m] = s.d_hits[m];
		}
		if (!paired) {
			a.seq[1] = a.seq[0];
			a.valid[1] = a.valid[0];
			a.off[1] = a.off[0];
			a.off_base[1] = a.off_base[0];
			a.hits[1] = nullptr;
		}
		CUDA_TRY(ctx, cudaEventRecord(s.copied, ctx->h2d));
		CUDA_TRY(ctx, cudaStreamWaitEvent(ctx->stream, s.copied, 0));
		double *slot_scores[2] = {nullptr, nullptr};
		if (want_scores) {
			slot_scores[0] = scores[0] ? s.d_scores[0] : nullptr;
			slot_scores[1] = paired && scores[1] ? s.d_scores[1] : nullptr;
		}
		int rc = run_kernels(ctx, a, s.d_cat, ctx->stream, want_scores ? slot_scores : nullptr,
				mate_bases);
		if (rc)
			return rc;
		CUDA_TRY(ctx, cudaEventRecord(s.computed, ctx->stream));
		CUDA_TRY(ctx, cudaStreamWaitEvent(ctx->d2h, s.computed, 0));
		/* results: straight into pinned destinations, through the slot's
		 * pinned staging buffer into pageable ones */
		struct Out {
			void *dst;
			const void *src;
			size_t bytes;
			bool pinned;
		} outs[5];
		int no = 0;
		const size_t hb = cnt * ctx->words * sizeof(uint64_t);
		if (r->hits)
			outs[no++] = {r->hits + i0 * ctx->words, s.d_hits[0], hb, out_pinned[0]};
		if (paired && r->hits2)
			outs[no++] = {r->hits2 + i0 * ctx->words, s.d_hits[1], hb, out_pinned[1]};
		if (r->category)
			outs[no++] = {r->category + i0, s.d_cat, cnt * sizeof(uint32_t), out_pinned[2]};
		for (int m = 0; m < 2; ++m)
			if (slot_scores[m])
				outs[no++] = {scores[m] + i0 * ctx->nf, slot_scores[m],
						cnt * ctx->nf * sizeof(double), out_pinned[3 + m]};
		size_t staged = 0;
		for (int o = 0; o < no; ++o)
			if (!outs[o].pinned)
				staged += (outs[o].bytes + 255) & ~(size_t)255;
		if (staged > s.stage_cap) {
			cudaFreeHost(s.h_stage);
			s.h_stage = nullptr;
			s.stage_cap = 0;
			CUDA_TRY(ctx, cudaMallocHost(&s.h_stage, staged));
			s.stage_cap = staged;
		}
		size_t at = 0;
		for (int o = 0; o < no; ++o) {
			if (outs[o].pinned) {
				CUDA_TRY(ctx, cudaMemcpyAsync(outs[o].dst, outs[o].src, outs[o].bytes,
						cudaMemcpyDeviceToHost, ctx->d2h));
			} else {
				CUDA_TRY(ctx, cudaMemcpyAsync(s.h_stage + at, outs[o].src, outs[o].bytes,
						cudaMemcpyDeviceToHost, ctx->d2h));
				s.pending.push_back({outs[o].dst, at, outs[o].bytes});
				at += (outs[o].bytes + 255) & ~(size_t)255;
			}
		}
		CUDA_TRY(ctx, cudaEventRecord(s.done, ctx->d2h));
		s.used = true;
		which ^= 1;
		i0 = i1;
	}
	CUDA_TRY(ctx, cudaEventRecord(ctx->ev_stop, ctx->stream));
	CUDA_TRY(ctx, cudaStreamSynchronize(ctx->d2h));
	CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
	for (Slot &s : ctx->slot) {
		flush_slot(s);
		s.used = false;
	}
	if (ctx->dust) {
		int rc = dust_check(ctx);
		if (rc)
			return rc;
	}
	ctx->reads_seen += n;
	ctx->last.reads = n * (paired ? 2 : 1);
	return BBT_OK;
}

/* A host batch over this context's devices: contiguous shards of reads in
 * proportion to the devices, classified concurrently (one host thread per
 * replica), results written in place; each context adds its shard to its own
 * summary counters, which bbt_summary adds up. */
static int classify_host_devices(bbt_ctx *ctx, const bbt_batch *b, bbt_result *r,
		double *const *scores)
{
	const size_t nd = ctx->peers.size() + 1;
	const uint64_t n = b->n_reads;
	std::vector<bbt_ctx *> c(nd);
	c[0] = ctx;
	for (size_t i = 1; i < nd; ++i)
		c[i] = ctx->peers[i - 1];
	std::vector<int> rcs(nd, BBT_OK);
	auto shard = [&](size_t d) {
		const uint64_t i0 = n * d / nd, i1 = n * (d + 1) / nd;
		bbt_batch sb = *b;
		sb.offsets = b->offsets + i0;
		if (b->offsets2)
			sb.offsets2 = b->offsets2 + i0;
		sb.n_reads = i1 - i0;
		bbt_result sr = *r;
		if (r->hits)
			sr.hits = r->hits + i0 * ctx->words;
		if (r->hits2)
			sr.hits2 = r->hits2 + i0 * ctx->words;
		if (r->category)
			sr.category = r->category + i0;
		double *sc[2] = {nullptr, nullptr};
		if (scores) {
			sc[0] = scores[0] ? scores[0] + i0 * ctx->nf : nullptr;
			sc[1] = scores[1] ? scores[1] + i0 * ctx->nf : nullptr;
		}
		cudaError_t e = cudaSetDevice(c[d]->dev);
		rcs[d] = e != cudaSuccess ? cuda_fail(c[d], e, "cudaSetDevice")
		                          : classify_host(c[d], &sb, &sr, scores ? sc : nullptr);
	};
	std::vector<std::thread> th;
	for (size_t d = 1; d < nd; ++d)
		th.emplace_back(shard, d);
	shard(0);
	for (std::thread &t : th)
		t.join();
	cudaSetDevice(ctx->dev);
	for (size_t d = 0; d < nd; ++d)
		if (rcs[d])
			return d ? fail(ctx, rcs[d], c[d]->err) : rcs[d];
	return BBT_OK;
}

static int classify_batch(bbt_ctx *ctx, const bbt_batch *batch, bbt_result *result,
		void *stream, double *const *scores, const char *who)
{
	if (!ctx || !batch || !result)
		return fail(ctx, BBT_ERR_ARG, std::string(who) + ": null argument");
	if (batch->n_reads == 0)
		return BBT_OK;
	if (!batch->seq || !batch->offsets || (batch->seq2 && !batch->offsets2))
		return fail(ctx, BBT_ERR_ARG, std::string(who) + ": missing sequence or offsets");
	if (batch->location != result->location)
		return fail(ctx, BBT_ERR_ARG,
				std::string(who) + ": batch and result must both be host or both device");
	if (batch->encoding != BBT_BASES_ASCII && batch->encoding != BBT_BASES_2BIT)
		return fail(ctx, BBT_ERR_ARG, std::string(who) + ": unknown base encoding");
	if (batch->encoding == BBT_BASES_2BIT) {
		if ((reinterpret_cast<uintptr_t>(batch->seq) & 3u) ||
				(batch->seq2 && (reinterpret_cast<uintptr_t>(batch->seq2) & 3u)))
			return fail(ctx, BBT_ERR_ARG, std::string(who) + ": 2-bit code words must be "
					"4-byte aligned");
		if (ctx->dust)
			return fail(ctx, BBT_ERR_UNSUPPORTED, std::string(who) + ": DUST masking reads "
					"ASCII bases; pass the batch as BBT_BASES_ASCII");
	}
	CUDA_TRY(ctx, cudaSetDevice(ctx->dev));
	if (batch->location == BBT_DEVICE) {
		cudaStream_t s = stream ? (cudaStream_t)stream : ctx->stream;
		return classify_device(ctx, batch, result, s, scores);
	}
	if (batch->location != BBT_HOST)
		return fail(ctx, BBT_ERR_ARG, std::string(who) + ": location must be BBT_HOST or BBT_DEVICE");
	if (!ctx->peers.empty() && batch->n_reads >= 2 * (ctx->peers.size() + 1))
		return classify_host_devices(ctx, batch, result, scores);
	return classify_host(ctx, batch, result, scores);
}

extern "C" int bbt_classify_batch(bbt_ctx *ctx, const bbt_batch *batch, bbt_result *result,
		void *stream)
{
	return classify_batch(ctx, batch, result, stream, nullptr, "bbt_classify_batch");
}

extern "C" int bbt_classify_batch_scores(bbt_ctx *ctx, const bbt_batch *batch,
		bbt_result *result, double *scores, double *scores2, void *stream)
{
	if (ctx && batch && batch->seq2 && scores2 == nullptr && scores != nullptr)
		return fail(ctx, BBT_ERR_ARG, "bbt_classify_batch_scores: pairs need scores2 too");
	double *sc[2] = {scores, batch && batch->seq2 ? scores2 : nullptr};
	return classify_batch(ctx, batch, result, stream, sc, "bbt_classify_batch_scores");
}

static int set_dust_one(bbt_ctx *ctx, int on, unsigned T, unsigned W)
{
	if (!ctx)
		return BBT_ERR_ARG;
	if (!on) {
		ctx->dust = false;
		return BBT_OK;
	}
	if (W < 3 || W > (unsigned)kDustMaxWindow)
		return fail(ctx, BBT_ERR_ARG, "bbt_set_dust: the window W must be in [3, " +
				std::to_string(kDustMaxWindow) + "]");
	if (T > 100000)
		return fail(ctx, BBT_ERR_ARG, "bbt_set_dust: T must be at most 100000");
	CUDA_TRY(ctx, cudaSetDevice(ctx->dev));
	CUDA_TRY(ctx, cudaDeviceSynchronize());
	/* pass-2 scratch: any read's perfect intervals fit in W^2 + 2W + 64 entries;
	 * as many threads as fit in 256 MB (at least 32) */
	const uint64_t per = (uint64_t)W * W + 2ull * W + 64;
	const uint64_t bytes_per = per * dust_perfect_bytes();
	uint64_t threads = (256ull << 20) / bytes_per;
	threads = std::max<uint64_t>(32, std::min<uint64_t>(2048, threads / 32 * 32));
	if (per != ctx->dust_per_thread || threads != ctx->dust_threads2) {
		cudaFree(ctx->d_dust_scratch);
		ctx->d_dust_scratch = nullptr;
		ctx->dust_per_thread = 0;
		ctx->dust_threads2 = 0;
		CUDA_TRY(ctx, cudaMalloc(&ctx->d_dust_scratch, threads * bytes_per));
		ctx->dust_per_thread = per;
		ctx->dust_threads2 = (uint32_t)threads;
	}
	if (!ctx->d_dust_cnt)
		CUDA_TRY(ctx, cudaMalloc(&ctx->d_dust_cnt, 2 * sizeof(unsigned long long)));
	ctx->dust = true;
	ctx->dust_T = (int)T;
	ctx->dust_W = (int)W;
	return BBT_OK;
}

extern "C" int bbt_set_dust(bbt_ctx *ctx, int on, unsigned T, unsigned W)
{
	int rc = set_dust_one(ctx, on, T, W);
	for (size_t i = 0; ctx && !rc && i < ctx->peers.size(); ++i)
		if ((rc = set_dust_one(ctx->peers[i], on, T, W)) != BBT_OK)
			fail(ctx, rc, ctx->peers[i]->err);
	return rc;
}

static int set_mode_one(bbt_ctx *ctx, int mode)
{
	if (!ctx)
		return BBT_ERR_ARG;
	if (mode < BBT_MODE_STD || mode > BBT_MODE_SCORES)
		return fail(ctx, BBT_ERR_ARG, "bbt_set_mode: unknown mode");
	ctx->mode = mode;
	return BBT_OK;
}

extern "C" int bbt_set_mode(bbt_ctx *ctx, int mode)
{
	int rc = set_mode_one(ctx, mode);
	for (size_t i = 0; ctx && !rc && i < ctx->peers.size(); ++i)
		if ((rc = set_mode_one(ctx->peers[i], mode)) != BBT_OK)
			fail(ctx, rc, ctx->peers[i]->err);
	return rc;
}

extern "C" int bbt_sync(bbt_ctx *ctx)
{
	if (!ctx)
		return BBT_ERR_ARG;
	for (bbt_ctx *peer : ctx->peers) {
		int rc = bbt_sync(peer);
		if (rc)
			return fail(ctx, rc, peer->err);
	}
	CUDA_TRY(ctx, cudaSetDevice(ctx->dev));
	CUDA_TRY(ctx, cudaDeviceSynchronize());
	return BBT_OK;
}

extern "C" int bbt_summary(bbt_ctx *ctx, uint64_t *counts, uint64_t *reads)
{
	if (!ctx)
		return BBT_ERR_ARG;
	CUDA_TRY(ctx, cudaSetDevice(ctx->dev));
	CUDA_TRY(ctx, cudaDeviceSynchronize());
	const size_t nc = 2 * (ctx->nf + 2) + 2;
	if (counts)
		CUDA_TRY(ctx, cudaMemcpy(counts, ctx->d_counts, sizeof(unsigned long long) * nc,
				cudaMemcpyDeviceToHost));
	if (reads)
		*reads = ctx->reads_seen;
	/* replicas on other devices: their counters add up (one host-side sum of
	 * the (F + 2)-entry summaries) */
	for (bbt_ctx *peer : ctx->peers) {
		std::vector<uint64_t> pc(nc);
		uint64_t pr = 0;
		int rc = bbt_summary(peer, pc.data(), &pr);
		if (rc)
			return fail(ctx, rc, peer->err);
		if (counts)
			for (size_t i = 0; i < nc; ++i)
				counts[i] += pc[i];
		if (reads)
			*reads += pr;
	}
	return BBT_OK;
}

extern "C" int bbt_reset_summary(bbt_ctx *ctx)
{
	if (!ctx)
		return BBT_ERR_ARG;
	CUDA_TRY(ctx, cudaSetDevice(ctx->dev));
	CUDA_TRY(ctx, cudaDeviceSynchronize());
	CUDA_TRY(ctx, cudaMemset(ctx->d_counts, 0,
			sizeof(unsigned long long) * (2 * (ctx->nf + 2) + 2)));
	ctx->reads_seen = 0;
	for (bbt_ctx *peer : ctx->peers) {
		int rc = bbt_reset_summary(peer);
		if (rc)
			return fail(ctx, rc, peer->err);
	}
	return BBT_OK;
}

extern "C" int bbt_summary_tsv(bbt_ctx *ctx, char *buf, size_t cap, size_t *len)
{
	if (!ctx)
		return BBT_ERR_ARG;
	std::vector<uint64_t> c(2 * (ctx->nf + 2) + 2);
	uint64_t reads = 0;
	int rc = bbt_summary(ctx, c.data(), &reads);
	if (rc)
		return rc;
	std::string t = summary_text(ctx, c, reads);
	if (len)
		*len = t.size();
	if (buf && cap) {
		size_t n = std::min(cap - 1, t.size());
		memcpy(buf, t.data(), n);
		buf[n] = 0;
	}
	return BBT_OK;
}

extern "C" int bbt_last_stats(bbt_ctx *ctx, bbt_stats *out)
{
	if (!ctx || !out)
		return BBT_ERR_ARG;
	CUDA_TRY(ctx, cudaSetDevice(ctx->dev));
	CUDA_TRY(ctx, cudaEventSynchronize(ctx->ev_stop));
	float ms = 0, kms = 0;
	CUDA_TRY(ctx, cudaEventElapsedTime(&ms, ctx->ev_start, ctx->ev_stop));
	CUDA_TRY(ctx, cudaEventElapsedTime(&kms, ctx->ev_k0, ctx->ev_k1));
	ctx->last.kernel_ms = ms;
	ctx->last.classify_ms = kms;
	if (ctx->lc.count) {
		unsigned long long st[3];
		CUDA_TRY(ctx, cudaMemcpy(st, ctx->d_stat, sizeof st, cudaMemcpyDeviceToHost));
		ctx->last.probes_issued = st[0];
		ctx->last.frames = st[1];
		ctx->last.probes_algorithmic = st[2];
	}
	*out = ctx->last;
	return BBT_OK;
}

static int set_inclusive_one(bbt_ctx *ctx, int inclusive)
{
	if (!ctx)
		return BBT_ERR_ARG;
	ctx->p.inclusive = inclusive ? 1 : 0;
	return BBT_OK;
}

extern "C" int bbt_set_inclusive(bbt_ctx *ctx, int inclusive)
{
	int rc = set_inclusive_one(ctx, inclusive);
	for (size_t i = 0; ctx && !rc && i < ctx->peers.size(); ++i)
		if ((rc = set_inclusive_one(ctx->peers[i], inclusive)) != BBT_OK)
			fail(ctx, rc, ctx->peers[i]->err);
	return rc;
}

/* Turn on probe/frame counting (diagnostics; adds atomics). */
static int set_counting_one(bbt_ctx *ctx, int on)
{
	if (!ctx)
		return BBT_ERR_ARG;
	ctx->lc.count = on ? 1 : 0;
	CUDA_TRY(ctx, cudaSetDevice(ctx->dev));
	CUDA_TRY(ctx, cudaMemset(ctx->d_stat, 0, 3 * sizeof(unsigned long long)));
	return BBT_OK;
}

extern "C" int bbt_set_counting(bbt_ctx *ctx, int on)
{
	int rc = set_counting_one(ctx, on);
	for (size_t i = 0; ctx && !rc && i < ctx->peers.size(); ++i)
		if ((rc = set_counting_one(ctx->peers[i], on)) != BBT_OK)
			fail(ctx, rc, ctx->peers[i]->err);
	return rc;
}

/* Change kernel path / launch shape after open (autotuner, bench). */
static int set_launch_one(bbt_ctx *ctx, int path, int warps_per_block, int seg)
{
	if (!ctx)
		return BBT_ERR_ARG;
	if (path != 0)
		ctx->p.path = path;
	if (warps_per_block)
		ctx->p.warps_per_block = (uint32_t)warps_per_block;
	if (seg)
		ctx->p.frames_per_lane = (uint32_t)seg;
	int cnt = ctx->lc.count;
	ctx->lc = pick_config(ctx);
	ctx->lc.count = cnt;
	return BBT_OK;
}

extern "C" int bbt_set_launch(bbt_ctx *ctx, int path, int warps_per_block, int seg)
{
	int rc = set_launch_one(ctx, path, warps_per_block, seg);
	for (size_t i = 0; ctx && !rc && i < ctx->peers.size(); ++i)
		if ((rc = set_launch_one(ctx->peers[i], path, warps_per_block, seg)) != BBT_OK)
			fail(ctx, rc, ctx->peers[i]->err);
	return rc;
}

static int set_steps_one(bbt_ctx *ctx, int steps)
{
	if (!ctx)
		return BBT_ERR_ARG;
	if (steps < BBT_STEPS_DECISION || steps > BBT_STEPS_WIDE_FULL)
		return fail(ctx, BBT_ERR_ARG, "bbt_set_steps: steps must be one of BBT_STEPS_*");
	ctx->steps = steps;
	int cnt = ctx->lc.count;
	ctx->lc = pick_config(ctx);
	ctx->lc.count = cnt;
	return BBT_OK;
}

extern "C" int bbt_set_steps(bbt_ctx *ctx, int steps)
{
	int rc = set_steps_one(ctx, steps);
	for (size_t i = 0; ctx && !rc && i < ctx->peers.size(); ++i)
		if ((rc = set_steps_one(ctx->peers[i], steps)) != BBT_OK)
			fail(ctx, rc, ctx->peers[i]->err);
	return rc;
}

static int set_bucketing_one(bbt_ctx *ctx, unsigned bucket_shift, unsigned phase_split,
		unsigned phase_min, uint64_t max_frames, unsigned levels_per_round)
{
	if (!ctx)
		return BBT_ERR_ARG;
	if (levels_per_round > 64)
		return fail(ctx, BBT_ERR_ARG, "bbt_set_bucketing: levels_per_round must be at most 64");
	if (bucket_shift && (bucket_shift < 12 || bucket_shift > 34))
		return fail(ctx, BBT_ERR_ARG, "bbt_set_bucketing: bucket_shift must be in [12, 34]");
	if (phase_split > kBkPhaseDen)
		return fail(ctx, BBT_ERR_ARG, "bbt_set_bucketing: phase_split must be at most 16");
	if (levels_per_round)
		ctx->bk_levels = levels_per_round;
	if (bucket_shift)
		ctx->bk_bshift = bucket_shift;
	if (phase_split)
		ctx->bk_phase_split = phase_split;
	if (phase_min)
		ctx->bk_phase_min = phase_min;
	if (max_frames)
		ctx->bk_max_frames = std::max<uint64_t>(max_frames, kBkWinFrames);
	return BBT_OK;
}

extern "C" int bbt_set_bucketing(bbt_ctx *ctx, unsigned bucket_shift, unsigned phase_split,
		unsigned phase_min, uint64_t max_frames, unsigned levels_per_round)
{
	int rc = set_bucketing_one(ctx, bucket_shift, phase_split, phase_min, max_frames,
			levels_per_round);
	for (size_t i = 0; ctx && !rc && i < ctx->peers.size(); ++i)
		if ((rc = set_bucketing_one(ctx->peers[i], bucket_shift, phase_split, phase_min,
				max_frames, levels_per_round)) != BBT_OK)
			fail(ctx, rc, ctx->peers[i]->err);
	return rc;
}

static int set_schedule_one(bbt_ctx *ctx, uint64_t long_bases)
{
	if (!ctx)
		return BBT_ERR_ARG;
	ctx->long_bases = long_bases;
	return BBT_OK;
}

extern "C" int bbt_set_schedule(bbt_ctx *ctx, uint64_t long_bases)
{
	int rc = set_schedule_one(ctx, long_bases);
	for (size_t i = 0; ctx && !rc && i < ctx->peers.size(); ++i)
		if ((rc = set_schedule_one(ctx->peers[i], long_bases)) != BBT_OK)
			fail(ctx, rc, ctx->peers[i]->err);
	return rc;
}

/* ---- autotuner ---- */

namespace {

/* One timed pass of the device batch b in launches of `chunk` reads. */
int time_pass(bbt_ctx *ctx, const bbt_batch *b, uint64_t chunk, uint64_t *h1, uint64_t *h2,
		cudaEvent_t e0, cudaEvent_t e1, float *ms)
{
	cudaStream_t s = ctx->stream;
	CUDA_TRY(ctx, cudaEventRecord(e0, s));
	for (uint64_t i = 0; i < b->n_reads; i += chunk) {
		bbt_batch sb = *b;
		sb.n_reads = std::min(chunk, b->n_reads - i);
		sb.offsets = b->offsets + i;
		if (b->seq2)
			sb.offsets2 = b->offsets2 + i;
		bbt_result r;
		r.hits = h1 + i * ctx->words;
		r.hits2 = b->seq2 ? h2 + i * ctx->words : nullptr;
		r.category = nullptr;
		r.location = BBT_DEVICE;
		int rc = classify_device(ctx, &sb, &r, s);
		if (rc)
			return rc;
	}
	CUDA_TRY(ctx, cudaEventRecord(e1, s));
	CUDA_TRY(ctx, cudaEventSynchronize(e1));
	CUDA_TRY(ctx, cudaEventElapsedTime(ms, e0, e1));
	return BBT_OK;
}

} // namespace

extern "C" int bbt_autotune(bbt_ctx *ctx, const bbt_batch *b, bbt_tune *out)
{
	if (!ctx || !b || b->location != BBT_DEVICE || b->n_reads == 0)
		return fail(ctx, BBT_ERR_ARG, "bbt_autotune: needs a non-empty device batch");
	CUDA_TRY(ctx, cudaSetDevice(ctx->dev));
	const uint64_t n = b->n_reads;
	const size_t nc = 2 * (ctx->nf + 2) + 2;
	std::vector<unsigned long long> saved(nc);
	CUDA_TRY(ctx, cudaDeviceSynchronize());
	CUDA_TRY(ctx, cudaMemcpy(saved.data(), ctx->d_counts, nc * 8, cudaMemcpyDeviceToHost));
	const uint64_t saved_reads = ctx->reads_seen;
	const bbt_params saved_p = ctx->p;
	const uint64_t saved_long = ctx->long_bases;
	uint64_t *h1 = nullptr, *h2 = nullptr;
	cudaEvent_t e0, e1;
	cudaEventCreate(&e0);
	cudaEventCreate(&e1);
	int rc = BBT_OK;
	if (cudaMalloc(&h1, n * ctx->words * 8) != cudaSuccess ||
			(b->seq2 && cudaMalloc(&h2, n * ctx->words * 8) != cudaSuccess))
		rc = fail(ctx, BBT_ERR_NOMEM, "bbt_autotune: cudaMalloc(results)");
	bbt_tune best;
	memset(&best, 0, sizeof best);
	float best_ms = 1e30f;
	const int saved_steps = ctx->steps;
	struct Cand {
		int path, warps, seg;
		uint64_t long_bases;
		int steps;
	};
	std::vector<Cand> cands;
	for (int w : {4, 8})
		for (int sg : {4, 8}) {
			cands.push_back({BBT_PATH_PLAIN, w, sg, 0, 0});
			/* the persistent kernel with steps sized to the read's decision
			 * (fewer probes: filters in HBM) and with full steps (fewer steps:
			 * filters held in L2), one or two frames per lane */
			for (int st : {BBT_STEPS_DECISION, BBT_STEPS_FULL, BBT_STEPS_WIDE,
					BBT_STEPS_WIDE_FULL}) {
				cands.push_back({BBT_PATH_PERSISTENT, w, sg, 0, st});
				cands.push_back({BBT_PATH_PERSISTENT, w, sg, 1024, st});
			}
			if (auto_path(ctx) == BBT_PATH_FILTER_MAJOR)
				cands.push_back({BBT_PATH_FILTER_MAJOR, w, sg, 0, 0});
		}
	if (bucketing_pays(ctx))
		cands.push_back({BBT_PATH_BUCKETED, 8, 4, 0, 0});
	const int cnt = ctx->lc.count;
	for (const Cand &c : cands) {
		if (rc)
			break;
		ctx->p.path = c.path;
		ctx->p.warps_per_block = c.warps;
		ctx->p.frames_per_lane = c.seg;
		ctx->steps = c.steps;
		ctx->lc = pick_config(ctx);
		ctx->lc.count = 0;
		ctx->long_bases = c.long_bases;
		float ms = 0;
		rc = time_pass(ctx, b, n, h1, h2, e0, e1, &ms); /* warm */
		if (!rc)
			rc = time_pass(ctx, b, n, h1, h2, e0, e1, &ms);
		if (!rc && ms < best_ms) {
			best_ms = ms;
			best.path = c.path;
			best.warps_per_block = c.warps;
			best.frames_per_lane = c.seg;
			best.long_bases = c.long_bases;
			best.steps = c.steps;
		}
	}
	/* reads per launch for the best kernel configuration */
	best.reads_per_launch = n;
	if (!rc) {
		ctx->p.path = best.path;
		ctx->p.warps_per_block = best.warps_per_block;
		ctx->p.frames_per_lane = best.frames_per_lane;
		ctx->steps = best.steps;
		ctx->lc = pick_config(ctx);
		ctx->lc.count = 0;
		ctx->long_bases = best.long_bases;
		float chunk_ms = best_ms;
		for (uint64_t ch : {1ull << 16, 1ull << 18, 1ull << 20}) {
			if (ch >= n || rc)
				break;
			float ms = 0;
			rc = time_pass(ctx, b, ch, h1, h2, e0, e1, &ms);
			if (!rc && ms < chunk_ms * 0.98f) {
				chunk_ms = ms;
				best.reads_per_launch = ch;
			}
		}
		best.reads_per_s = (double)n * (b->seq2 ? 2 : 1) / (std::min(best_ms, chunk_ms) * 1e-3);
		if (best.reads_per_launch == n)
			best.reads_per_launch = 0; /* no split beat one launch: launch whole batches */
	}
	cudaFree(h1);
	cudaFree(h2);
	cudaEventDestroy(e0);
	cudaEventDestroy(e1);
	/* the tuning passes leave the summary as it was */
	cudaMemcpy(ctx->d_counts, saved.data(), nc * 8, cudaMemcpyHostToDevice);
	ctx->reads_seen = saved_reads;
	if (rc) {
		ctx->p = saved_p;
		ctx->long_bases = saved_long;
		ctx->steps = saved_steps;
		ctx->lc = pick_config(ctx);
		ctx->lc.count = cnt;
		return rc;
	}
	ctx->lc.count = cnt;
	if (out)
		*out = best;
	return BBT_OK;
}

/* ---- CUDA graphs over device batches ---- */

struct bbt_graph {
	bbt_ctx *ctx = nullptr;
	cudaGraph_t graph = nullptr;
	cudaGraphExec_t exec = nullptr;
	cudaStream_t capture = nullptr;
	uint64_t reads = 0, launches = 0;
};

extern "C" int bbt_graph_create(bbt_ctx *ctx, const bbt_batch *b, const bbt_result *r,
		uint64_t reads_per_launch, bbt_graph **out)
{
	if (!ctx || !b || !r || !out || b->location != BBT_DEVICE || r->location != BBT_DEVICE)
		return fail(ctx, BBT_ERR_ARG, "bbt_graph_create: needs device batch and results");
	if (!r->hits || (b->seq2 && !r->hits2))
		return fail(ctx, BBT_ERR_ARG, "bbt_graph_create: result hit arrays are required");
	if (ctx->lc.path == BBT_PATH_FILTER_MAJOR || ctx->lc.path == BBT_PATH_BUCKETED)
		return fail(ctx, BBT_ERR_UNSUPPORTED, "bbt_graph_create: the filter-major and bucketed "
				"paths plan their sub-batches on the host; use the plain or persistent path "
				"in a graph");
	if (ctx->dust)
		return fail(ctx, BBT_ERR_UNSUPPORTED, "bbt_graph_create: DUST masking sizes its "
				"buffers on the host and cannot be captured");
	CUDA_TRY(ctx, cudaSetDevice(ctx->dev));
	const uint64_t n = b->n_reads;
	const uint64_t chunk = reads_per_launch ? std::min(reads_per_launch, std::max<uint64_t>(n, 1))
	                                        : std::max<uint64_t>(n, 1);
	/* buffers the launches grow must exist before capture */
	if (ctx->long_bases && ctx->lc.path != BBT_PATH_PLAIN) {
		int rc = grow(ctx, &ctx->d_order, ctx->order_cap, chunk * (b->seq2 ? 2 : 1));
		if (rc)
			return rc;
	}
	if (ctx->p.scoring == BBT_SCORE_BINOMIAL) { /* thresholds before capture */
		std::vector<uint64_t> lens;
		int rc = device_lengths(ctx, b, ctx->stream, lens);
		if (!rc)
			rc = ensure_bthres(ctx, lens);
		if (rc)
			return rc;
	}
	bbt_graph *g = new bbt_graph();
	g->ctx = ctx;
	g->reads = n;
	ctx->capturing = true;
	cudaError_t e = cudaStreamCreateWithFlags(&g->capture, cudaStreamNonBlocking);
	if (e == cudaSuccess)
		e = cudaStreamBeginCapture(g->capture, cudaStreamCaptureModeThreadLocal);
	int rc = e == cudaSuccess ? BBT_OK : cuda_fail(ctx, e, "cudaStreamBeginCapture");
	for (uint64_t i = 0; rc == BBT_OK && i < n; i += chunk) {
		bbt_batch sb = *b;
		sb.n_reads = std::min(chunk, n - i);
		sb.offsets = b->offsets + i;
		if (b->seq2)
			sb.offsets2 = b->offsets2 + i;
		bbt_result sr = *r;
		sr.hits = r->hits + i * ctx->words;
		sr.hits2 = b->seq2 ? r->hits2 + i * ctx->words : nullptr;
		sr.category = r->category ? r->category + i : nullptr;
		rc = classify_device(ctx, &sb, &sr, g->capture);
		++g->launches;
	}
	cudaGraph_t graph = nullptr;
	e = cudaStreamEndCapture(g->capture, &graph);
	ctx->capturing = false;
	if (rc == BBT_OK && e != cudaSuccess)
		rc = cuda_fail(ctx, e, "cudaStreamEndCapture");
	g->graph = graph;
	if (rc == BBT_OK) {
		e = cudaGraphInstantiate(&g->exec, graph, 0);
		if (e != cudaSuccess)
			rc = cuda_fail(ctx, e, "cudaGraphInstantiate");
	}
	ctx->reads_seen -= std::min(ctx->reads_seen, n); /* capture did not run anything */
	if (rc) {
		bbt_graph_destroy(g);
		return rc;
	}
	*out = g;
	return BBT_OK;
}

extern "C" int bbt_graph_launch(bbt_graph *g, void *stream)
{
	if (!g || !g->exec)
		return BBT_ERR_ARG;
	bbt_ctx *ctx = g->ctx;
	CUDA_TRY(ctx, cudaSetDevice(ctx->dev));
	CUDA_TRY(ctx, cudaGraphLaunch(g->exec, stream ? (cudaStream_t)stream : ctx->stream));
	ctx->reads_seen += g->reads;
	return BBT_OK;
}

extern "C" int bbt_graph_launches(const bbt_graph *g, uint64_t *launches)
{
	if (!g || !launches)
		return BBT_ERR_ARG;
	*launches = g->launches;
	return BBT_OK;
}

extern "C" int bbt_graph_destroy(bbt_graph *g)
{
	if (!g)
		return BBT_OK;
	if (g->exec)
		cudaGraphExecDestroy(g->exec);
	if (g->graph)
		cudaGraphDestroy(g->graph);
	if (g->capture)
		cudaStreamDestroy(g->capture);
	delete g;
	return BBT_OK;
}

/* ---- concurrent classification for the serving engine ---- */

int bbt::bf_scratch_init(bbt_ctx *ctx, BfScratch &sc, uint64_t max_reads)
{
	CUDA_TRY(ctx, cudaSetDevice(ctx->dev));
	CUDA_TRY(ctx, cudaMalloc(&sc.work, sizeof(unsigned long long)));
	CUDA_TRY(ctx, cudaMalloc(&sc.order_cnt, 2 * sizeof(unsigned long long)));
	CUDA_TRY(ctx, cudaMalloc(&sc.order, std::max<uint64_t>(max_reads, 1) * 2 * sizeof(uint64_t)));
	sc.order_cap = std::max<uint64_t>(max_reads, 1) * 2;
	return BBT_OK;
}

void bbt::bf_scratch_free(BfScratch &sc)
{
	cudaFree(sc.work);
	cudaFree(sc.order_cnt);
	cudaFree(sc.order);
	sc = BfScratch();
}

int bbt::bf_classify_slot(bbt_ctx *ctx, const uint8_t *seq, const uint64_t *off,
		const uint8_t *seq2, const uint64_t *off2, uint64_t n, uint64_t *hits, uint64_t *hits2,
		uint32_t *category, cudaStream_t s, BfScratch &sc)
{
	if (n == 0)
		return BBT_OK;
	const bool paired = seq2 != nullptr;
	ClassifyArgs a = base_args(ctx);
	a.probes = a.frames = a.alg_probes = nullptr;
	a.seq[0] = seq;
	a.off[0] = off;
	a.seq[1] = paired ? seq2 : seq;
	a.off[1] = paired ? off2 : off;
	a.n = n;
	a.mates = paired ? 2 : 1;
	a.hits[0] = hits;
	a.hits[1] = paired ? hits2 : nullptr;
	a.work = sc.work;
	if (ctx->dust)
		return fail(ctx, BBT_ERR_UNSUPPORTED, "the serving engine does not run DUST masking");
	LaunchConfig lc = ctx->lc;
	lc.count = 0;
	if (lc.path == BBT_PATH_FILTER_MAJOR)
		lc.path = BBT_PATH_PERSISTENT;
	if (ctx->mode == BBT_MODE_BESTHIT) {
		ScoreArgs sa;
		sa.scores[0] = sa.scores[1] = nullptr;
		sa.fpr = ctx->d_fpr;
		sa.besthit = 1;
		CUDA_TRY(ctx, launch_scores(a, sa, lc, s));
	} else if (lc.path != BBT_PATH_PLAIN) {
		CUDA_TRY(ctx, cudaMemsetAsync(sc.work, 0, sizeof(unsigned long long), s));
		if (ctx->long_bases && n * a.mates <= sc.order_cap) {
			CUDA_TRY(ctx, cudaMemsetAsync(sc.order_cnt, 0, 2 * sizeof(unsigned long long), s));
			CUDA_TRY(ctx, launch_long_first(a, ctx->long_bases, sc.order, sc.order_cnt,
					ctx->num_sms, s));
			a.order = sc.order;
		}
	}
	if (ctx->mode != BBT_MODE_BESTHIT)
		CUDA_TRY(ctx, launch_classify(a, lc, s));
	CUDA_TRY(ctx, launch_summarize(a.hits[0], paired ? a.hits[1] : nullptr, n, ctx->nf,
			ctx->words, ctx->p.inclusive, ctx->mode == BBT_MODE_ORDERED, category,
			ctx->d_counts, ctx->num_sms, s));
	return BBT_OK;
}

extern "C" int bbt_set_stdout(bbt_ctx *ctx, int on, int inverse)
{
	if (!ctx)
		return BBT_ERR_ARG;
	ctx->to_stdout = on != 0;
	ctx->inverse = inverse != 0;
	return BBT_OK;
}
