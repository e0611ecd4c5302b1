/*
 * server.cpp -- the serving engine behind bbt_server.h.
 *
 * Threads: one scheduler (admission) and one worker per slot.  The scheduler
 * takes queued requests in arrival order; a request is admitted when a slot is
 * idle and its device buffers fit in the free part of the budget, managed by a
 * first-fit allocator over one device allocation made at creation (so serving
 * never calls cudaMalloc).  The worker copies the request in on its own stream,
 * runs the Bloom or miBF kernels with its own per-stream scratch (work
 * counters, read order, per-batch summary), copies the results out, waits for
 * its stream, releases the memory and wakes whoever waits for the request.
 * Workers on different slots overlap on the device.
 */
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "bbt_server.h"
#include "ctx.hpp"
#include "mibf_ctx.hpp"

namespace bbt {
namespace {

constexpr size_t kAlign = 256;

size_t align_up(size_t n)
{
	return (n + kAlign - 1) & ~(kAlign - 1);
}

/* First-fit allocator of offsets in [0, cap). */
class Arena {
public:
	void init(size_t cap)
	{
		cap_ = cap;
		free_.clear();
		free_[0] = cap;
		used_ = 0;
	}
	bool alloc(size_t n, size_t &off)
	{
		n = align_up(n);
		for (auto it = free_.begin(); it != free_.end(); ++it) {
			if (it->second < n)
				continue;
			off = it->first;
			const size_t rest = it->second - n;
			free_.erase(it);
			if (rest)
				free_[off + n] = rest;
			used_ += n;
			return true;
		}
		return false;
	}
	void release(size_t off, size_t n)
	{
		n = align_up(n);
		used_ -= n;
		auto it = free_.emplace(off, n).first;
		auto next = std::next(it);
		if (next != free_.end() && it->first + it->second == next->first) {
			it->second += next->second;
			free_.erase(next);
		}
		if (it != free_.begin()) {
			auto prev = std::prev(it);
			if (prev->first + prev->second == it->first) {
				prev->second += it->second;
				free_.erase(it);
			}
		}
	}
	size_t cap() const { return cap_; }
	size_t used() const { return used_; }

private:
	size_t cap_ = 0, used_ = 0;
	std::map<size_t, size_t> free_;
};

/* Device layout of one chunk of a request inside its reservation. */
struct Layout {
	uint64_t chunk = 0;                  /* reads per chunk */
	size_t seq[2] = {0, 0}, off[2] = {0, 0};
	size_t out[3] = {0, 0, 0};           /* bloom: hits, hits2, category; miBF: hits, n, sat */
	size_t bytes = 0;
};

struct Req {
	uint64_t ticket = 0;
	bbt_request r;
	bbt_request_stats st;
	Layout lay;
	size_t off = 0;
	bool done = false;
	std::string err;
};

struct ServeSlot {
	std::thread th;
	cudaStream_t s = nullptr;
	BfScratch bf;
	MibfScratch mi;
	uint64_t *h_off = nullptr;           /* pinned: rebased offsets of a chunk (two mates) */
	Req *job = nullptr;
};

uint64_t max_chunk_bases(const uint64_t *off, uint64_t n, uint64_t chunk)
{
	uint64_t most = 0;
	for (uint64_t i = 0; i < n; i += chunk)
		most = std::max(most, off[std::min(n, i + chunk)] - off[i]);
	return most;
}

} // namespace
} // namespace bbt

using namespace bbt;

struct bbt_server {
	bbt_ctx *bf = nullptr;
	bbt_mibf *mi = nullptr;
	bbt_server_params p;
	int dev = 0;
	std::mutex mu;
	std::condition_variable cv;
	std::deque<Req *> queue;
	std::map<uint64_t, Req *> reqs;
	std::vector<ServeSlot> slots;
	Arena arena;
	char *d_arena = nullptr;
	std::thread sched;
	bool stop = false;
	uint64_t next_ticket = 1;
	uint64_t in_flight = 0;
	uint64_t releases = 0;   /* memory releases so far (admission waits on it) */
	std::chrono::steady_clock::time_point t0;
	std::string err;
	std::mutex bf_mu;
	double now() const
	{
		return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
	}
};

namespace {

/* Buffer layout of a request for chunks of c reads. */
Layout layout_for(const bbt_server *srv, const bbt_request &r, uint64_t c)
{
	Layout L;
	L.chunk = c;
	const bool paired = r.seq2 != nullptr;
	size_t at = 0;
	auto take = [&](size_t n) {
		size_t o = at;
		at += align_up(std::max<size_t>(n, 1));
		return o;
	};
	for (int m = 0; m < (paired ? 2 : 1); ++m) {
		const uint64_t *off = m ? r.offsets2 : r.offsets;
		L.seq[m] = take(r.n_reads ? max_chunk_bases(off, r.n_reads, c) : 0);
		L.off[m] = take((c + 1) * 8);
	}
	if (r.kind == BBT_REQ_BLOOM) {
		const uint64_t words = srv->bf ? srv->bf->words : 1;
		L.out[0] = take(c * words * 8);
		if (paired)
			L.out[1] = take(c * words * 8);
		L.out[2] = take(c * 4);
	} else {
		L.out[0] = take(c * (uint64_t)std::max<uint32_t>(r.mi_max_hits, 1) * sizeof(bbt_mibf_hit));
		L.out[1] = take(c * 4);
		L.out[2] = take(c * 4);
	}
	L.bytes = at;
	return L;
}

int run_chunk(bbt_server *srv, ServeSlot &sl, Req &q, char *base, uint64_t i0, uint64_t i1)
{
	const bbt_request &r = q.r;
	const uint64_t c = i1 - i0;
	const bool paired = r.seq2 != nullptr;
	cudaStream_t s = sl.s;
	const Layout &L = q.lay;
	const uint8_t *dseq[2] = {nullptr, nullptr};
	const uint64_t *doff[2] = {nullptr, nullptr};
	for (int m = 0; m < (paired ? 2 : 1); ++m) {
		const uint64_t *off = m ? r.offsets2 : r.offsets;
		const char *seq = m ? r.seq2 : r.seq;
		uint64_t *h = sl.h_off + m * (srv->p.chunk_reads + 1);
		for (uint64_t i = 0; i <= c; ++i)
			h[i] = off[i0 + i] - off[i0];
		const uint64_t nb = off[i1] - off[i0];
		if (nb && cudaMemcpyAsync(base + L.seq[m], seq + off[i0], nb, cudaMemcpyHostToDevice, s) !=
				cudaSuccess)
			return BBT_ERR_CUDA;
		if (cudaMemcpyAsync(base + L.off[m], h, (c + 1) * 8, cudaMemcpyHostToDevice, s) !=
				cudaSuccess)
			return BBT_ERR_CUDA;
		dseq[m] = (const uint8_t *)(base + L.seq[m]);
		doff[m] = (const uint64_t *)(base + L.off[m]);
	}
	int rc = BBT_OK;
	if (r.kind == BBT_REQ_BLOOM) {
		const uint64_t words = srv->bf->words;
		uint64_t *dh = (uint64_t *)(base + L.out[0]);
		uint64_t *dh2 = paired ? (uint64_t *)(base + L.out[1]) : nullptr;
		uint32_t *dc = (uint32_t *)(base + L.out[2]);
		rc = bf_rows_for(srv->bf, sl.h_off, paired ? sl.h_off + srv->p.chunk_reads + 1 : nullptr, c);
		if (rc)
			return rc;
		rc = bf_classify_slot(srv->bf, dseq[0], doff[0], dseq[1], doff[1], c, dh, dh2, dc, s,
				sl.bf);
		if (rc)
			return rc;
		if (r.hits && cudaMemcpyAsync(r.hits + i0 * words, dh, c * words * 8,
				cudaMemcpyDeviceToHost, s) != cudaSuccess)
			return BBT_ERR_CUDA;
		if (paired && r.hits2 && cudaMemcpyAsync(r.hits2 + i0 * words, dh2, c * words * 8,
				cudaMemcpyDeviceToHost, s) != cudaSuccess)
			return BBT_ERR_CUDA;
		if (r.category && cudaMemcpyAsync(r.category + i0, dc, c * 4, cudaMemcpyDeviceToHost, s) !=
				cudaSuccess)
			return BBT_ERR_CUDA;
		std::lock_guard<std::mutex> lk(srv->bf_mu);
		srv->bf->reads_seen += c;
	} else {
		rc = mibf_rows_for(srv->mi, sl.h_off, paired ? sl.h_off + srv->p.chunk_reads + 1 : nullptr,
				c);
		if (rc)
			return rc;
		const uint32_t mh = std::max<uint32_t>(r.mi_max_hits, 1);
		bbt_mibf_hit *dh = (bbt_mibf_hit *)(base + L.out[0]);
		uint32_t *dn = (uint32_t *)(base + L.out[1]);
		uint32_t *ds = (uint32_t *)(base + L.out[2]);
		rc = mibf_classify_slot(srv->mi, c, dseq[0], doff[0], dseq[1], doff[1], dh,
				r.mi_max_hits, dn, ds, s, sl.mi);
		if (rc)
			return rc;
		if (r.mi_hits && r.mi_max_hits && cudaMemcpyAsync(r.mi_hits + i0 * mh, dh,
				c * mh * sizeof(bbt_mibf_hit), cudaMemcpyDeviceToHost, s) != cudaSuccess)
			return BBT_ERR_CUDA;
		if (cudaMemcpyAsync(r.mi_n_hits + i0, dn, c * 4, cudaMemcpyDeviceToHost, s) !=
				cudaSuccess)
			return BBT_ERR_CUDA;
		if (cudaMemcpyAsync(r.mi_sat + i0, ds, c * 4, cudaMemcpyDeviceToHost, s) != cudaSuccess)
			return BBT_ERR_CUDA;
	}
	/* the pinned offsets are rewritten by the next chunk */
	if (cudaStreamSynchronize(s) != cudaSuccess)
		return BBT_ERR_CUDA;
	if (r.kind == BBT_REQ_MIBF) {
		unsigned int flag = 0;
		if (cudaMemcpyAsync(&flag, sl.mi.flags, 4, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
				cudaStreamSynchronize(s) != cudaSuccess)
			return BBT_ERR_CUDA;
		if (flag)
			return BBT_ERR_OVERFLOW;
	}
	return BBT_OK;
}

void worker(bbt_server *srv, size_t idx)
{
	cudaSetDevice(srv->dev);
	ServeSlot &sl = srv->slots[idx];
	for (;;) {
		Req *q = nullptr;
		{
			std::unique_lock<std::mutex> lk(srv->mu);
			srv->cv.wait(lk, [&] { return sl.job != nullptr || srv->stop; });
			if (!sl.job)
				return;
			q = sl.job;
		}
		char *base = srv->d_arena + q->off;
		int rc = BBT_OK;
		for (uint64_t i = 0; i < q->r.n_reads && rc == BBT_OK; i += q->lay.chunk)
			rc = run_chunk(srv, sl, *q, base, i, std::min(q->r.n_reads, i + q->lay.chunk));
		if (rc == BBT_ERR_CUDA)
			q->err = std::string("CUDA error: ") + cudaGetErrorString(cudaGetLastError());
		else if (rc == BBT_ERR_OVERFLOW)
			q->err = "a read has more significant IDs than mi_max_hits";
		else if (rc && q->r.kind == BBT_REQ_MIBF)
			q->err = srv->mi->err;
		else if (rc)
			q->err = srv->bf->err;
		cudaStreamSynchronize(sl.s);
		{
			std::lock_guard<std::mutex> lk(srv->mu);
			srv->arena.release(q->off, q->lay.bytes);
			++srv->releases;
			q->st.status = rc;
			q->st.t_done = srv->now();
			q->done = true;
			sl.job = nullptr;
			--srv->in_flight;
		}
		srv->cv.notify_all();
	}
}

void scheduler(bbt_server *srv)
{
	std::unique_lock<std::mutex> lk(srv->mu);
	for (;;) {
		srv->cv.wait(lk, [&] {
			if (srv->stop && srv->queue.empty())
				return true;
			if (srv->queue.empty())
				return false;
			for (ServeSlot &sl : srv->slots)
				if (!sl.job)
					return srv->arena.cap() - srv->arena.used() >= srv->queue.front()->lay.bytes;
			return false;
		});
		if (srv->queue.empty())
			return;
		Req *q = srv->queue.front();
		size_t off = 0;
		if (!srv->arena.alloc(q->lay.bytes, off)) {
			/* enough bytes free but not in one piece: wait for a release */
			const uint64_t v = srv->releases;
			srv->cv.wait(lk, [&] { return srv->releases != v; });
			continue;
		}
		size_t idx = 0;
		while (srv->slots[idx].job)
			++idx;
		srv->queue.pop_front();
		q->off = off;
		q->st.t_admit = srv->now();
		q->st.device_bytes = q->lay.bytes;
		q->st.slot = (uint32_t)idx;
		srv->slots[idx].job = q;
		++srv->in_flight;
		srv->cv.notify_all();
	}
}

int srv_fail(bbt_server *srv, int code, const std::string &msg)
{
	if (srv)
		srv->err = msg;
	else
		set_global_error(msg);
	return code;
}

} // namespace

extern "C" int bbt_server_create(bbt_ctx *bloom, bbt_mibf *mibf, const bbt_server_params *params,
		bbt_server **out)
{
	if (!out || (!bloom && !mibf))
		return srv_fail(nullptr, BBT_ERR_ARG, "bbt_server_create: need a context");
	*out = nullptr;
	bbt_server *srv = new bbt_server();
	srv->bf = bloom;
	srv->mi = mibf;
	if (params)
		srv->p = *params;
	else
		memset(&srv->p, 0, sizeof srv->p);
	if (!srv->p.slots)
		srv->p.slots = 4;
	if (!srv->p.chunk_reads)
		srv->p.chunk_reads = 1ull << 20;
	if (!srv->p.max_frames)
		srv->p.max_frames = 16384;
	srv->dev = bloom ? bloom->dev : mibf->dev;
	srv->t0 = std::chrono::steady_clock::now();
	auto bail = [&](int rc, const std::string &m) {
		set_global_error(m);
		bbt_server_destroy(srv);
		return rc;
	};
	if (cudaSetDevice(srv->dev) != cudaSuccess)
		return bail(BBT_ERR_CUDA, "cudaSetDevice failed");
	if (bloom && bloom->dust)
		return bail(BBT_ERR_UNSUPPORTED, "bbt_server_create: the serving engine does not run "
				"DUST masking (switch it off with bbt_set_dust)");
	if (bloom && bf_reserve_rows(bloom, (uint64_t)srv->p.max_frames + bloom->kmax))
		return bail(BBT_ERR_NOMEM, "cannot reserve the binomial threshold rows: " + bloom->err);
	if (mibf && mibf_reserve_rows(mibf, srv->p.max_frames + 1))
		return bail(BBT_ERR_NOMEM, "cannot reserve the miBF minCount rows: " + mibf->err);
	size_t free_b = 0, total_b = 0;
	cudaMemGetInfo(&free_b, &total_b);
	const uint64_t budget = srv->p.mem_budget ? srv->p.mem_budget
	                                          : (uint64_t)(0.4 * (double)free_b);
	if (cudaMalloc(&srv->d_arena, budget) != cudaSuccess)
		return bail(BBT_ERR_NOMEM, "cannot allocate the serving memory budget");
	srv->arena.init(budget);
	srv->p.mem_budget = budget;
	srv->slots.resize(srv->p.slots);
	for (ServeSlot &sl : srv->slots) {
		if (cudaStreamCreateWithFlags(&sl.s, cudaStreamNonBlocking) != cudaSuccess ||
				cudaMallocHost(&sl.h_off, 2 * (srv->p.chunk_reads + 1) * 8) != cudaSuccess)
			return bail(BBT_ERR_NOMEM, "cannot create a serving slot");
		if (bloom && bf_scratch_init(bloom, sl.bf, srv->p.chunk_reads))
			return bail(BBT_ERR_NOMEM, "cannot allocate Bloom scratch: " + bloom->err);
		if (mibf && mibf_scratch_init(mibf, sl.mi))
			return bail(BBT_ERR_NOMEM, "cannot allocate miBF scratch: " + mibf->err);
	}
	for (size_t i = 0; i < srv->slots.size(); ++i)
		srv->slots[i].th = std::thread(worker, srv, i);
	srv->sched = std::thread(scheduler, srv);
	*out = srv;
	return BBT_OK;
}

extern "C" int bbt_server_submit(bbt_server *srv, const bbt_request *req, uint64_t *ticket)
{
	if (!srv || !req || !ticket)
		return srv_fail(srv, BBT_ERR_ARG, "bbt_server_submit: NULL argument");
	if (req->kind == BBT_REQ_BLOOM ? !srv->bf : (req->kind == BBT_REQ_MIBF ? !srv->mi : true))
		return srv_fail(srv, BBT_ERR_ARG, "bbt_server_submit: no context for this request kind");
	if (req->n_reads && (!req->seq || !req->offsets || (req->seq2 && !req->offsets2)))
		return srv_fail(srv, BBT_ERR_ARG, "bbt_server_submit: reads missing");
	if (req->kind == BBT_REQ_MIBF && (!req->mi_n_hits || !req->mi_sat ||
			(req->mi_max_hits && !req->mi_hits)))
		return srv_fail(srv, BBT_ERR_ARG, "bbt_server_submit: miBF result arrays missing");
	Req *q = new Req();
	q->r = *req;
	memset(&q->st, 0, sizeof q->st);
	/* chunk size: the largest that fits the budget (halving from chunk_reads) */
	uint64_t c = std::max<uint64_t>(1, std::min<uint64_t>(req->n_reads, srv->p.chunk_reads));
	q->lay = layout_for(srv, q->r, c);
	while (q->lay.bytes > srv->arena.cap() && c > 1) {
		c = (c + 1) / 2;
		q->lay = layout_for(srv, q->r, c);
	}
	if (q->lay.bytes > srv->arena.cap()) {
		delete q;
		return srv_fail(srv, BBT_ERR_NOMEM, "a read does not fit the serving memory budget");
	}
	{
		std::lock_guard<std::mutex> lk(srv->mu);
		q->ticket = srv->next_ticket++;
		q->st.t_submit = srv->now();
		srv->reqs[q->ticket] = q;
		srv->queue.push_back(q);
		*ticket = q->ticket;
	}
	srv->cv.notify_all();
	return BBT_OK;
}

extern "C" int bbt_server_wait(bbt_server *srv, uint64_t ticket, double timeout_s,
		bbt_request_stats *stats)
{
	if (!srv)
		return BBT_ERR_ARG;
	std::unique_lock<std::mutex> lk(srv->mu);
	auto it = srv->reqs.find(ticket);
	if (it == srv->reqs.end())
		return srv_fail(srv, BBT_ERR_ARG, "unknown ticket");
	Req *q = it->second;
	auto ready = [&] { return q->done; };
	if (timeout_s < 0)
		srv->cv.wait(lk, ready);
	else if (!srv->cv.wait_for(lk, std::chrono::duration<double>(timeout_s), ready))
		return BBT_ERR_TIMEOUT;
	if (stats)
		*stats = q->st;
	if (q->st.status)
		srv->err = q->err;
	srv->reqs.erase(it);
	delete q;
	return BBT_OK;
}

extern "C" int bbt_server_load(bbt_server *srv, uint64_t *queued, uint64_t *in_flight,
		uint64_t *reserved)
{
	if (!srv)
		return BBT_ERR_ARG;
	std::lock_guard<std::mutex> lk(srv->mu);
	if (queued)
		*queued = srv->queue.size();
	if (in_flight)
		*in_flight = srv->in_flight;
	if (reserved)
		*reserved = srv->arena.used();
	return BBT_OK;
}

extern "C" int bbt_server_destroy(bbt_server *srv)
{
	if (!srv)
		return BBT_OK;
	{
		std::unique_lock<std::mutex> lk(srv->mu);
		srv->cv.wait(lk, [&] { return srv->queue.empty() && srv->in_flight == 0; });
		srv->stop = true;
	}
	srv->cv.notify_all();
	if (srv->sched.joinable())
		srv->sched.join();
	for (ServeSlot &sl : srv->slots)
		if (sl.th.joinable())
			sl.th.join();
	cudaSetDevice(srv->dev);
	for (ServeSlot &sl : srv->slots) {
		if (sl.s)
			cudaStreamDestroy(sl.s);
		cudaFreeHost(sl.h_off);
		bf_scratch_free(sl.bf);
		mibf_scratch_free(sl.mi);
	}
	cudaFree(srv->d_arena);
	for (auto &kv : srv->reqs)
		delete kv.second;
	delete srv;
	return BBT_OK;
}

extern "C" const char *bbt_server_last_error(const bbt_server *srv)
{
	return srv ? srv->err.c_str() : bbt_last_error(nullptr);
}
