/*
 * bbt_server.h -- serving engine of libbbt.so: a request loop that keeps a
 * Bloom-filter context and a miBF context resident on one GPU and classifies
 * requests of any size as they arrive (continuous batching).
 *
 * No reference counterpart: the reference classifies one file set per process
 * (BioBloomClassifier::filter, MIBFClassifier::filter).  Results are those of
 * bbt_classify_batch / bbt_mibf_classify_batch on the same reads, bit for bit,
 * whatever else is in flight.
 *
 * Model.  bbt_server_submit queues a request and returns at once.  A scheduler
 * admits queued requests in arrival order as soon as a slot (a CUDA stream and
 * its worker thread) is idle and the request's device buffers fit in the free
 * part of the server's device-memory budget (admission by free HBM).  An
 * admitted request is copied in from its host buffers on its slot's stream,
 * classified with the context's tuned kernels in launches of at most
 * chunk_reads reads, and copied out; requests on different slots overlap on
 * the device.  A request larger than the budget is processed in smaller chunks
 * inside its slot.  Serving allocates no device memory after creation.
 */
#ifndef BBT_SERVER_H
#define BBT_SERVER_H

#include <stddef.h>
#include <stdint.h>

#include "bbt.h"
#include "bbt_mibf.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct bbt_server bbt_server;

#define BBT_REQ_BLOOM 0
#define BBT_REQ_MIBF 1

typedef struct {
	uint64_t mem_budget;     /* device bytes for requests in flight; 0 = 40% of free HBM */
	uint32_t slots;          /* requests in flight at once; 0 = 4 */
	uint64_t chunk_reads;    /* reads per launch inside a request; 0 = 1M */
	uint32_t max_frames;     /* longest read (frames) a request may hold; 0 = 16384 */
} bbt_server_params;

/* One request: host reads (pairs when seq2 != NULL) and host result arrays,
 * which must stay valid until the request is done.  Bloom requests fill
 * hits (n x words uint64, words = (filters + 63) / 64), hits2 for pairs, and
 * category (n uint32), as bbt_classify_batch does.  miBF requests fill
 * mi_hits (n x mi_max_hits), mi_n_hits and mi_sat as bbt_mibf_classify_batch
 * does; a read with more than mi_max_hits results ends the request with
 * BBT_ERR_OVERFLOW (n_hits stays exact; that chunk's summary is not counted). */
typedef struct {
	int kind;                /* BBT_REQ_BLOOM or BBT_REQ_MIBF */
	const char *seq;
	const uint64_t *offsets; /* n_reads + 1 entries */
	const char *seq2;
	const uint64_t *offsets2;
	uint64_t n_reads;
	uint64_t *hits;
	uint64_t *hits2;
	uint32_t *category;
	bbt_mibf_hit *mi_hits;
	uint32_t mi_max_hits;
	uint32_t *mi_n_hits;
	uint32_t *mi_sat;
} bbt_request;

/* Timings of a finished request, in seconds since the server was created. */
typedef struct {
	int status;              /* BBT_OK or the request's error */
	double t_submit, t_admit, t_done;
	uint64_t device_bytes;   /* what admission reserved */
	uint32_t slot;
} bbt_request_stats;

/* Either context may be NULL (requests of that kind are then refused).  The
 * caller must not use the contexts while the server runs.  Bloom requests
 * follow the context's filtering mode (bbt_set_mode): ORDERED and BESTHIT
 * give their hit words and summary; SCORES gives the STD hits (requests carry
 * no scores).  A context with DUST masking on is refused. */
int bbt_server_create(bbt_ctx *bloom, bbt_mibf *mibf, const bbt_server_params *params,
		bbt_server **out);
/* Queue a request; *ticket identifies it. */
int bbt_server_submit(bbt_server *srv, const bbt_request *req, uint64_t *ticket);
/* Wait up to timeout_s seconds (< 0: forever) for a request; returns
 * BBT_ERR_TIMEOUT if it is not done by then.  The request's own status is in
 * stats->status (its message in bbt_server_last_error).  A ticket can be
 * waited for once. */
int bbt_server_wait(bbt_server *srv, uint64_t ticket, double timeout_s, bbt_request_stats *stats);
/* Requests queued, in flight, and the device bytes reserved right now. */
int bbt_server_load(bbt_server *srv, uint64_t *queued, uint64_t *in_flight, uint64_t *reserved);
/* Finish everything queued, then stop the workers and free the server. */
int bbt_server_destroy(bbt_server *srv);
const char *bbt_server_last_error(const bbt_server *srv);

#ifdef __cplusplus
}
#endif
#endif
