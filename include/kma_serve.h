/*
 * kma_serve.h -- the served form of the KMA heap (libkma_b200.so): a
 * request loop that keeps one heap resident on the device, admits
 * requests as slots and heap room free up (continuous batching: work of
 * requests admitted at different times overlaps on the device), and
 * reports per-request latency.
 *
 * No counterpart in the reference; every allocation goes through the
 * device heap (clArrayList growth over kma_malloc_warp, kma_structs.cuh).
 *
 * Request (seed, N): a random graph on N vertices whose degrees follow a
 * power law P(d) ~ d^-gamma on 1..deg_max (gamma = 2.1) with uint32
 * neighbour ids drawn uniformly from [0, N).  Its three kernels, on the
 * request's slot stream:
 *   build   every vertex grows its own clArrayList of neighbour ids in
 *           pages of 8, 16, 32, ... objects (one heap block per page);
 *   verify  every vertex walks its pages, checks each id against the
 *           seed's draw, and folds its list into the request checksum;
 *   free    every vertex clears its list (all blocks back to the heap).
 * The checksum depends only on (seed, N), never on where the blocks
 * landed, so a request gives the same result alone and in any mix.
 */
#ifndef KMA_SERVE_H
#define KMA_SERVE_H

#include <stdint.h>
#include "kma.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct kma_serve_s *kma_serve_t;

typedef struct kma_serve_cfg {
	uint32_t slots;          /* requests on the device at once (1..64) */
	uint32_t max_vertices;   /* largest N accepted */
	uint32_t deg_max;        /* degree cap (1..65535) */
	uint32_t block_dim;      /* threads per block of the request kernels (0 = 256) */
	float gamma;             /* degree exponent (> 1) */
	float occupancy_limit;   /* admit while reserved bytes <= limit * heap bytes (e.g. 0.85) */
} kma_serve_cfg;

typedef struct kma_serve_req {
	uint32_t n_vertices;
	uint32_t pad;
	uint64_t seed;
	double arrival_s;        /* release time, seconds after the run starts */
} kma_serve_req;

#define KMA_SERVE_OK 0
#define KMA_SERVE_NOMEM 1    /* a page malloc returned NULL (heap exhausted) */
#define KMA_SERVE_MISMATCH 2 /* verify found a neighbour id that differs */
#define KMA_SERVE_TOO_BIG 3  /* N above max_vertices, or larger than the heap */

typedef struct kma_serve_result {
	uint64_t checksum;       /* sum over vertices of the hash of the vertex's list */
	uint64_t edges;          /* neighbour ids written */
	uint64_t mallocs, frees, nulls;
	double admit_s;          /* when the request was admitted */
	double done_s;           /* when its last kernel finished (device events) */
	uint64_t reserved_bytes; /* the admission estimate */
	uint32_t slot, status;   /* KMA_SERVE_* */
} kma_serve_result;

typedef struct kma_serve_summary {
	double wall_s;           /* first release to last completion */
	uint64_t ops;            /* mallocs + frees over all requests */
	uint32_t max_running;    /* most requests on the device at once */
	uint32_t max_sb_in_use;  /* most superblocks in use seen after a build */
	double max_occupancy;    /* max_sb_in_use / superblocks on the free list at reset */
	double max_reserved;     /* most admission estimates held at once / heap bytes
				  * (the admission rule keeps it <= occupancy_limit) */
	uint32_t admit_waits;    /* admissions deferred because the heap room, not a
				  * slot, was missing */
	uint32_t pad;
} kma_serve_summary;

int kma_serve_create(kma_heap_t h, const kma_serve_cfg *cfg, kma_serve_t *out);
int kma_serve_destroy(kma_serve_t s);
/* Call style of later runs: KMA_MODE_WARP (the default: each warp's page
 * mallocs and frees go to the heap as one warp-collaborative call) or
 * KMA_MODE_PLAIN (every vertex's thread calls kma_malloc / kma_free
 * itself, the reference's per-work-item calls, kma.cl:279-373).  There is
 * no PMA form: a heap that frees nothing cannot stay resident under a
 * stream of requests. */
int kma_serve_set_mode(kma_serve_t s, int mode);
/* Expected heap bytes of a request of n vertices (the admission estimate). */
uint64_t kma_serve_estimate(kma_serve_t s, uint32_t n_vertices);
/* Serve `n` requests (sorted by arrival_s).  realtime != 0 releases each
 * at its arrival time on the host clock; 0 releases all at the start.
 * Blocks until every request finished; res[i] is request i's result. */
int kma_serve_run(kma_serve_t s, const kma_serve_req *reqs, uint32_t n, int realtime, kma_serve_result *res,
		  kma_serve_summary *sum);

#ifdef __cplusplus
}
#endif

#endif /* KMA_SERVE_H */
