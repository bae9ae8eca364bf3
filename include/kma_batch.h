/*
 * kma_batch.h -- the batched form of the KMA heap (libkma_b200.so): many
 * uneven allocation-heavy jobs run in one persistent, CUDA-graph-captured
 * launch on one heap, and a native autotuner picks the superblock size,
 * block shape and per-warp cache depth.
 *
 * No counterpart in the reference, whose jobs are one OpenCL kernel each
 * (test/tb_kma.c); every allocation still goes through kma_malloc_warp /
 * kma_free_warp of kma_device.cuh.
 *
 * Job program (per thread of a job, R rounds): free the blocks whose
 * lifetime ended this round (verifying their tags), then malloc one block
 * of a Zipf(1.2) size over 8..4096 bytes in steps of 8, tag every word with
 * the thread's global index, and keep it for a Geometric(1/4) number of
 * rounds; after the last round everything left is verified and freed.
 * Per-warp cache depth d: up to d freed blocks per size class stay with
 * the warp and serve its next mallocs of that class without touching the
 * heap (d = 0: every call goes to the heap).
 */
#ifndef KMA_BATCH_H
#define KMA_BATCH_H

#include <stdint.h>
#include "kma.h"
#include "kma_structs.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct kma_batch_s *kma_batch_t;

typedef struct kma_batch_job {
	uint32_t threads; /* work-items of the job */
	uint32_t pad;
	uint64_t seed;    /* the job's PRNG seed */
} kma_batch_job;

typedef struct kma_batch_stats {
	uint64_t mallocs, frees, nulls, bad_tags;
	uint64_t fill_bytes, verify_bytes;
	uint64_t cache_hits;  /* mallocs served by the warp cache */
	uint64_t cache_puts;  /* frees kept by the warp cache */
	uint64_t retired;     /* blocks freed early because a thread's table was full */
	uint64_t refused;     /* NULL mallocs whose size exceeds the heap's largest
			       * request (superblock - 16); `nulls` counts them too,
			       * the rest of `nulls` found the heap exhausted */
} kma_batch_stats;

#define KMA_BATCH_MAX_CACHE 8

/* A batch of `njobs` jobs (<= 4096) running `rounds` rounds on heap h
 * (at most 16 GiB). */
int kma_batch_create(kma_heap_t h, const kma_batch_job *jobs, uint32_t njobs, uint32_t rounds,
		     kma_batch_t *out);
/* The same batch on the PMA heap p (at most 32 GiB): the same kernel,
 * compiled for the bump heap (kma_backend.cuh), as the reference runs its
 * drivers over pma.cl for comparison (test/tb_clArrayList.c:221-223).
 * Frees do nothing there, so the jobs need the sum of all their requests;
 * a run resets p first.  Cache depth must be 0. */
int kma_batch_create_pma(kma_pma_t p, const kma_batch_job *jobs, uint32_t njobs, uint32_t rounds,
			 kma_batch_t *out);
/* Call style of later runs and captures: KMA_MODE_WARP (the default:
 * kma_malloc_warp / kma_free_warp, and the warp cache) or KMA_MODE_PLAIN
 * (every thread calls kma_malloc / kma_free itself, the reference's
 * per-work-item calls, kma.cl:279-373; cache depth must be 0). */
int kma_batch_set_mode(kma_batch_t b, int mode);
int kma_batch_destroy(kma_batch_t b);
uint64_t kma_batch_items(kma_batch_t b);

/* One run, stream-ordered: heap reset, job seeding, then the persistent
 * rounds kernel (all rounds and the final drain in one launch).
 * block_dim 128/256/512 (0 = 256); cache_depth 0..KMA_BATCH_MAX_CACHE. */
int kma_batch_run(kma_batch_t b, uint32_t block_dim, uint32_t cache_depth, void *stream);
/* Capture the same run into a CUDA graph (replacing a previous one); the
 * capture happens on `stream`, which must not be the legacy default stream. */
int kma_batch_capture(kma_batch_t b, uint32_t block_dim, uint32_t cache_depth, void *stream);
/* Launch the captured graph on `stream`. */
int kma_batch_launch(kma_batch_t b, void *stream);
/* Counters of the last run (synchronises the stream). */
int kma_batch_stats_get(kma_batch_t b, void *stream, kma_batch_stats *out);

typedef struct kma_batch_tune_entry {
	uint32_t sb_size_log2, block_dim, cache_depth;
	uint32_t serves_all;   /* 1 when the superblock size serves every size the
				* jobs draw (up to 4096 bytes); only such entries win */
	float ms;              /* mean device time of one captured run */
	float mops;            /* (mallocs + frees) / time, M ops/s */
	kma_batch_stats stats; /* of the last timed run */
} kma_batch_tune_entry;

/* Autotuner: for every superblock size in sb_log2s (each a fresh heap of
 * heap_bytes on `device`), block dim in block_dims and cache depth in
 * depths (heaps with at most `shards` class-table shards per class, 0 =
 * the heap default), capture the run as a graph, launch it `warmup` times untimed and
 * `reps` times timed (CUDA events), and record the entry; *best is the
 * index of the configuration with the most successful calls per second
 * (mallocs that returned a block, plus frees) among those whose superblock
 * size serves every size the jobs draw (4 KiB superblocks serve at most
 * 4080 bytes, so they cannot) and whose runs kept every tag intact and set
 * no heap error flag; 0xffffffff when none qualifies.
 * entries must hold n_sb * n_bd * n_depth entries. */
int kma_batch_autotune(const kma_batch_job *jobs, uint32_t njobs, uint32_t rounds, uint64_t heap_bytes,
		       uint32_t shards,
		       const uint32_t *sb_log2s, uint32_t n_sb, const uint32_t *block_dims, uint32_t n_bd,
		       const uint32_t *depths, uint32_t n_depth, uint32_t warmup, uint32_t reps, int device,
		       kma_batch_tune_entry *entries, uint32_t *best);

#ifdef __cplusplus
}
#endif

#endif /* KMA_BATCH_H */
