/*
 * kma_structs.h -- host C ABI of the lock-free structures and the PMA bump
 * heap (libkma_b200.so); device code is in kma_structs.cuh.
 *
 * Conventions as kma.h: CUDA ordinal for the device (-1 = current), a
 * cudaStream_t passed as void* (NULL = legacy default stream), KMA_E*
 * return codes, the library owns the device memory it allocates and frees
 * it in *_destroy.  Each create call replaces the reference's host create
 * call (which takes an OpenCL device, context, queue and program and
 * returns a cl_mem the caller releases) and runs the structure's init
 * kernel on the stream.
 *
 * The *_replay_host calls run an op stream one operation at a time (one
 * device thread) and are what the parity tests compare with the reference;
 * kma_c3_* run the concurrent microbenchmarks.
 */
#ifndef KMA_STRUCTS_H
#define KMA_STRUCTS_H

#include <stdint.h>
#include <stddef.h>
#include "kma.h"

#ifdef __cplusplus
extern "C" {
#endif

/* ---- PMA bump heap ------------------------------------------------ */
typedef struct kma_pma_s *kma_pma_t;
struct kma_pma;

/* pma_create (pma.c:31-53 + clheap_init, pma.cl:24-30): a bump heap of
 * `bytes` data bytes (the reference's `sblocks` argument is a byte count).
 * Allocations are accepted up to bytes + 24 from the data base, as the
 * reference's limit check counts its 24-byte header (pma.cl:36); the
 * library allocates that slack. */
int kma_pma_create(uint64_t bytes, int device, void *stream, kma_pma_t *out);
int kma_pma_destroy(kma_pma_t p);
/* struct kma_pma* for kernels (kma_pma_malloc / kma_pma_free) */
struct kma_pma *kma_pma_device_ptr(kma_pma_t p);
/* device address of the data base (offsets in replays are from here) */
void *kma_pma_base(kma_pma_t p);
/* head back to 0 (clheap_init again), stream-ordered */
int kma_pma_reset(kma_pma_t p, void *stream);
/* current head (bytes handed out, including refused requests) */
int kma_pma_head(kma_pma_t p, void *stream, uint64_t *head);
/* ops (n x 2 int64, host): (0, size) malloc -> offset from the data base or
 * -1; (1, k) free the result of op k -> 0.  One device thread. */
int kma_pma_replay_host(kma_pma_t p, const int64_t *ops, int64_t n, int64_t *out);

/* ---- structure handles ----------------------------------------------- */
typedef struct kma_clqueue_s *kma_clqueue_t;
typedef struct kma_iqueue_s *kma_iqueue_t;
typedef struct kma_cltree_s *kma_cltree_t;
typedef struct kma_clarraylist_s *kma_clarraylist_t;
struct kma_clqueue;
struct kma_iqueue;
struct kma_cltree;
struct kma_clarraylist;

/* clQueue_create (clQueue.c:62-104) + clQueue_init: an empty queue. */
int kma_clqueue_create(int device, void *stream, kma_clqueue_t *out);
int kma_clqueue_destroy(kma_clqueue_t q);
struct kma_clqueue *kma_clqueue_device_ptr(kma_clqueue_t q);

/* clIndexedQueue_create (clIndexedQueue.c:64-113) + clIndexedQueue_init:
 * items are the `capacity` slots of (1 << stride_l2) bytes at the device
 * address `base` (stride_l2 >= 3: an item's first 8 bytes are its link);
 * `first` (one of them) becomes the dummy.  shards: 1 = the reference's
 * queue; up to 4096 independent queues over the same items, picked by
 * global thread id. */
int kma_iqueue_create(void *base, uint32_t stride_l2, uint32_t capacity, void *first,
		      uint32_t shards, int device, void *stream, kma_iqueue_t *out);
int kma_iqueue_destroy(kma_iqueue_t q);
struct kma_iqueue *kma_iqueue_device_ptr(kma_iqueue_t q);
/* KMA_FLAG_TIMEOUT when a spin expired; clear != 0 resets it */
int kma_iqueue_error_flags(kma_iqueue_t q, void *stream, uint32_t *flags, int clear);

/* An empty clTree (clTree.h:30-32: one root pointer; the reference's
 * driver allocates it itself, test/tb_clTree.c). */
int kma_cltree_create(int device, void *stream, kma_cltree_t *out);
int kma_cltree_destroy(kma_cltree_t t);
struct kma_cltree *kma_cltree_device_ptr(kma_cltree_t t);

/* clArrayList_create (clArrayList.c:58-104) + clArrayList_init: an empty
 * list of obj_size-byte objects on a KMA heap or a PMA heap (exactly one
 * non-NULL), on that heap's device. */
int kma_clarraylist_create(uint32_t obj_size, kma_heap_t kma, kma_pma_t pma, void *stream,
			   kma_clarraylist_t *out);
int kma_clarraylist_destroy(kma_clarraylist_t l);
struct kma_clarraylist *kma_clarraylist_device_ptr(kma_clarraylist_t l);

/* ---- clQueue ------------------------------------------------------- */
/* One-thread replay of a clQueue (clQueue.cl:27-118) over `n_items` items
 * of 16 bytes that the call allocates: ops (0, i) enqueue item i -> 1/0,
 * (1, 0) dequeue -> item index or -1 when empty.  final (n_items + 2
 * int64): head item, tail item, then each item's link as an item index,
 * -1 for NULL, -2 for POISON. */
int kma_clqueue_replay_host(uint32_t n_items, const int64_t *ops, int64_t n, int64_t *out,
			    int64_t *final_state);

/* ---- clIndexedQueue ------------------------------------------------- */
/* One-thread replay of an indexed queue (clIndexedQueue.cl:93-290) over
 * items 0..n_items-1 of (1 << stride_l2) bytes that the call allocates;
 * item 0 is the initial dummy (clIndexedQueue_init's `first`).  ops (0, i)
 * enqueue item i -> 1/0, (1, 0) dequeue -> item index (the old dummy) or
 * -1.  final (n_items + 2): head item, tail item, then each item's link as
 * an item index (-1 = none). */
int kma_iqueue_replay_host(uint32_t n_items, uint32_t stride_l2, const int64_t *ops, int64_t n,
			   int64_t *out, int64_t *final_state);

/* ---- fault injection (tests) ------------------------------------------ */
/* No counterpart in the reference.  Builds a stuck queue on the device and
 * runs one dequeue on it with the given spin limit: kind KMA_C3_CLQUEUE
 * with state 0 (the head item's link left POISON by a dequeuer that is
 * gone) or 1 (an append that exchanged the tail and never linked), kind
 * KMA_C3_IQUEUE with state 0 (the head's hold tag left odd).  Nothing ever
 * frees the queue, so the dequeue gives up after spin_limit tries in which
 * the head did not move: *taken = -1 (NULL), *flags = the error flags it
 * raised (KMA_FLAG_TIMEOUT), no device fault.  KMA_EINVAL for other
 * kinds / states. */
int kma_debug_queue_stuck_dequeue(int kind, int state, uint32_t spin_limit, int device, int64_t *taken,
				  uint32_t *flags);

/* No counterpart in the reference.  FIFO order through the warp and block
 * forms, in one block of `tpb` threads (a multiple of 32, at most 512):
 * for each of `calls` rounds the block's warps append 32 items each, one
 * warp after another (warp forms, chain log on); then the block makes
 * `calls` block-form dequeues.  out[c * tpb + t] = the item thread t got
 * in dequeue c, as its enqueue number (0, 1, ...; the indexed queue's
 * initial dummy comes out first as -2), -1 for NULL.  *err: error flags.
 * kind: KMA_C3_CLQUEUE or KMA_C3_IQUEUE. */
int kma_debug_queue_block_fifo(int kind, uint32_t tpb, uint32_t calls, int device, int64_t *out, uint32_t *err);

/* ---- clTree ---------------------------------------------------------- */
/* One-thread replay of a clTree (clTree.cl:27-74) with one 24-byte node per
 * op that the call allocates: ops (0, key) add -> 1 inserted, 0 exists,
 * 2 revived; (1, key) get -> op index of the node found or -1; (2, key)
 * remove (logical) -> 1/0.  keys_out receives the live keys in order
 * (capacity n), *n_keys their count. */
int kma_cltree_replay_host(const int64_t *ops, int64_t n, int64_t *out, uint32_t *keys_out,
			   int64_t *n_keys);

/* ---- clArrayList ----------------------------------------------------- */
/* One-thread replay of a clArrayList (clArrayList.cl:23-216) created on
 * the given heap (exactly one of kma / pma non-NULL): ops (0, objs) grow
 * -> offset of the objects from the heap's data base (the first
 * superblock for KMA) or -1; (1, i) get -> offset or -1; (2, 0) clear ->
 * 0; (3, objs) grow through the warp form by lane 0 alone -> offset or -1. */
int kma_clarraylist_replay_host(kma_heap_t kma, kma_pma_t pma, uint32_t obj_size,
				const int64_t *ops, int64_t n, int64_t *out);
/* One group of n threads (1..1024) grows a fresh list together
 * (clArrayList_grow_local, clArrayList.cl:111-176): mode 0 = one block
 * (kma_clarraylist_grow_block), mode 1 = each warp on its own
 * (kma_clarraylist_grow_warp).  out[t] = offset of thread t's objects from
 * the heap's data base, or -1. */
int kma_clarraylist_group_host(kma_heap_t kma, kma_pma_t pma, uint32_t obj_size,
			       const uint32_t *objs, uint32_t n, int mode, int64_t *out);

/* ---- chain log (kma_structs.cuh) ----------------------------------------- */
/* A log of `records` (a power of two, at most 2^24) chain records for the
 * warp forms of the queues: warp enqueues record each chain's items, warp
 * dequeues take a recorded chain at the head in one step instead of
 * walking it.  256 bytes per record; records are reused round robin and
 * are only hints (checked against the queue before use), so any size is
 * correct and a size at least the number of chains queued at once is
 * fastest.  No counterpart in the reference. */
typedef struct kma_chain_log_s *kma_chain_log_t;
struct kma_chain_log;
int kma_chain_log_create(uint32_t records, int device, void *stream, kma_chain_log_t *out);
int kma_chain_log_destroy(kma_chain_log_t l);
/* struct kma_chain_log* to pass to kma_clqueue_enqueue_warp / _dequeue_warp */
struct kma_chain_log *kma_chain_log_device_ptr(kma_chain_log_t l);
/* Attach a log to an indexed queue's warp forms (NULL detaches). */
int kma_iqueue_set_chain_log(kma_iqueue_t q, kma_chain_log_t l, void *stream);

/* ---- concurrent microbenchmarks -------------------------------------- */
#define KMA_C3_CLQUEUE 0
#define KMA_C3_IQUEUE 1
/* or'ed into the kind: every enqueue and dequeue through the warp forms
 * (kma_clqueue_enqueue_warp / _dequeue_warp, kma_iqueue_enqueue_warp_shard
 * / _dequeue_warp_shard): a warp's items for one queue go in as one chain
 * and its dequeues take consecutive items together; the queues get a
 * chain log of one record per 16 payloads (a power of two) */
#define KMA_C3_WARP 0x100
/* or'ed into the kind: enqueues through the warp forms, dequeues through
 * the block forms (kma_clqueue_dequeue_block, kma_iqueue_dequeue_block):
 * a block of 256 threads takes its items with one thread, several logged
 * chains per hold of the head.  One queue only (shards must be 1). */
#define KMA_C3_BLOCK 0x200

typedef struct kma_c3_queue_stats {
	uint64_t enqueued;       /* successful enqueues */
	uint64_t dequeued;       /* items returned by dequeue (for the indexed queue
				  * including the initial dummies) */
	uint64_t empty;          /* dequeues that found the queue empty */
	uint64_t remaining;      /* items still linked after the dequeue phase */
	uint64_t out_count;      /* payloads seen (dequeued + remaining) */
	uint64_t out_xor, out_sum;   /* over the payloads seen */
	uint64_t in_xor, in_sum;     /* over the payloads enqueued */
	uint32_t err;            /* KMA_FLAG_TIMEOUT if a spin expired */
	uint32_t walk_ok;        /* 1 when every shard's list ends at its tail with no cycle */
	float enqueue_ms, dequeue_ms;
	uint32_t log_chains;     /* warp forms: chains dequeued whole from their log records */
	uint32_t pad;
} kma_c3_queue_stats;

/* Config-3 queue run: `threads` device threads each enqueue `per_thread`
 * items carrying a seeded permutation of 0..n-1 (n = threads * per_thread
 * payloads, u32), then each dequeues `per_thread` times; conservation is
 * checked on the device (multiset hashes of payloads in vs. out, plus a
 * walk of what is left).  shards: 1 = the reference's single queue; more
 * spreads threads over independent queues (FIFO per shard). */
int kma_c3_queue_run(int kind, uint32_t threads, uint32_t per_thread, uint32_t shards,
		     uint64_t seed, int device, kma_c3_queue_stats *st);

typedef struct kma_c3_tree_stats {
	uint64_t live_keys;      /* live keys after the run (in-order walk) */
	uint64_t keys_xor, keys_sum; /* over the live keys */
	uint32_t sorted;         /* 1 when the in-order walk is strictly increasing */
	uint32_t err;
	float ms;
} kma_c3_tree_stats;

/* Config-3 tree run on host op arrays: op j is (kinds[j], keys[j]) with
 * kind 0 insert, 1 lookup, 2 remove; every op on a key runs on one thread
 * (owner = key % threads), in op order, so the result equals the
 * sequential replay.  results[j] receives the op's return (add: 1/0/2,
 * lookup: 1 found / 0, remove: 1/0).  Nodes come from a pool of one per op. */
int kma_c3_tree_run(const uint8_t *kinds, const uint32_t *keys, uint64_t n_ops, uint32_t threads,
		    int device, int8_t *results, kma_c3_tree_stats *st);

#ifdef __cplusplus
}
#endif

#endif /* KMA_STRUCTS_H */
