/*
 * kma.h -- host C ABI of the B200 KMA heap (libkma_b200.so).
 *
 * Plain C: opaque handles, plain pointers and sizes, integer error codes.
 * Device code uses include/kma_device.cuh (kma_malloc/kma_free and the
 * lock-free structures); kma_heap_device_ptr() hands a heap to a kernel.
 *
 * Each entry point names the reference interface it replaces.  The
 * reference's host calls take (cl_device_id, cl_context, cl_command_queue,
 * cl_program): here the device is a CUDA ordinal, the command queue a
 * cudaStream_t passed as void* (NULL = legacy default stream), and the
 * context/program are the device's primary context and this library.
 * Unlike the reference (which prints and returns NULL, kma.c:39-41,
 * 112-114) errors are returned as KMA_E* codes; the library owns the
 * device memory it allocates (the reference leaves the cl_mem to the
 * caller, test/tb_kma.c:316) and frees it in the *_destroy calls.
 * Calls on one handle are stream-ordered and not thread-safe.
 */
#ifndef KMA_H
#define KMA_H

#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define KMA_OK 0
#define KMA_EINVAL (-1)
#define KMA_ENOMEM (-2)
#define KMA_ECUDA (-3)
#define KMA_ETIMEDOUT (-4)
#define KMA_ENODEV (-5)
#define KMA_EFAULT (-6)

/* heap error flags (kma_error_flags) */
#define KMA_FLAG_TIMEOUT 1u  /* a bounded device spin expired */
#define KMA_FLAG_BADFREE 2u  /* free of a pointer that is not a live block */
/* bits 8..16 name the wait that set KMA_FLAG_TIMEOUT (KMA_ERR_AT_* in
 * kma_device.cuh): MS queue, ring enqueue, ring count, ring dequeue, plain
 * claim, plain reservation, plain free, warp reservation, warp turns */

/* allocation modes of the workload / replay kernels */
#define KMA_MODE_PLAIN 0     /* per-thread kma_malloc / kma_free */
#define KMA_MODE_WARP 1      /* warp-collaborative kma_malloc_warp / kma_free_warp */
#define KMA_MODE_PROFILE 2   /* flag for kma_wl_rounds/kma_wl_drain: also count the cycles
			      * each warp spends per phase (kma_wl_phase_cycles) */

typedef struct kma_heap_s *kma_heap_t;
struct kma_heap; /* device-side header, see kma_device.cuh */

/* kma_config.flags */
#define KMA_CFG_COMPAT 1u /* the reference's structures: one class table and the
			   * tagged-CAS MS queue as the superblock free list */

typedef struct kma_config {
	uint32_t sblocks;      /* superblocks, as kma_create(..., sblocks) (kma.c:79) */
	uint32_t sb_size_log2; /* 12..16: 4 KiB (the reference's KMA_SB_SIZE, kma.h:27) .. 64 KiB */
	uint32_t spin_limit;   /* bound on every device spin; 0 = default (1<<22) */
	int32_t device;        /* CUDA ordinal; -1 = current device */
	uint32_t shards;       /* most class-table shards per class (1..2048); a warp uses
				* shard (global warp id) % shards(class).  Each class gets
				* (sblocks-1)/32 shards clamped to [1, shards]; 0 = 2048.
				* COMPAT forces 1 (the reference's single table) */
	uint32_t flags;        /* KMA_CFG_* */
} kma_config;

typedef struct kma_info {
	uint64_t region_bytes;   /* sblocks << sb_size_log2 */
	uint64_t device_bytes;   /* total device memory owned by the heap */
	uint32_t sblocks, pages, sb_size_log2, nclasses;
	uint32_t max_request;    /* largest request served: SB - 16 (kma.cl:126) */
	uint32_t cls_size[16];   /* block size per class (kma.cl:55-90) */
	uint32_t cls_slots[16];  /* slots per superblock per class (kma.cl:95-113) */
	uint32_t cls_shards[16]; /* class-table shards per class */
	uint32_t cls_lines;      /* class-table words in all: sum of cls_shards */
	uint32_t flags;          /* KMA_CFG_* in effect */
} kma_info;

/* ---- size-class tables: pure host functions, no GPU needed ---------- */
/* kma.cl:55-90 (_kma_size_by_sbid); sbid == nclasses divides by zero in
 * the reference (kma.cl:61,87) and returns 0 here, like out-of-range ids */
uint32_t kma_size_by_sbid(uint32_t sb_size_log2, int sbid);
/* kma.cl:95-113 (_kma_slots_by_size) */
int kma_slots_by_size(uint32_t sb_size_log2, uint64_t size);
/* kma.cl:119-148 (_kma_sbid_by_size): smallest class >= size, -1 above
 * SB-16; sizes 0..3 give class 0 */
int kma_sbid_by_size(uint32_t sb_size_log2, uint64_t size);

/* ---- heap lifetime ---------------------------------------------------- */
/* kma.c:79-127 kma_create(dev, ctx, cq, prg, sblocks) with 4 KiB
 * superblocks: NULL when sblocks == 0 or on any error.  Blocking. */
kma_heap_t kma_create(int device, void *stream, unsigned int sblocks);
/* kma_create with a full configuration; returns KMA_OK or KMA_E*. */
int kma_create_ex(const kma_config *cfg, void *stream, kma_heap_t *out);
/* Frees the heap's device memory (the reference's clReleaseMemObject,
 * test/tb_kma.c:316; the reference has no kma_destroy). */
int kma_destroy(kma_heap_t h);
/* Re-initialise in place, stream-ordered: the state clheap_init
 * (kma.cl:27-52) leaves, written by parallel bulk stores. */
int kma_reset(kma_heap_t h, void *stream);
/* The struct kma_heap* that kernels pass to kma_malloc/kma_free. */
struct kma_heap *kma_heap_device_ptr(kma_heap_t h);
int kma_get_info(kma_heap_t h, kma_info *out);
/* Sticky device error flags (KMA_FLAG_*); clear != 0 resets them.
 * Synchronises the stream. */
int kma_error_flags(kma_heap_t h, void *stream, uint32_t *flags, int clear);
/* Stream-ordered copy of the error flags into *dst (device or pinned host
 * memory), without waiting: lets a caller record the flags of each of
 * several queued runs (a reset clears them).  No counterpart in the
 * reference. */
int kma_error_flags_async(kma_heap_t h, void *stream, uint32_t *dst);
const char *kma_strerror(int err);
/* Library build id string. */
const char *kma_version(void);

/* ---- heap image for checkers ------------------------------------------ */
/* Copies to host (any NULL destination is skipped), synchronising stream:
 *   cls[cls_lines]   raw class-table words, class-major: class c's shards
 *                    are words [sum of cls_shards[<c]] .. + cls_shards[c]
 *                    (0 empty, 1 POISON, s+2 superblock s)
 *   state[sblocks]   class<<28 | slots<<14 | free
 *   freelist[sblocks], *freelist_len: the superblock free list in FIFO
 *                    order, head (the next one handed out) first; length
 *                    UINT64_MAX if the list does not end (a cycle)
 * region_off/len: bytes of the superblock region (offset from the first
 * superblock) copied to region_dst. */
int kma_snapshot(kma_heap_t h, void *stream, uint32_t *cls, uint32_t *state,
		uint32_t *freelist, uint64_t *freelist_len, uint64_t region_off,
		uint64_t region_len, void *region_dst);
/* Gather the allocation bitmap of every superblock into dst
 * (sblocks x words u32, word k of superblock s at dst[s*words + k]),
 * words = ceil(slots of class 0 / 32).  Device pointer dst. */
int kma_gather_bitmaps(kma_heap_t h, void *stream, uint32_t *dst_dev, uint32_t words);

/* ---- heap images: save and restore ------------------------------------- */
/* A heap image is a position-independent copy of a heap's whole state: the
 * class table, the per-superblock state and home shard, the free list and
 * the superblock region (blocks, residue words and bitmaps).  Every link
 * the heap keeps is a superblock index or an offset from the first
 * superblock, so an image loads into any heap of the same geometry -- in
 * another process, on another GPU, at another address -- and the loaded
 * heap hands out the same offsets the saved one would have.  (Pointers
 * that callers stored inside their blocks are theirs to relocate.)  The
 * reference has no counterpart; its heap is one cl_mem buffer a host can
 * only copy verbatim into the same context.
 *
 * Layout (little-endian): this header, then the sections at the offsets it
 * gives, each 256-byte aligned:
 *   off_cls     u32[cls_lines]  class words, class-major (0 empty, s+2
 *                               superblock s; see kma_snapshot)
 *   off_state   u32[sblocks]    class<<28 | slots<<14 | free
 *   off_home    u16[sblocks]    home shard of each superblock
 *   off_flist   u64[flist_words] free-list words: ring slots {seq:32 | sb:32}
 *                               (ring != 0) or MS-queue links {tag:32 | idx+1:32}
 *   off_region  u8[sblocks << sb_log2] the superblocks */
#define KMA_IMAGE_MAGIC "KMAHEAP1"
#define KMA_IMAGE_VERSION 1u
typedef struct kma_image_header {
	char magic[8];            /* KMA_IMAGE_MAGIC, no terminator */
	uint32_t version;         /* KMA_IMAGE_VERSION */
	uint32_t header_bytes;    /* sizeof(kma_image_header) */
	uint32_t sb_log2, sblocks, pages;
	uint32_t ring;            /* 1: ticket-ring free list, 0: MS queue */
	uint32_t nclasses, cls_lines, flist_words;
	uint32_t err;             /* the heap's KMA_FLAG_* word */
	uint64_t free_head, free_tail; /* ring tickets, or MS-queue {tag | idx+1} words */
	uint32_t ring_avail, reserved;
	uint32_t cls_shards[16];  /* shards of each class (nclasses used) */
	uint64_t off_cls, off_state, off_home, off_flist, off_region;
	uint64_t total_bytes;     /* the image's size */
} kma_image_header;

/* Bytes an image of h takes (header, metadata and the superblock region). */
int kma_image_bytes(kma_heap_t h, uint64_t *bytes);
/* Write an image of h to dst (host or device memory, dst_bytes >=
 * kma_image_bytes), stream-ordered after earlier work on `stream`, and
 * wait for it.  The heap must be quiescent: no kernel on any stream may
 * use it meanwhile (an image with a refill in flight is refused by
 * kma_image_load).  KMA_EINVAL if dst_bytes is too small. */
int kma_image_save(kma_heap_t h, void *stream, void *dst, uint64_t dst_bytes);
/* Replace h's whole state with the image at src (host or device memory),
 * stream-ordered, and wait for it.  h keeps its own spin limit.  Returns
 * KMA_EINVAL, leaving h unchanged, when the image is truncated, of another
 * version, of a heap of other geometry (superblock size, superblocks,
 * free-list kind, shards per class), or holds any word that could address
 * outside the heap (a class word, a free-list entry or a home shard out of
 * range, a state with an unknown class or more free than slots, a refill
 * in flight). */
int kma_image_load(kma_heap_t h, void *stream, const void *src, uint64_t src_bytes);

/* ---- serial replay ---------------------------------------------------- */
/* One-thread-at-a-time replay of an op stream on the device:
 * ops[2i] = kind, ops[2i+1] = arg; kind 0 = malloc(arg) -> out[i] = offset
 * of the block from the first superblock or -1 (NULL); kind 1 =
 * free(block of op out[arg]) (arg < 0: free(NULL)) -> out[i] = 0.
 * mode KMA_MODE_PLAIN or KMA_MODE_WARP (one active lane).  *_dev: device
 * pointers; the _host form copies in and out (synchronous). */
int kma_replay(kma_heap_t h, const int64_t *ops_dev, int64_t n, int64_t *out_dev, int mode,
		void *stream);
int kma_replay_host(kma_heap_t h, const int64_t *ops, int64_t n, int64_t *out, int mode);

/* ---- stress workloads (the per-work-item programs of kma.cl:424-526
 *      generalised; see oracle/workload.h for the exact programs) ------- */
#define KMA_WL_C1 1  /* malloc / tag every word / verify / free per round */
#define KMA_WL_C2 2  /* malloc per round, free a seeded 50% of the live set */

typedef struct kma_wl_s *kma_wl_t;

typedef struct kma_wl_stats {
	uint64_t mallocs, frees, nulls, bad_tags;
	uint64_t offset_hash;   /* XOR over items of each item's ordered hash */
	uint64_t fill_bytes;    /* payload bytes tagged after malloc */
	uint64_t verify_bytes;  /* payload bytes verified before free */
} kma_wl_stats;

/* Workload state for `items` work-items: per-item PRNG, live-block table
 * (32 entries) and counters, in device scratch memory owned by the
 * handle. */
int kma_wl_create(kma_heap_t h, int program, uint64_t items, kma_wl_t *out);
int kma_wl_destroy(kma_wl_t w);
/* Seed every item (seed ^ gid*0x9E3779B97F4A7C15), empty live sets, zero counters. */
int kma_wl_begin(kma_wl_t w, uint64_t seed, void *stream);
/* Seed item g with seeds_dev[g] instead (device pointer). */
int kma_wl_begin_seeds(kma_wl_t w, const uint64_t *seeds_dev, void *stream);
/* Run rounds [r0, r0+nrounds) on every item concurrently (one thread per
 * item, block_dim threads per block; 0 = default 256). */
int kma_wl_rounds(kma_wl_t w, uint32_t nrounds, int mode, uint32_t block_dim, void *stream);
/* Free every live block (verifying its tags). */
int kma_wl_drain(kma_wl_t w, int mode, uint32_t block_dim, void *stream);
/* Deterministic one-thread version: round_major 0 runs items to
 * completion in gid order, 1 runs every item's round r before round r+1;
 * includes the drain. */
int kma_wl_serial(kma_wl_t w, uint32_t nrounds, int round_major, int mode, void *stream);
/* End to end from host buffers, the call a host program makes per batch:
 * reset the heap, copy seeds_host[items] in, seed every item, run
 * `nrounds` rounds, drain, copy each item's ordered malloc hash to
 * hashes_host[items] and the counters to *stats (either may be NULL).
 * Synchronous on `stream`; pinned host buffers make the copies async. */
int kma_wl_run_host(kma_wl_t w, const uint64_t *seeds_host, uint32_t nrounds, int mode,
		uint64_t *hashes_host, kma_wl_stats *stats, void *stream);
/* Allocation-free run.  No counterpart in the reference.  For hosts that
 * must not call cudaMalloc/cudaFree while they run a batch -- those calls
 * synchronise with the whole device, stalling every other stream a serving
 * loop keeps busy, and a host framework with its own caching allocator may
 * own the memory budget so that a private allocation fails -- this runs
 * the same workload as kma_wl_run_host (reset the heap, seed item g with
 * seeds_dev[g], `nrounds` rounds, drain; `serial` != 0 runs one thread,
 * round by round, like kma_wl_serial) without a kma_wl handle: the
 * per-item scratch (PRNG, live-block table, counters) lives in a fixed
 * KMA_WL_NOALLOC_SCRATCH_BYTES array inside the library, which every GPU
 * that loads the library holds until the process exits.  Inputs and
 * outputs are the caller's device memory: seeds_dev[items] in,
 * hashes_dev[items] (each item's ordered malloc hash) and *stats_dev out.
 * It allocates nothing.  items > KMA_WL_NOALLOC_MAX_ITEMS returns
 * KMA_EINVAL.  The first call on a device looks up the array's device
 * address (cudaGetSymbolAddress), so make that first call before any
 * stream capture.  Every call reuses the same array (each call clears
 * what must start at zero): calls that overlap on the GPU, on any stream,
 * race and corrupt each other.  Stream-ordered; returns before the work
 * completes. */
#define KMA_WL_NOALLOC_MAX_ITEMS 8192
#define KMA_WL_NOALLOC_SCRATCH_BYTES (4u << 20)
int kma_wl_run_noalloc(kma_heap_t h, int program, uint64_t items, const uint64_t *seeds_dev,
		uint32_t nrounds, int mode, int serial, uint64_t *hashes_dev, kma_wl_stats *stats_dev,
		void *stream);
/* Counters to host (synchronises the stream). */
int kma_wl_stats_get(kma_wl_t w, void *stream, kma_wl_stats *out);
/* Cycles summed over warps since kma_wl_begin, per phase of the C2 round,
 * for runs launched with KMA_MODE_PROFILE: [0] malloc, [1] tag fill,
 * [2] verify, [3] free (synchronises the stream). */
int kma_wl_phase_cycles(kma_wl_t w, void *stream, uint64_t cycles[4]);
/* Event counts of kma_malloc_warp in KMA_MODE_PROFILE runs since
 * kma_wl_begin, indexed by KMA_T_* of kma_device.cuh (leader turns,
 * reservation attempts, POISON waits, stale slots, lost CASes, refills,
 * claim steps, empty claim steps). */
int kma_wl_tally(kma_wl_t w, void *stream, uint64_t counts[8]);
/* Per-item ordered malloc hashes (device pointer, items x u64). */
const uint64_t *kma_wl_item_hashes(kma_wl_t w);
/* Live blocks to host: nlive[items], off[32*items] (entry i of item g at
 * i*items+g; offsets from the first superblock), size[32*items]. */
int kma_wl_live(kma_wl_t w, void *stream, uint32_t *nlive, uint64_t *off, uint32_t *size);

/* ---- fault injection (tests) ------------------------------------------ */
/* No counterpart in the reference.  Writes raw class-table word `cls`
 * (0 empty, 1 POISON, s+2 superblock s), stream-ordered.  Setting POISON
 * with no refill in flight makes every request of that class wait on a
 * flag nothing clears: each one gives up after the heap's spin_limit,
 * returns NULL and raises KMA_FLAG_TIMEOUT, with no device fault. */
int kma_debug_set_class_word(kma_heap_t h, uint32_t cls, uint32_t value, void *stream);

/* ---- microbenchmarks -------------------------------------------------- */
/* L2 atomic throughput: `threads` threads each do `iters` 32-bit
 * atomicAdd (returning form) on a private word spaced stride_words apart
 * (distinct != 0) or all on one word (distinct == 0).  Device scratch is
 * allocated and freed inside.  Returns elapsed milliseconds (CUDA events)
 * in *ms. */
int kma_bench_atomics(int distinct, uint64_t threads, uint32_t iters, uint32_t stride_words,
		void *stream, float *ms);

#ifdef __cplusplus
}
#endif
#endif /* KMA_H */
