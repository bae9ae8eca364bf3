/*
 * kma_device.cuh -- device-side API of the B200 KMA heap (sm_100a).
 *
 * Drop-in for the reference's device API (clheap.h:37-39, kma.cl:279-373):
 *   void *kma_malloc(kma_heap *heap, size_t size);   NULL on failure
 *   void  kma_free(kma_heap *heap, void *p);         kma_free(h, NULL) is a no-op
 * plus warp-collaborative forms (any subset of a warp may call them, with
 * different sizes per lane):
 *   void *kma_malloc_warp(kma_heap *heap, size_t size);
 *   void  kma_free_warp(kma_heap *heap, void *p);
 * The lock-free structures (clqueue, clindexedqueue, cltree, clarraylist)
 * and the PMA bump heap are in kma_structs.cuh.
 *
 * Heap layout in HBM (one cudaMalloc per heap, owned by kma_create):
 *   [kma_heap header | sb_state[nsb] u32 | sb_home[nsb] u16 |
 *    free-list words | superblocks]
 *   Superblock s lives at sb_base + s*SB: bytes [0,12) are reserved so that
 *   every block offset equals the reference's (its in-band 12-byte header,
 *   kma.h:71-78); blocks start at +12; the allocation bitmap sits at the
 *   tail and grows downward (bitmap word k = slots 32k..32k+31 at u32 index
 *   SB/4-1-k, kma.cl:183-188).  The header fields live in coalesced side
 *   arrays: sb_state[s] = class<<28 | slots<<14 | free (the reference packs
 *   slots<<16 | free, kma.cl:180; the class field makes a stale reservation
 *   detectable) and sb_home[s] = the shard whose class table holds s.
 *
 * Class table (kma.h:84): each class c has cls_nsh[c] words ("shards"),
 * each 0 (empty), 1 (POISON, refill in progress) or s+2 (superblock s is
 * that shard's current superblock for class c), every one on its own
 * 128-byte line.  A warp uses shard (global warp id) % cls_nsh[c], so one
 * thread of warp 0 -- a serial replay -- always uses shard 0; a heap with
 * one shard per class is the reference's single table.  Only a shard's
 * current superblock is contended, so kma_create gives every class
 * pages/32 shards (at most 2048): enough to spread a full GPU's warps,
 * few enough that the superblocks pinned as shards' current ones leave
 * the heap room.
 *
 * Superblock free list, FIFO with the reference's order and its rule that
 * one superblock always stays behind as the queue's dummy
 * (clIndexedQueue.cl:254-290 returns the old dummy; the first superblock
 * handed out is superblock 0):
 *   KMA_HEAP_RING (default): a ticket ring -- fetch-and-add on the head and
 *     tail tickets, one {seq:32 | sb:32} word per slot, an availability
 *     count -- so concurrent refills do not retry CAS loops on one word;
 *   otherwise: the Michael-Scott queue with a dummy node over superblock
 *     indices, links in sb_next[] as 64-bit {tag:32 | idx+1:32} words
 *     (ABA-safe), as the reference builds it (clIndexedQueue.cl:194-290).
 *
 * One-thread-at-a-time execution never observes POISON, a lost CAS or a
 * second shard, so every configuration returns the reference's offsets
 * under serial replay.
 *
 * Every spin (POISON wait, CAS retry, queue helpers) is bounded by
 * heap->spin_limit iterations; on expiry the call fails (NULL / 0), sets
 * KMA_ERR_TIMEOUT in heap->err and never traps.
 */
#ifndef KMA_DEVICE_CUH
#define KMA_DEVICE_CUH

#include <stdint.h>
#include <stddef.h>

#define KMA_MAX_CLASSES 16
#define KMA_MAX_SHARDS 2048    /* per class */
#define KMA_MAX_CLS_LINES 32768 /* sum over classes */
#define KMA_SB_HDR 12u
#define KMA_POISON 1u
#define KMA_CLS_BASE 2u
/* classes with at most this many slots per superblock refill privately
 * instead of queueing behind another warp's refill (kma_malloc_warp) */
#define KMA_PRIVATE_REFILL_SLOTS 8u

#define KMA_ST_FREE_MASK 0x3fffu
#define KMA_ST_SLOTS_SHIFT 14
#define KMA_ST_CLASS_SHIFT 28

/* heap->flags */
#define KMA_HEAP_RING 1u

/* heap->err bits */
#define KMA_ERR_TIMEOUT 1u
#define KMA_ERR_BADFREE 2u
/* with KMA_ERR_TIMEOUT: which bounded wait expired */
#define KMA_ERR_AT_MSQ (1u << 8)        /* MS-queue free list */
#define KMA_ERR_AT_RING_ENQ (1u << 9)   /* ring: slot not yet released */
#define KMA_ERR_AT_RING_AVAIL (1u << 10)/* ring: availability count */
#define KMA_ERR_AT_RING_DEQ (1u << 11)  /* ring: slot not yet filled */
#define KMA_ERR_AT_CLAIM (1u << 12)     /* plain malloc: bitmap claim */
#define KMA_ERR_AT_MALLOC (1u << 13)    /* plain malloc: reservation */
#define KMA_ERR_AT_FREE (1u << 14)      /* plain free: count update */
#define KMA_ERR_AT_RESERVE (1u << 15)   /* warp malloc: reservation (POISON / stale waits) */
#define KMA_ERR_AT_WARP (1u << 16)      /* warp malloc: leader turns */

struct __align__(128) kma_line32 {
	uint32_t v;
	uint32_t pad_[31];
};
struct __align__(128) kma_line64 {
	unsigned long long v;
	unsigned long long pad_[15];
};

struct __align__(128) kma_heap {
	/* geometry: written by kma_create, read-only afterwards */
	unsigned char *sb_base;
	uint32_t *sb_state;
	uint16_t *sb_home;
	unsigned long long *sb_next; /* MS-queue links [nsb] (no KMA_HEAP_RING) */
	unsigned long long *ring;    /* ring slots [ring_cap] (KMA_HEAP_RING) */
	unsigned long long region_bytes; /* nsb << sb_log2 */
	uint32_t sb_log2;
	uint32_t sb_size;
	uint32_t nsb;        /* superblocks allocated (the reference's sblocks) */
	uint32_t pages;      /* superblocks on the free list: sblocks-1 (kma.cl:42) */
	uint32_t nclasses;   /* KMA_SB_SIZE_BUCKETS = log2 - 1 (kma.h:29) */
	uint32_t max_request;/* SB - 16 (kma.cl:126) */
	uint32_t spin_limit;
	uint32_t flags;
	uint32_t cls_lines;  /* sum of cls_nsh[] */
	uint32_t ring_cap;
	uint32_t cls_nsh[KMA_MAX_CLASSES];   /* shards per class */
	uint32_t cls_base[KMA_MAX_CLASSES];  /* first line of the class in cls[] */
	uint32_t cls_size[KMA_MAX_CLASSES];  /* kma.cl:55-90 */
	uint32_t cls_slots[KMA_MAX_CLASSES]; /* kma.cl:95-113 */
	uint32_t cls_magic[KMA_MAX_CLASSES]; /* floor(2^32/size)+1: exact x/size for x < 2^16 */
	uint32_t cls_words[KMA_MAX_CLASSES]; /* bitmap words = ceil(slots/32) */
	/* hot words, one line each */
	kma_line64 free_head; /* MS-queue head, or ring head ticket */
	kma_line64 free_tail; /* MS-queue tail, or ring tail ticket */
	kma_line32 ring_avail;
	kma_line32 err;
	kma_line32 cls[KMA_MAX_CLS_LINES];
};

/* ------------------------------------------------------------------ */
/* memory-model helpers (gpu scope)                                    */
/* ------------------------------------------------------------------ */
namespace kma_detail {

__device__ __forceinline__ uint32_t ld_relaxed(const uint32_t *p)
{
	uint32_t v;
	asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
	return v;
}
__device__ __forceinline__ uint32_t ld_relaxed16(const uint16_t *p)
{
	uint16_t v;
	asm volatile("ld.relaxed.gpu.global.u16 %0, [%1];" : "=h"(v) : "l"(p) : "memory");
	return v;
}
__device__ __forceinline__ uint32_t ld_acquire(const uint32_t *p)
{
	uint32_t v;
	asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
	return v;
}
__device__ __forceinline__ unsigned long long ld_acquire64(const unsigned long long *p)
{
	unsigned long long v;
	asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
	return v;
}
__device__ __forceinline__ void st_release(uint32_t *p, uint32_t v)
{
	asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ void st_release64(unsigned long long *p, unsigned long long v)
{
	asm volatile("st.release.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ uint32_t cas_acqrel(uint32_t *p, uint32_t cmp, uint32_t val)
{
	uint32_t old;
	asm volatile("atom.acq_rel.gpu.global.cas.b32 %0, [%1], %2, %3;"
		     : "=r"(old) : "l"(p), "r"(cmp), "r"(val) : "memory");
	return old;
}
__device__ __forceinline__ unsigned long long cas64_acqrel(unsigned long long *p,
		unsigned long long cmp, unsigned long long val)
{
	unsigned long long old;
	asm volatile("atom.acq_rel.gpu.global.cas.b64 %0, [%1], %2, %3;"
		     : "=l"(old) : "l"(p), "l"(cmp), "l"(val) : "memory");
	return old;
}
__device__ __forceinline__ uint32_t add_acqrel(uint32_t *p, uint32_t v)
{
	uint32_t old;
	asm volatile("atom.acq_rel.gpu.global.add.u32 %0, [%1], %2;"
		     : "=r"(old) : "l"(p), "r"(v) : "memory");
	return old;
}
__device__ __forceinline__ unsigned long long add64_acqrel(unsigned long long *p, unsigned long long v)
{
	unsigned long long old;
	asm volatile("atom.acq_rel.gpu.global.add.u64 %0, [%1], %2;"
		     : "=l"(old) : "l"(p), "l"(v) : "memory");
	return old;
}
__device__ __forceinline__ uint32_t or_acqrel(uint32_t *p, uint32_t v)
{
	uint32_t old;
	asm volatile("atom.acq_rel.gpu.global.or.b32 %0, [%1], %2;"
		     : "=r"(old) : "l"(p), "r"(v) : "memory");
	return old;
}
__device__ __forceinline__ uint32_t and_acqrel(uint32_t *p, uint32_t v)
{
	uint32_t old;
	asm volatile("atom.acq_rel.gpu.global.and.b32 %0, [%1], %2;"
		     : "=r"(old) : "l"(p), "r"(v) : "memory");
	return old;
}
__device__ __forceinline__ void fence_acqrel()
{
	asm volatile("fence.acq_rel.gpu;" ::: "memory");
}
/* Relaxed forms for the hot path.  Slot claims and releases are decided by
 * these atomics at L2, the coherence point; a claim is issued only after
 * the reservation it depends on has returned (the GPU does not speculate),
 * and the only plain stores another thread must see first -- a refill's
 * bitmap zeroing and a free's word-0 residue -- are fenced before their
 * publication (sb_format, and_release). */
__device__ __forceinline__ uint32_t cas_relaxed(uint32_t *p, uint32_t cmp, uint32_t val)
{
	uint32_t old;
	asm volatile("atom.relaxed.gpu.global.cas.b32 %0, [%1], %2, %3;"
		     : "=r"(old) : "l"(p), "r"(cmp), "r"(val) : "memory");
	return old;
}
/* Allocation-bitmap words sit at the superblock tails, in lines they
 * share with payload that the workloads write and read as evict-first
 * (streaming); their atomics ask L2 to keep the line (evict_last): the
 * claims and frees then find it in L2 (config 2's rounds launch measured
 * 7.58 vs 7.66 ms).  A cache hint only: ordering and results unchanged. */
__device__ __forceinline__ unsigned long long keep_policy()
{
	unsigned long long pol;
	asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(pol));
	return pol;
}
__device__ __forceinline__ uint32_t bm_or(uint32_t *p, uint32_t v)
{
	uint32_t old;
	asm volatile("atom.relaxed.gpu.global.or.L2::cache_hint.b32 %0, [%1], %2, %3;"
		     : "=r"(old) : "l"(p), "r"(v), "l"(keep_policy()) : "memory");
	return old;
}
__device__ __forceinline__ uint32_t bm_and(uint32_t *p, uint32_t v)
{
	uint32_t old;
	asm volatile("atom.relaxed.gpu.global.and.L2::cache_hint.b32 %0, [%1], %2, %3;"
		     : "=r"(old) : "l"(p), "r"(v), "l"(keep_policy()) : "memory");
	return old;
}
__device__ __forceinline__ uint32_t bm_and_release(uint32_t *p, uint32_t v)
{
	uint32_t old;
	asm volatile("atom.release.gpu.global.and.L2::cache_hint.b32 %0, [%1], %2, %3;"
		     : "=r"(old) : "l"(p), "r"(v), "l"(keep_policy()) : "memory");
	return old;
}
__device__ __forceinline__ uint32_t cas_release(uint32_t *p, uint32_t cmp, uint32_t val)
{
	uint32_t old;
	asm volatile("atom.release.gpu.global.cas.b32 %0, [%1], %2, %3;"
		     : "=r"(old) : "l"(p), "r"(cmp), "r"(val) : "memory");
	return old;
}
__device__ __forceinline__ unsigned long long add64_relaxed(unsigned long long *p, unsigned long long v)
{
	unsigned long long old;
	asm volatile("atom.relaxed.gpu.global.add.u64 %0, [%1], %2;"
		     : "=l"(old) : "l"(p), "l"(v) : "memory");
	return old;
}
__device__ __forceinline__ unsigned long long ld_relaxed64(const unsigned long long *p)
{
	unsigned long long v;
	asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
	return v;
}
__device__ __forceinline__ void st_relaxed64(unsigned long long *p, unsigned long long v)
{
	asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ uint32_t lane_id()
{
	uint32_t l;
	asm volatile("mov.u32 %0, %%laneid;" : "=r"(l));
	return l;
}
__device__ __forceinline__ uint32_t sm_id()
{
	uint32_t s;
	asm volatile("mov.u32 %0, %%smid;" : "=r"(s));
	return s;
}
__device__ __forceinline__ uint32_t lanemask_lt()
{
	uint32_t m;
	asm volatile("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
	return m;
}
/* position of the n-th (0-based) set bit of m, counting from bit 0;
 * requires n < popc(m) */
__device__ __forceinline__ uint32_t nth_set_bit(uint32_t m, uint32_t n)
{
	uint32_t pos = 0;
#pragma unroll
	for (uint32_t w = 16; w > 0; w >>= 1) {
		uint32_t c = __popc((m >> pos) & ((1u << w) - 1u));
		if (n >= c) {
			n -= c;
			pos += w;
		}
	}
	return pos;
}
__device__ __forceinline__ void backoff(uint32_t it)
{
	if (it > 4)
		__nanosleep(it < 64 ? 32u : 256u);
}
__device__ __forceinline__ void set_err(kma_heap *h, uint32_t e)
{
	atomicOr(&h->err.v, e);
}

/* state word */
__device__ __forceinline__ uint32_t st_free(uint32_t s) { return s & KMA_ST_FREE_MASK; }
__device__ __forceinline__ uint32_t st_slots(uint32_t s) { return (s >> KMA_ST_SLOTS_SHIFT) & KMA_ST_FREE_MASK; }
__device__ __forceinline__ uint32_t st_class(uint32_t s) { return s >> KMA_ST_CLASS_SHIFT; }
__device__ __forceinline__ uint32_t st_make(uint32_t c, uint32_t slots, uint32_t fr)
{
	return (c << KMA_ST_CLASS_SHIFT) | (slots << KMA_ST_SLOTS_SHIFT) | fr;
}

/* tagged index words {tag:32 | idx:32}, idx 0 = null, idx = item + 1 */
__device__ __forceinline__ uint32_t tw_idx(unsigned long long w) { return (uint32_t)w; }
__device__ __forceinline__ uint32_t tw_tag(unsigned long long w) { return (uint32_t)(w >> 32); }
__device__ __forceinline__ unsigned long long tw_make(uint32_t tag, uint32_t idx)
{
	return ((unsigned long long)tag << 32) | idx;
}

__device__ __forceinline__ unsigned char *sb_addr(const kma_heap *h, uint32_t s)
{
	return h->sb_base + ((size_t)s << h->sb_log2);
}
/* bitmap word k of superblock sb (u32 index SB/4-1-k from the SB start) */
__device__ __forceinline__ uint32_t *bitmap_word(const kma_heap *h, unsigned char *sb, uint32_t k)
{
	return reinterpret_cast<uint32_t *>(sb + h->sb_size) - 1 - k;
}
/* linear id of the calling warp in the grid (stable for its lifetime) */
__device__ __forceinline__ unsigned long long global_warp()
{
	unsigned long long blk = ((unsigned long long)blockIdx.z * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x;
	uint32_t tpb = blockDim.x * blockDim.y * blockDim.z;
	uint32_t t = (threadIdx.z * blockDim.y + threadIdx.y) * blockDim.x + threadIdx.x;
	return blk * ((tpb + 31) / 32) + t / 32;
}
__device__ __forceinline__ uint32_t my_shard(const kma_heap *h, uint32_t c)
{
	uint32_t n = h->cls_nsh[c];
	return n > 1 ? (uint32_t)(global_warp() % n) : 0u;
}
__device__ __forceinline__ uint32_t *cls_word(kma_heap *h, uint32_t c, uint32_t shard)
{
	return &h->cls[h->cls_base[c] + shard].v;
}

} /* namespace kma_detail */

/* ------------------------------------------------------------------ */
/* size classes (kma.cl:55-148)                                        */
/* ------------------------------------------------------------------ */

/* The reference's _kma_sbid_by_size (kma.cl:119-148) returns the smallest
 * class whose block size is >= size (its MSB approximation never starts
 * above that class, and it only ever walks up); sizes above SB-16 give -1.
 * Sizes 0..3 read an uninitialised variable there; here they map to
 * class 0, which is what a zero-initialised reference build returns. */
__device__ __forceinline__ int kma_class_of(const kma_heap *h, size_t size)
{
	if (size > __ldg(&h->max_request))
		return -1;
	uint32_t s = (uint32_t)size;
	int c = s < 4 ? 0 : (int)(29 - __clz(s)); /* floor(log2 s) - 2 */
	while (__ldg(&h->cls_size[c]) < s)
		c++;
	return c;
}

/* ------------------------------------------------------------------ */
/* superblock free list                                                */
/* ------------------------------------------------------------------ */
namespace kma_detail {

/* MS queue (clIndexedQueue.cl:194-247 idxd_enqueue).  Returns 1, or 0 on
 * spin-limit expiry. */
__device__ __forceinline__ int msq_enqueue(kma_heap *h, uint32_t s)
{
	unsigned long long *link = &h->sb_next[s];
	uint32_t idx = s + 1;
	unsigned long long old = *((volatile unsigned long long *)link);
	st_release64(link, tw_make(tw_tag(old) + 1, 0));
	uint32_t lim = h->spin_limit;
	for (uint32_t it = 0; it < lim; it++) {
		unsigned long long t = ld_acquire64(&h->free_tail.v);
		unsigned long long *tl = &h->sb_next[tw_idx(t) - 1];
		unsigned long long n = ld_acquire64(tl);
		if (t != ld_acquire64(&h->free_tail.v))
			continue;
		if (tw_idx(n) == 0) {
			if (cas64_acqrel(tl, n, tw_make(tw_tag(n) + 1, idx)) == n) {
				cas64_acqrel(&h->free_tail.v, t, tw_make(tw_tag(t) + 1, idx));
				return 1;
			}
		} else {
			cas64_acqrel(&h->free_tail.v, t, tw_make(tw_tag(t) + 1, tw_idx(n)));
		}
		backoff(it);
	}
	set_err(h, KMA_ERR_TIMEOUT | KMA_ERR_AT_MSQ);
	return 0;
}

/* MS queue dequeue (clIndexedQueue.cl:249-290): the superblock index, -1
 * when only the dummy is left, -2 on spin-limit expiry. */
__device__ __forceinline__ int64_t msq_dequeue(kma_heap *h)
{
	uint32_t lim = h->spin_limit;
	for (uint32_t it = 0; it < lim; it++) {
		unsigned long long hd = ld_acquire64(&h->free_head.v);
		unsigned long long t = ld_acquire64(&h->free_tail.v);
		unsigned long long n = ld_acquire64(&h->sb_next[tw_idx(hd) - 1]);
		if (hd != ld_acquire64(&h->free_head.v))
			continue;
		if (tw_idx(hd) == tw_idx(t)) {
			if (tw_idx(n) == 0)
				return -1;
			cas64_acqrel(&h->free_tail.v, t, tw_make(tw_tag(t) + 1, tw_idx(n)));
		} else if (cas64_acqrel(&h->free_head.v, hd, tw_make(tw_tag(hd) + 1, tw_idx(n))) == hd) {
			return (int64_t)tw_idx(hd) - 1;
		}
		backoff(it);
	}
	set_err(h, KMA_ERR_TIMEOUT | KMA_ERR_AT_MSQ);
	return -2;
}

/* Ticket ring.  Slot p % cap holds {seq:32 | sb:32}; seq == p+1 means
 * "filled by the enqueue with ticket p", seq == p means "free for the
 * enqueue with ticket p".  ring_avail counts completed enqueues not yet
 * claimed by a dequeue; a dequeue needs two (one stays behind, as the
 * reference's dummy does).  The ring carries only superblock numbers: the
 * enqueuer publishes with a release store (ordering its detach of the
 * superblock first), and everything a dequeuer then writes is addressed
 * through the number it read, so tickets, counts and the slot read are
 * relaxed; a count seen before its slot store only makes a dequeuer wait
 * on the slot's sequence number. */
__device__ __forceinline__ int ring_enqueue(kma_heap *h, uint32_t s)
{
	unsigned long long pos = add64_relaxed(&h->free_tail.v, 1ull);
	unsigned long long *slot = &h->ring[pos % h->ring_cap];
	uint32_t lim = h->spin_limit;
	for (uint32_t it = 0; it < lim; it++) {
		unsigned long long w = ld_relaxed64(slot);
		if ((uint32_t)(w >> 32) == (uint32_t)pos) {
			st_release64(slot, ((unsigned long long)(uint32_t)(pos + 1) << 32) | s);
			atomicAdd(&h->ring_avail.v, 1u);
			return 1;
		}
		backoff(it);
	}
	set_err(h, KMA_ERR_TIMEOUT | KMA_ERR_AT_RING_ENQ);
	return 0;
}

__device__ __forceinline__ int64_t ring_dequeue(kma_heap *h)
{
	int32_t *avail = reinterpret_cast<int32_t *>(&h->ring_avail.v);
	int32_t old = atomicSub(avail, 1);
	if (old < 2) {
		/* near empty: undo, then claim only a count that is really there */
		atomicAdd(avail, 1);
		int32_t a = (int32_t)ld_relaxed(&h->ring_avail.v);
		uint32_t lim = h->spin_limit, it = 0;
		for (;;) {
			if (a < 2)
				return -1;
			int32_t seen = (int32_t)atomicCAS((unsigned *)&h->ring_avail.v, (uint32_t)a, (uint32_t)(a - 1));
			if (seen == a)
				break;
			a = seen;
			if (++it >= lim) {
				set_err(h, KMA_ERR_TIMEOUT | KMA_ERR_AT_RING_AVAIL);
				return -2;
			}
		}
	}
	unsigned long long pos = add64_relaxed(&h->free_head.v, 1ull);
	unsigned long long *slot = &h->ring[pos % h->ring_cap];
	uint32_t lim = h->spin_limit;
	for (uint32_t it = 0; it < lim; it++) {
		unsigned long long w = ld_relaxed64(slot);
		if ((uint32_t)(w >> 32) == (uint32_t)(pos + 1)) {
			st_relaxed64(slot, (unsigned long long)(uint32_t)(pos + h->ring_cap) << 32);
			return (int64_t)(uint32_t)w;
		}
		backoff(it);
	}
	set_err(h, KMA_ERR_TIMEOUT | KMA_ERR_AT_RING_DEQ);
	return -2;
}

__device__ __forceinline__ int sb_enqueue(kma_heap *h, uint32_t s)
{
	return (h->flags & KMA_HEAP_RING) ? ring_enqueue(h, s) : msq_enqueue(h, s);
}
__device__ __forceinline__ int64_t sb_dequeue(kma_heap *h)
{
	return (h->flags & KMA_HEAP_RING) ? ring_dequeue(h) : msq_dequeue(h);
}

/* Prepare superblock s for class c: zero its bitmap except the bits in
 * [pre_lo, slots), which are pre-set (claimed by the refiller), record its
 * home shard, then publish state = (c, slots, free).  kma.cl:177-189, with
 * the bitmap written before the state becomes visible. */
__device__ __forceinline__ void sb_format(kma_heap *h, uint32_t s, uint32_t c, uint32_t pre_lo,
		uint32_t fr, uint32_t shard)
{
	unsigned char *sb = sb_addr(h, s);
	uint32_t slots = h->cls_slots[c];
	uint32_t words = h->cls_words[c];
	for (uint32_t k = 0; k < words; k++) {
		uint32_t lo = k * 32, hi = lo + 32;
		uint32_t v = 0;
		if (pre_lo < hi && slots > lo) {
			uint32_t a = pre_lo > lo ? pre_lo : lo;
			uint32_t b = slots < hi ? slots : hi;
			if (b > a) {
				uint32_t n = b - a;
				v = (n == 32 ? 0xffffffffu : ((1u << n) - 1u)) << (a - lo);
			}
		}
		*bitmap_word(h, sb, k) = v;
	}
	h->sb_home[s] = (uint16_t)shard;
	st_release(&h->sb_state[s], st_make(c, slots, fr));
}

} /* namespace kma_detail */

/* ------------------------------------------------------------------ */
/* plain per-thread malloc/free: the reference algorithm                */
/* (kma.cl:150-373) with its atomics, made safe against recycling:      */
/*  - a reservation CAS only succeeds on a state word whose class field */
/*    is the requested class (a stale cursor whose superblock was       */
/*    recycled for another class fails and retries);                   */
/*  - taking the last free slot detaches with CAS(cls, cursor, 0), not  */
/*    an unconditional exchange (kma.cl:217).                           */
/* In one-thread-at-a-time execution both are identical to the         */
/* reference, so serial replay returns the reference's offsets.         */
/* ------------------------------------------------------------------ */
namespace kma_detail {

/* A class slot that names a superblock which cannot serve its class (no
 * free count left, or recycled for another class) is cleared by the
 * thread that finds it, not waited on.  The thread that takes a
 * superblock's last slots clears the slot it read the superblock from;
 * if the superblock was recycled meanwhile and republished in another
 * shard's slot of the same class, that slot keeps naming it, full, until
 * all its blocks are freed -- and the threads waiting on that slot may be
 * the ones holding them.  Clearing at worst hides a superblock whose
 * slots were freed again since the read; it returns to the free list
 * when all its blocks are freed, as any detached one.  One-thread
 * execution never finds such a slot (a taker always clears the slot it
 * read), so serial replay is unchanged. */
__device__ __forceinline__ void clear_stale(uint32_t *clsw, uint32_t cur)
{
	cas_relaxed(clsw, cur, 0);
}

/* kma.cl:232-273: claim a bitmap bit at or above `hint` (wrapping),
 * write the hint into word 0 of the block. */
__device__ __forceinline__ void *sb_get_block(kma_heap *h, uint32_t s, uint32_t c, uint32_t hint)
{
	unsigned char *sb = sb_addr(h, s);
	uint32_t slots = h->cls_slots[c];
	uint32_t size = h->cls_size[c];
	uint32_t words = h->cls_words[c];
	uint32_t slot = hint;
	uint32_t lim = h->spin_limit;
	for (uint32_t it = 0; it < lim; it++) {
		uint32_t k = slot >> 5;
		uint32_t *wp = bitmap_word(h, sb, k);
		uint32_t v = ld_relaxed(wp);
		uint32_t valid = (k == words - 1 && (slots & 31)) ? ((1u << (slots & 31)) - 1u) : 0xffffffffu;
		uint32_t cand = ~v & valid & (0xffffffffu << (slot & 31));
		while (cand) {
			uint32_t b = __ffs(cand) - 1;
			uint32_t bit = 1u << b;
			uint32_t old = bm_or(wp, bit);
			if (!(old & bit)) {
				unsigned char *p = sb + KMA_SB_HDR + (size_t)(k * 32 + b) * size;
				*reinterpret_cast<uint32_t *>(p) = hint;
				return p;
			}
			cand &= ~old;
			cand &= ~bit;
		}
		slot = (k + 1) * 32;
		if (slot >= slots)
			slot = 0;
	}
	set_err(h, KMA_ERR_TIMEOUT | KMA_ERR_AT_CLAIM);
	return NULL;
}

} /* namespace kma_detail */

/* kma.cl:279-303 (with _kma_reserve_block, kma.cl:150-225) */
__device__ inline void *kma_malloc(kma_heap *h, size_t size)
{
	using namespace kma_detail;
	int c = kma_class_of(h, size);
	if (c < 0)
		return NULL;
	uint32_t shard = my_shard(h, (uint32_t)c);
	uint32_t *clsw = cls_word(h, (uint32_t)c, shard);
	uint32_t lim = h->spin_limit;
	for (uint32_t it = 0; it < lim; it++) {
		/* kma.cl:163: CAS 0 -> POISON doubles as the read of the slot */
		uint32_t cur = cas_relaxed(clsw, 0, KMA_POISON);
		if (cur == 0) {
			/* refill, kma.cl:166-195 */
			int64_t s = sb_dequeue(h);
			if (s < 0) {
				atomicExch(clsw, 0);
				return NULL;
			}
			uint32_t slots = h->cls_slots[c];
			sb_format(h, (uint32_t)s, c, slots, slots - 1, shard);
			/* kma.cl:191 publishes the superblock even when the refill
			 * took its only slot (1-slot classes); every later request
			 * of that class then spins on a full superblock until the
			 * block is freed (kma.cl:203-204).  Leave the class empty
			 * instead, which is what taking the last slot does. */
			cas_release(clsw, KMA_POISON, slots == 1 ? 0u : (uint32_t)s + KMA_CLS_BASE);
			return sb_get_block(h, (uint32_t)s, c, slots - 1);
		}
		if (cur == KMA_POISON) {
			backoff(it);
			continue;
		}
		uint32_t s = cur - KMA_CLS_BASE;
		uint32_t *stp = &h->sb_state[s];
		/* kma.cl:198 reads the state with atom_add(.., 0) */
		uint32_t st = atomicAdd(stp, 0u);
		if (st_class(st) != (uint32_t)c || st_free(st) == 0) {
			clear_stale(clsw, cur);
			continue;
		}
		uint32_t fr = st_free(st) - 1;
		if (cas_relaxed(stp, st, st - 1) != st)
			continue;
		if (fr == 0)
			cas_relaxed(clsw, cur, 0); /* kma.cl:216-218 */
		return sb_get_block(h, s, c, fr);
	}
	set_err(h, KMA_ERR_TIMEOUT | KMA_ERR_AT_MALLOC);
	return NULL;
}

namespace kma_detail {
/* Locate the superblock / class / slot of a live block. */
__device__ __forceinline__ bool block_locate(const kma_heap *h, const void *p, uint32_t &s,
		uint32_t &c, uint32_t &slot)
{
	size_t off = (const unsigned char *)p - h->sb_base;
	if (off >= h->region_bytes)
		return false;
	s = (uint32_t)(off >> h->sb_log2);
	uint32_t in = (uint32_t)(off & (h->sb_size - 1));
	uint32_t st = ld_relaxed(&h->sb_state[s]);
	c = st_class(st);
	if (st == 0 || in < KMA_SB_HDR || c >= h->nclasses)
		return false;
	slot = (uint32_t)(((unsigned long long)(in - KMA_SB_HDR) * h->cls_magic[c]) >> 32);
	return slot < h->cls_slots[c];
}

/* Return superblock s (class c) to the free list once all its slots are
 * free: kma.cl:362-367. */
__device__ __forceinline__ void sb_recycle(kma_heap *h, uint32_t s, uint32_t c)
{
	/* The home shard of this incarnation was stored before the release
	 * that published its state (sb_format).  This load issues only after
	 * the caller's CAS on that state has returned (it decides whether to
	 * recycle), and a gpu-scope relaxed load is served at L2, where that
	 * store already was: it sees the current home.  A plain load may be
	 * served from this SM's L1, where a line of sb_home read during an
	 * earlier incarnation can still sit: the slot of the old home would be
	 * cleared and the current one left naming a superblock on the free
	 * list. */
	uint32_t home = ld_relaxed16(&h->sb_home[s]);
	cas_relaxed(cls_word(h, c, home), s + KMA_CLS_BASE, 0);
	sb_enqueue(h, s);
}
} /* namespace kma_detail */

/* The start of the heap block that contains p (p may point inside it), or
 * NULL when p is not inside a superblock in use.  For structures that
 * place an aligned object inside a 4-byte aligned block and must free the
 * block itself.  No counterpart in the reference. */
__device__ __forceinline__ void *kma_block_of(kma_heap *h, const void *p)
{
	using namespace kma_detail;
	uint32_t s, c, slot;
	if (!p || !block_locate(h, p, s, c, slot))
		return NULL;
	return sb_addr(h, s) + KMA_SB_HDR + (size_t)slot * h->cls_size[c];
}

/* kma.cl:305-373 */
__device__ inline void kma_free(kma_heap *h, void *p)
{
	using namespace kma_detail;
	if (p == NULL)
		return;
	uint32_t s, c, slot;
	if (!block_locate(h, p, s, c, slot)) {
		set_err(h, KMA_ERR_BADFREE);
		return;
	}
	unsigned char *sb = sb_addr(h, s);
	uint32_t bit = 1u << (slot & 31);
	uint32_t *wp = bitmap_word(h, sb, slot >> 5);
	/* kma.cl:336-338 leaves the bitmap word as it was before the clear in
	 * word 0 of the block, but stores it after the clear: by then another
	 * thread may already own the slot and have written that word.  Store
	 * the same value first, then clear the bit with release semantics. */
	uint32_t cur = ld_relaxed(wp);
	if (!(cur & bit)) {
		/* double free: the reference increments the free count anyway
		 * and corrupts the superblock (kma.cl:333-335); refuse it */
		set_err(h, KMA_ERR_BADFREE);
		return;
	}
	*reinterpret_cast<volatile uint32_t *>(p) = cur;
	uint32_t old = bm_and_release(wp, ~bit);
	if (!(old & bit)) {
		set_err(h, KMA_ERR_BADFREE); /* a concurrent double free */
		return;
	}
	uint32_t *stp = &h->sb_state[s];
	uint32_t lim = h->spin_limit;
	for (uint32_t it = 0; it < lim; it++) {
		uint32_t st = atomicAdd(stp, 0u); /* kma.cl:343 */
		uint32_t slots = st_slots(st);
		uint32_t fr = st_free(st) + 1;
		bool enq = fr == slots;
		uint32_t nst = st_make(st_class(st), slots, enq ? 0 : fr);
		if (cas_relaxed(stp, st, nst) == st) {
			if (enq)
				sb_recycle(h, s, c);
			return;
		}
	}
	set_err(h, KMA_ERR_TIMEOUT | KMA_ERR_AT_FREE);
}

/* ------------------------------------------------------------------ */
/* warp-collaborative malloc/free                                      */
/* ------------------------------------------------------------------ */
/* Lanes are grouped by size class with __match_any_sync.  The group   */
/* leader reserves k slots with one CAS on the current superblock's     */
/* state word (refilling from the free list when needed; a group that   */
/* needs a whole superblock takes a fresh one without touching the      */
/* class table), then claims the bitmap bits one word at a time with    */
/* one atomicOr per word; the claimed (superblock, word, mask) is       */
/* broadcast with __shfl_sync and each lane picks its bit by rank.  One */
/* atomic per warp per superblock (and per bitmap word) reaches L2      */
/* instead of two or three per lane.  A single calling lane follows     */
/* exactly the plain path's choices.                                    */
/* ------------------------------------------------------------------ */
namespace kma_detail {

} /* namespace kma_detail */

/* Optional event counts of the warp-collaborative calls (diagnostics):
 * pass a pointer to a per-thread tally to kma_malloc_warp/kma_free_warp;
 * with the default null pointer the counting compiles away. */
struct kma_tally {
	uint32_t n[8];
};
#define KMA_T_ITER 0      /* leader turns in kma_malloc_warp */
#define KMA_T_TRY 1       /* reservation attempts */
#define KMA_T_POISON 2    /* waits on a refill in progress */
#define KMA_T_STALE 3     /* class slot pointing at a full or stale superblock */
#define KMA_T_CASFAIL 4   /* lost reservation CASes */
#define KMA_T_REFILL 5    /* superblocks taken from the free list */
#define KMA_T_CLAIM 6     /* bitmap claim steps */
#define KMA_T_EMPTY 7     /* claim steps that got no bit */

namespace kma_detail {

__device__ __forceinline__ void tally(kma_tally *t, int k)
{
	if (t)
		t->n[k]++;
}

/* Leader-side state of one group's reservation.  kword/known: the last
 * bitmap word this reservation touched and its value as the atomicOr
 * returned it (claims go blind on a word first: setting a bit that is
 * already set changes nothing, and the returned word says what is free). */
struct warp_resv {
	uint32_t sb, cls, left, cursor, pre_hi, hint, kword, known;
	bool pre;
};

/* Reserve up to `want` slots of class c.  On success fills r (sb, left =
 * number reserved, cursor = first slot to scan from, hint) and returns 1;
 * returns 0 when the heap is exhausted or a spin expired. */
__device__ __forceinline__ int warp_reserve(kma_heap *h, uint32_t c, uint32_t want, warp_resv &r,
		kma_tally *tl, uint32_t *hint)
{
	uint32_t slots = h->cls_slots[c];
	uint32_t shard = my_shard(h, c);
	if (want >= slots && slots > 1) {
		/* the group fills a whole superblock: take a fresh one privately
		 * (it would be detached at once anyway) */
		tally(tl, KMA_T_REFILL);
		int64_t s = sb_dequeue(h);
		if (s < 0)
			return 0;
		sb_format(h, (uint32_t)s, c, 0, 0, shard);
		r.sb = (uint32_t)s;
		r.cls = c;
		r.left = slots;
		r.cursor = 0;
		r.pre_hi = slots;
		r.hint = slots - 1;
		r.pre = true;
		r.kword = 0xffffffffu;
		return 1;
	}
	uint32_t *clsw = cls_word(h, c, shard);
	uint32_t lim = h->spin_limit;
	/* the superblock this warp last reserved from in class c: its state is
	 * loaded together with the class word, and used when the class word
	 * still names it (saving the dependent load) */
	uint32_t guess = hint ? hint[c] : 0u;
	for (uint32_t it = 0; it < lim; it++) {
		tally(tl, KMA_T_TRY);
		uint32_t cur = ld_relaxed(clsw);
		uint32_t st_guess = guess ? ld_relaxed(&h->sb_state[guess - KMA_CLS_BASE]) : 0u;
		const bool poisoned = cur == KMA_POISON;
		if (cur == 0 || (poisoned && slots <= KMA_PRIVATE_REFILL_SLOTS)) {
			/* cur == 0: the reference's refill under POISON (kma.cl:166-195).
			 * POISON on a class with few slots per superblock: the refill in
			 * flight yields about one group's worth, so rather than queue
			 * behind it take a fresh superblock without holding the class
			 * slot, and publish the leftover slots only if the slot is empty
			 * by then.  Serial execution never observes POISON. */
			bool locked = false;
			if (!poisoned) {
				if (cas_relaxed(clsw, 0, KMA_POISON) != 0)
					continue;
				locked = true;
			}
			tally(tl, KMA_T_REFILL);
			int64_t s = sb_dequeue(h);
			if (s < 0) {
				if (locked)
					atomicExch(clsw, 0);
				return 0;
			}
			uint32_t t = want < slots ? want : slots;
			sb_format(h, (uint32_t)s, c, slots - t, slots - t, shard);
			/* the refiller takes the top t slots, which are exactly the
			 * hints slots-1 .. slots-t of t serial reservations */
			uint32_t pub = t == slots ? 0u : (uint32_t)s + KMA_CLS_BASE;
			/* release: a thread that finds s in the slot must find
			 * its formatted state (a stale one would read as full and
			 * get s detached with free slots nobody can reach) */
			if (locked)
				cas_release(clsw, KMA_POISON, pub);
			else if (pub)
				cas_release(clsw, 0, pub);
			if (hint && pub)
				hint[c] = pub;
			r.sb = (uint32_t)s;
			r.cls = c;
			r.left = t;
			r.cursor = slots - t;
			r.pre_hi = slots;
			r.hint = slots - 1;
			r.pre = true;
			r.kword = 0xffffffffu;
			return 1;
		}
		if (poisoned) {
			tally(tl, KMA_T_POISON);
			backoff(it);
			continue;
		}
		uint32_t s = cur - KMA_CLS_BASE;
		uint32_t *stp = &h->sb_state[s];
		const bool speculated = cur == guess;
		uint32_t st = speculated ? st_guess : ld_relaxed(stp);
		guess = cur;
		if (st_class(st) != c || st_free(st) == 0) {
			tally(tl, KMA_T_STALE);
			/* the speculative state load may be older than cur */
			if (speculated)
				st = ld_relaxed(stp);
			if (st_class(st) != c || st_free(st) == 0)
				clear_stale(clsw, cur);
			continue;
		}
		uint32_t fr = st_free(st);
		uint32_t t = want < fr ? want : fr;
		/* the first bitmap word the claim will visit is known already:
		 * load it alongside the CAS instead of after it */
		uint32_t k0 = (fr - t) >> 5;
		uint32_t spec = ld_relaxed(bitmap_word(h, sb_addr(h, s), k0));
		if (cas_relaxed(stp, st, st - t) != st) {
			tally(tl, KMA_T_CASFAIL);
			continue;
		}
		if (fr == t)
			cas_relaxed(clsw, cur, 0);
		if (hint)
			hint[c] = cur;
		r.sb = s;
		r.cls = c;
		r.left = t;
		r.cursor = fr - t; /* lowest of the t serial hints fr-1 .. fr-t */
		r.pre = false;
		r.kword = k0;
		r.known = spec;
		r.hint = fr - 1;
		return 1;
	}
	set_err(h, KMA_ERR_TIMEOUT | KMA_ERR_AT_RESERVE);
	return 0;
}

/* One claim step on the reservation: claims bits in one bitmap word.
 * Returns the claimed mask (possibly 0 when another thread won the bits
 * and the word must be re-read), and the word index in `word`. */
__device__ __forceinline__ uint32_t warp_claim_step(kma_heap *h, warp_resv &r, uint32_t &word)
{
	uint32_t slots = h->cls_slots[r.cls];
	uint32_t k = r.cursor >> 5;
	word = k;
	uint32_t lo = r.cursor & 31;
	if (r.pre) {
		/* bits [cursor, pre_hi) were set by sb_format */
		uint32_t hi = r.pre_hi < (k + 1) * 32 ? r.pre_hi - k * 32 : 32;
		uint32_t n = hi - lo;
		uint32_t got = (n == 32 ? 0xffffffffu : ((1u << n) - 1u)) << lo;
		r.cursor = k * 32 + hi;
		r.left -= n;
		return got;
	}
	unsigned char *sb = sb_addr(h, r.sb);
	uint32_t *wp = bitmap_word(h, sb, k);
	uint32_t words = h->cls_words[r.cls];
	uint32_t valid = (k == words - 1 && (slots & 31)) ? ((1u << (slots & 31)) - 1u) : 0xffffffffu;
	/* first visit of a word: assume its bits are clear; the atomicOr's
	 * result then says which ones really were */
	uint32_t v = r.kword == k ? r.known : 0u;
	uint32_t cand = ~v & valid & (0xffffffffu << lo);
	uint32_t pick = 0;
	/* take the lowest `left` candidate bits */
	if (__popc(cand) <= (int)r.left) {
		pick = cand;
	} else {
		uint32_t top = nth_set_bit(cand, r.left - 1);
		pick = cand & (top == 31 ? 0xffffffffu : ((2u << top) - 1u));
	}
	uint32_t got = 0;
	if (pick) {
		uint32_t old = bm_or(wp, pick);
		got = pick & ~old;
		r.kword = k;
		r.known = old | pick;
	}
	r.left -= __popc(got);
	if (got == pick) {
		/* every candidate we wanted is ours: move on if more are needed */
		if (r.left && __popc(cand) <= __popc(pick)) {
			r.cursor = (k + 1) * 32;
			if (r.cursor >= slots)
				r.cursor = 0;
			/* what is known of this word may predate the reservation
			 * (the speculative load): the next visit, possibly of this
			 * same word after a wrap, claims afresh.  An atomicOr's
			 * result always shows at least `left` clear bits, which
			 * is what guarantees progress. */
			r.kword = 0xffffffffu;
		}
	}
	return got;
}

} /* namespace kma_detail */

/* hint (optional): this warp's KMA_MAX_CLASSES words, zeroed once, best
 * in shared memory; the warp's leaders remember there, per class, the
 * superblock they last reserved from, and load its state together with
 * the class word on the next call.  Only a speed hint: any content is
 * safe, a stale one costs the dependent load it would have saved. */
__device__ inline void *kma_malloc_warp(kma_heap *h, size_t size, kma_tally *tl = nullptr,
		uint32_t *hint = nullptr)
{
	using namespace kma_detail;
	const uint32_t active = __activemask();
	const uint32_t lane = lane_id();
	int c = kma_class_of(h, size);
	uint32_t peers = __match_any_sync(active, c);
	uint32_t leader = __ffs(peers) - 1;
	uint32_t rank = __popc(peers & lanemask_lt());
	uint32_t gsize = __popc(peers);
	bool need = c >= 0;
	void *res = NULL;

	/* leader-only state: the leader serves its whole group, not only itself */
	warp_resv r;
	r.left = 0;
	uint32_t served = 0;
	bool failed = false;
	const uint32_t lim = h->spin_limit;
	uint32_t rounds = 0;

	while (__any_sync(active, need)) {
		/* every lane runs every iteration, so this bound ends the loop for
		 * all of them together */
		if (++rounds > lim) {
			if (need) {
				need = false;
				set_err(h, KMA_ERR_TIMEOUT | KMA_ERR_AT_WARP);
			}
			continue;
		}
		uint32_t bsb = 0, bword = 0, bgot = 0, bbase = 0, bhint = 0, bfail = 0;
		if (lane == leader && c >= 0 && served < gsize && !failed) {
			tally(tl, KMA_T_ITER);
			if (r.left == 0) {
				if (!warp_reserve(h, (uint32_t)c, gsize - served, r, tl, hint))
					failed = true;
			}
			if (!failed) {
				uint32_t w;
				uint32_t hint0 = r.hint;
				uint32_t got = warp_claim_step(h, r, w);
				tally(tl, KMA_T_CLAIM);
				if (!got)
					tally(tl, KMA_T_EMPTY);
				bsb = r.sb;
				bword = w;
				bgot = got;
				bbase = served;
				bhint = hint0;
				served += __popc(got);
				r.hint -= __popc(got);
			}
			bfail = failed;
		}
		bsb = __shfl_sync(active, bsb, leader);
		bword = __shfl_sync(active, bword, leader);
		bgot = __shfl_sync(active, bgot, leader);
		bbase = __shfl_sync(active, bbase, leader);
		bhint = __shfl_sync(active, bhint, leader);
		bfail = __shfl_sync(active, bfail, leader);
		if (need) {
			uint32_t n = __popc(bgot);
			if (rank >= bbase && rank < bbase + n) {
				/* rank j of this claim takes the j-th highest claimed bit,
				 * matching the serial hint order fr-1, fr-2, ... */
				uint32_t j = rank - bbase;
				uint32_t b = nth_set_bit(bgot, n - 1 - j);
				uint32_t slot = bword * 32 + b;
				unsigned char *p = sb_addr(h, bsb) + KMA_SB_HDR + (size_t)slot * h->cls_size[c];
				*reinterpret_cast<uint32_t *>(p) = bhint - j;
				res = p;
				need = false;
			} else if (bfail) {
				need = false;
			}
		}
	}
	return res;
}

__device__ inline void kma_free_warp(kma_heap *h, void *p)
{
	using namespace kma_detail;
	const uint32_t active = __activemask();
	const uint32_t lane = lane_id();
	uint32_t s = 0xffffffffu, c = 0, slot = 0;
	bool valid = false;
	if (p != NULL) {
		valid = block_locate(h, p, s, c, slot);
		if (!valid)
			set_err(h, KMA_ERR_BADFREE);
	}
	/* 1) clear bitmap bits: one atomicAnd per (superblock, word) */
	uint32_t word = valid ? (slot >> 5) : 0xffffffffu;
	unsigned long long key = ((unsigned long long)s << 32) | word;
	uint32_t wpeers = __match_any_sync(active, key);
	uint32_t bit = valid ? (1u << (slot & 31)) : 0u;
	uint32_t mask = __reduce_or_sync(wpeers, bit);
	uint32_t wleader = __ffs(wpeers) - 1;
	uint32_t *wp = valid ? bitmap_word(h, sb_addr(h, s), word) : NULL;
	uint32_t old = 0;
	if (__popc(__ballot_sync(active, valid)) == 1) {
		/* one block: the reference's side effect, the bitmap word as it
		 * was before the clear, in word 0 of the block (kma.cl:338) --
		 * stored before the release, as in kma_free.  Every call of a
		 * one-thread-at-a-time execution takes this path. */
		if (valid) {
			uint32_t cur = ld_relaxed(wp);
			if (cur & bit) {
				*reinterpret_cast<volatile uint32_t *>(p) = cur;
				old = bm_and_release(wp, ~mask);
			} else {
				old = cur;
			}
		}
	} else if (valid && lane == wleader) {
		/* several blocks at once: freed memory has no defined contents,
		 * so the residue (a load, a store and a fence) is skipped */
		old = bm_and(wp, ~mask);
	}
	old = __shfl_sync(active, old, wleader);
	bool good = valid && (old & bit);
	if (valid && !good)
		set_err(h, KMA_ERR_BADFREE); /* double free, see kma_free */
	/* 2) return k slots to the superblock: one fetch-and-add per
	 * superblock, after the bits are clear (a count that reaches `slots`
	 * lets the superblock be recycled and reformatted) */
	uint32_t speers = __match_any_sync(active, good ? s : 0xffffffffu);
	uint32_t k = __popc(speers);
	uint32_t sleader = __ffs(speers) - 1;
	if (good && lane == sleader) {
		uint32_t *stp = &h->sb_state[s];
		uint32_t prev = atomicAdd(stp, k);
		uint32_t slots = st_slots(prev);
		if (st_free(prev) + k == slots) {
			/* kma.cl:350-367: all free -- free count 0 and recycle, unless
			 * a reservation got in first */
			uint32_t full = prev + k;
			if (cas_relaxed(stp, full, st_make(st_class(prev), slots, 0)) == full)
				sb_recycle(h, s, c);
		}
	}
}

#endif /* KMA_DEVICE_CUH */
