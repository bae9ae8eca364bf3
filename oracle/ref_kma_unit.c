/*
 * ref_kma_unit.c -- builds the reference KMA heap (clIndexedQueue.cl +
 * kma.cl, unmodified, compiled where they lie) into a host library and
 * exports a small C API for the tests and the CPU baseline.
 *
 * TEST INFRASTRUCTURE ONLY (the oracle).  Built by oracle/Makefile into
 * oracle/_ref/libkmaref_<SB>.so.  Never linked by the product.
 *
 * Superblock size: ORACLE_SB_LOG2 = 12 uses the reference's own kma.h
 * (KMA_SB_SIZE 4096, kma.h:27-29).  Other sizes restate kma.h:27-29 and
 * the two structs of kma.h:71-85 with only the size macros changed, as the
 * reference intends them to be edited; every function still comes from
 * kma.cl / clIndexedQueue.cl unmodified.
 */
#include "ref_shim.h"

#ifndef ORACLE_SB_LOG2
#define ORACLE_SB_LOG2 12
#endif

#if ORACLE_SB_LOG2 == 12
#include "kma.h"
#else
#define KMA_H
#include "clheap.h"
#include "clIndexedQueue.h"
#define KMA_SB_SIZE (1 << ORACLE_SB_LOG2)
#define KMA_SB_SIZE_LOG2 ORACLE_SB_LOG2
#define KMA_SB_SIZE_BUCKETS KMA_SB_SIZE_LOG2 - 1
struct kma_sb {
	clIndexedQueue_item q;
	volatile unsigned int state;
	unsigned int size;
	char data[KMA_SB_SIZE - 8 - sizeof(clIndexedQueue_item)];
};
struct clheap {
	size_t bytes;
	clIndexedQueue free;
	volatile struct kma_sb __global *sb[KMA_SB_SIZE_BUCKETS];
};
#endif

#include "clIndexedQueue.cl"
#include "kma.cl"

#undef malloc
#undef free

__thread struct oref_workitem oref_wi = { 1, {0, 0, 0}, {1, 1, 1}, {0, 0, 0}, {1, 1, 1}, NULL };

struct oref_kma {
	struct clheap *heap;
	unsigned char *raw;
	size_t bytes;
	unsigned int sblocks;
};

unsigned int oref_sb_size(void) { return KMA_SB_SIZE; }
unsigned int oref_sb_log2(void) { return KMA_SB_SIZE_LOG2; }
unsigned int oref_buckets(void) { return KMA_SB_SIZE_BUCKETS; }
unsigned int oref_header_bytes(void) { return (unsigned int)sizeof(struct clheap); }

/* kma.cl:55-90 */
uint64_t oref_size_by_sbid(int sbid)
{
	/* kma.cl:61 lets sbid == BUCKETS through and divides by zero at :87;
	 * report that case as 0 instead of executing it. */
	if (sbid == KMA_SB_SIZE_BUCKETS)
		return 0;
	return _kma_size_by_sbid(sbid);
}

/* kma.cl:95-113 */
int oref_slots_by_size(uint64_t size) { return _kma_slots_by_size((size_t)size); }

/* kma.cl:119-148 (sizes 0..3 read an uninitialised sbid in the
 * reference; this library is built with -ftrivial-auto-var-init=zero so
 * they resolve to class 0) */
int oref_sbid_by_size(uint64_t size) { return _kma_sbid_by_size((size_t)size); }

/* kma.c:79-127 + kma.cl:27-52: zero-filled buffer (queue tags derive from
 * prior contents, clIndexedQueue.cl:104), header.bytes written, one
 * work-item runs clheap_init. */
void *oref_kma_create(unsigned int sblocks)
{
	struct oref_kma *k;
	size_t bytes;
	void *raw;

	if (sblocks == 0)
		return NULL;
	bytes = (size_t)sblocks * KMA_SB_SIZE + sizeof(struct clheap);
	k = calloc(1, sizeof(*k));
	if (!k)
		return NULL;
	if (posix_memalign(&raw, 4096, bytes + 4096)) {
		free(k);
		return NULL;
	}
	memset(raw, 0, bytes + 4096);
	k->raw = raw;
	k->bytes = bytes;
	k->sblocks = sblocks;
	k->heap = (struct clheap *)raw;
	k->heap->bytes = bytes;
	clheap_init(k->heap);
	return k;
}

void oref_kma_destroy(void *h)
{
	struct oref_kma *k = h;
	if (!k)
		return;
	free(k->raw);
	free(k);
}

static inline uintptr_t oref_first_sb(struct oref_kma *k)
{
	return (uintptr_t)k->heap + sizeof(struct clheap);
}

/* Offsets are relative to the first superblock; -1 is NULL. */
int64_t oref_kma_malloc(void *h, uint64_t size)
{
	struct oref_kma *k = h;
	void *p = kma_malloc(k->heap, (size_t)size);
	if (!p)
		return -1;
	return (int64_t)((uintptr_t)p - oref_first_sb(k));
}

void oref_kma_free(void *h, int64_t off)
{
	struct oref_kma *k = h;
	if (off < 0) {
		kma_free(k->heap, NULL);
		return;
	}
	kma_free(k->heap, oref_first_sb(k) + (uintptr_t)off);
}

/* Serial replay of an op stream: ops[2i] = kind, ops[2i+1] = arg.
 * kind 0: malloc(arg) -> out[i] = offset or -1
 * kind 1: free(out[arg]) (arg < 0: free(NULL)) -> out[i] = 0 */
void oref_kma_replay(void *h, const int64_t *ops, int64_t n, int64_t *out)
{
	int64_t i;
	for (i = 0; i < n; i++) {
		int64_t kind = ops[2 * i], arg = ops[2 * i + 1];
		if (kind == 0) {
			out[i] = oref_kma_malloc(h, (uint64_t)arg);
		} else {
			oref_kma_free(h, arg < 0 ? -1 : out[arg]);
			out[i] = 0;
		}
	}
}

unsigned char *oref_kma_sb_base(void *h) { return (unsigned char *)oref_first_sb(h); }
unsigned char *oref_kma_raw(void *h) { return ((struct oref_kma *)h)->raw; }

/* Decode the heap into the canonical form shared by every implementation:
 *   cls[b]       SB index attached to class b, -1 empty, -2 POISON
 *   sb_size[s], sb_slots[s], sb_free[s]   from the in-band SB header
 *   freelist[]   SB indices from head (the dummy) to tail
 * Returns the free-list length, or -1 if it does not end within
 * max_list entries (a cycle). */
int64_t oref_kma_decode(void *h, int64_t *cls, uint32_t *sb_size,
		uint32_t *sb_slots, uint32_t *sb_free, int64_t *freelist,
		int64_t max_list)
{
	struct oref_kma *k = h;
	uintptr_t first = oref_first_sb(k);
	unsigned int b, s;
	int64_t n = 0;
	uint32_t idx;

	for (b = 0; b < KMA_SB_SIZE_BUCKETS; b++) {
		uintptr_t p = (uintptr_t)k->heap->sb[b];
		if (p == 0)
			cls[b] = -1;
		else if (p == 1)
			cls[b] = -2;
		else
			cls[b] = (int64_t)((p - first) >> KMA_SB_SIZE_LOG2);
	}
	for (s = 0; s < k->sblocks; s++) {
		struct kma_sb *sb = (struct kma_sb *)(first + (uintptr_t)s * KMA_SB_SIZE);
		sb_size[s] = sb->size;
		sb_slots[s] = sb->state >> 16;
		sb_free[s] = sb->state & 0xffff;
	}
	/* the shim's free->kma_free macro also renamed the member clheap.free */
	idx = IDX(k->heap->kma_free.head);
	while (idx != 0) {
		struct kma_sb *sb;
		if (n >= max_list)
			return -1;
		freelist[n++] = idx - 1;
		sb = (struct kma_sb *)(first + ((uintptr_t)(idx - 1) << KMA_SB_SIZE_LOG2));
		idx = IDX(sb->q.next);
	}
	return n;
}

#include "workload.h"

/* Run a C1/C2 workload program over this heap.
 * which: 1 = C1, 2 = C2.  mode: 0 = serial item-major, 1 = serial
 * round-major, 2 = pthreads (threads > 0).  stats[5] receives
 * {mallocs, frees, nulls, bad_tags, offset_hash}. */
int oref_kma_run_workload(void *h, int which, uint64_t items, uint32_t rounds,
		uint64_t seed, int mode, unsigned int threads, uint64_t *stats,
		double *seconds)
{
	struct wl_heap hp = { h, oref_kma_malloc, oref_kma_free, oref_kma_sb_base(h) };
	struct wl_stats st;
	int rc;

	if (seconds)
		*seconds = 0;
	if (mode == 2)
		rc = which == 1 ? wl_run_c1_threads(&hp, items, rounds, seed, threads, &st, seconds)
				: wl_run_c2_threads(&hp, items, rounds, seed, threads, &st, seconds);
	else
		rc = which == 1 ? wl_run_c1_serial(&hp, items, rounds, seed, mode, &st)
				: wl_run_c2_serial(&hp, items, rounds, seed, mode, &st);
	stats[0] = st.mallocs;
	stats[1] = st.frees;
	stats[2] = st.nulls;
	stats[3] = st.bad_tags;
	stats[4] = st.offset_hash;
	return rc;
}
