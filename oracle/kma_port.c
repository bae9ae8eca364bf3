/*
 * kma_port.c -- CPU restatement of the reference KMA heap (the oracle for
 * heaps the reference's own format cannot express).
 *
 * TEST INFRASTRUCTURE ONLY.  Built into oracle/libkmaport.so by
 * oracle/Makefile; read by tests/ and bench.py's CPU-baseline fallback.
 *
 * Follows kma.cl:27-373 and clIndexedQueue.cl:125-290 step by step, with
 * one change: the indexed-queue word is widened from the reference's
 * {poison:1, idx:16, tag:10} u32 (clIndexedQueue.cl:170-172) to a
 * {tag:32 | idx:32} u64 kept in a side array, so heaps above 65 535
 * superblocks (and any superblock size 2^12..2^16) can be replayed.  The
 * superblock keeps the reference's in-band 12-byte header (state at +4,
 * size at +8, kma.h:71-78), its data at +12 and its bitmap at the tail.
 * Atomics are GCC __atomic builtins at the reference's atom_* sites, so
 * the threaded driver reproduces the reference's concurrency (including
 * its races); the reference's unbounded loops get an iteration bound here
 * that makes the call fail instead of hanging.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include "workload.h"

#define PORT_POISON 1u
#define PORT_SPIN (1u << 20)

struct port_heap {
	uint32_t log2, sb, buckets, sblocks, pages;
	unsigned char *region;     /* first superblock */
	uint64_t *next;            /* per-SB queue link {tag:32|idx:32} */
	uint64_t head, tail;       /* free list */
	uint64_t cls[16];          /* 0 empty, 1 POISON, s+2 */
	void *raw;
};

#define ATOMIC_CAS(p, c, v) __sync_val_compare_and_swap((p), (c), (v))
#define ATOMIC_XCHG(p, v) __atomic_exchange_n((p), (v), __ATOMIC_SEQ_CST)
#define ATOMIC_ADD(p, v) __atomic_fetch_add((p), (v), __ATOMIC_SEQ_CST)
#define ATOMIC_OR(p, v) __atomic_fetch_or((p), (v), __ATOMIC_SEQ_CST)
#define ATOMIC_AND(p, v) __atomic_fetch_and((p), (v), __ATOMIC_SEQ_CST)
#define FENCE() __atomic_thread_fence(__ATOMIC_SEQ_CST)
#define LOAD(p) __atomic_load_n((p), __ATOMIC_SEQ_CST)

static inline uint32_t tw_idx(uint64_t w) { return (uint32_t)w; }
static inline uint32_t tw_tag(uint64_t w) { return (uint32_t)(w >> 32); }
static inline uint64_t tw_make(uint32_t tag, uint32_t idx) { return ((uint64_t)tag << 32) | idx; }

static inline unsigned char *sb_ptr(struct port_heap *h, uint32_t s)
{
	return h->region + ((size_t)s << h->log2);
}
static inline uint32_t *sb_state(struct port_heap *h, uint32_t s) { return (uint32_t *)(sb_ptr(h, s) + 4); }
static inline uint32_t *sb_size(struct port_heap *h, uint32_t s) { return (uint32_t *)(sb_ptr(h, s) + 8); }

/* kma.cl:55-90 */
uint32_t oport_size_by_sbid(uint32_t log2, int block)
{
	uint64_t bytes, items, alloc_bytes, total;
	int buckets = (int)log2 - 1;
	uint64_t sb = 1ull << log2;
	if (block > buckets || block < 0)
		return 0;
	if (block == buckets) /* kma.cl:87 divides by zero for this id */
		return 0;
	block += 2;
	if (block <= (int)(log2 >> 1))
		return 1u << block;
	bytes = 1ull << block;
	items = sb / bytes;
	alloc_bytes = items >> 3;
	alloc_bytes += (items & 0x7) ? 1 : 0;
	alloc_bytes += (alloc_bytes & 0x3) ? (4 - (alloc_bytes & 0x3)) : 0;
	total = sb - (12 + alloc_bytes);
	return (uint32_t)((total / items) & ~0x3ull);
}

/* kma.cl:95-113 */
int oport_slots_by_size(uint32_t log2, uint64_t size)
{
	int64_t slots;
	uint64_t space = (1ull << log2) - 12;
	if (size == 0)
		return 0;
	slots = (int64_t)(space / size);
	if (slots & 0x1f)
		slots += 32;
	slots >>= 3;
	slots &= ~0x3;
	space -= (uint64_t)slots;
	return (int)(space / size);
}

/* kma.cl:119-148, the loop as written (sbid starts at 0 for sizes < 4,
 * which is what a zero-initialised reference build does) */
int oport_sbid_by_size(uint32_t log2, uint64_t size)
{
	int sbid = 0, i, test;
	uint64_t ssize;
	int buckets = (int)log2 - 1;
	if (size > (1ull << log2) - 16)
		return -1;
	ssize = size >> 2;
	for (i = 0; i < buckets; i++, ssize >>= 1)
		if (ssize & 1)
			sbid = i;
	for (;;) {
		test = (int)oport_size_by_sbid(log2, sbid);
		if (size > (uint64_t)test && test > 0)
			sbid++;
		else if (size < oport_size_by_sbid(log2, sbid - 1))
			sbid--;
		else
			return sbid;
	}
}

/* clIndexedQueue.cl:194-247 (idxd_enqueue) over widened words */
static int port_enqueue(struct port_heap *h, uint32_t s)
{
	uint32_t idx = s + 1, it;
	uint64_t old = LOAD(&h->next[s]);
	__atomic_store_n(&h->next[s], tw_make(tw_tag(old), 0), __ATOMIC_SEQ_CST);
	for (it = 0; it < PORT_SPIN; it++) {
		uint64_t t = LOAD(&h->tail);
		uint64_t *tl = &h->next[tw_idx(t) - 1];
		uint64_t n = LOAD(tl);
		FENCE();
		if (LOAD(&h->tail) != t)
			continue;
		if (tw_idx(n) == 0) {
			if (ATOMIC_CAS(tl, n, tw_make(tw_tag(n) + 1, idx)) == n) {
				ATOMIC_CAS(&h->tail, t, tw_make(tw_tag(t) + 1, idx));
				return 1;
			}
		} else {
			ATOMIC_CAS(&h->tail, t, tw_make(tw_tag(t) + 1, tw_idx(n)));
		}
	}
	return 0;
}

/* clIndexedQueue.cl:249-290 (idxd_dequeue): returns the old dummy or -1 */
static int64_t port_dequeue(struct port_heap *h)
{
	uint32_t it;
	for (it = 0; it < PORT_SPIN; it++) {
		uint64_t hd = LOAD(&h->head);
		uint64_t t = LOAD(&h->tail);
		uint64_t n = LOAD(&h->next[tw_idx(hd) - 1]);
		FENCE();
		if (LOAD(&h->head) != hd)
			continue;
		if (tw_idx(hd) == tw_idx(t)) {
			if (tw_idx(n) == 0)
				return -1;
			ATOMIC_CAS(&h->tail, t, tw_make(tw_tag(t) + 1, tw_idx(n)));
		} else if (ATOMIC_CAS(&h->head, hd, tw_make(tw_tag(hd) + 1, tw_idx(n))) == hd) {
			return (int64_t)tw_idx(hd) - 1;
		}
	}
	return -1;
}

/* kma.cl:27-52: class table empty, superblock 0 the dummy, 1..pages-1
 * enqueued in order */
void *oport_create(uint32_t sblocks, uint32_t log2)
{
	struct port_heap *h;
	uint32_t s;
	if (sblocks == 0 || log2 < 12 || log2 > 16)
		return NULL;
	h = calloc(1, sizeof(*h));
	if (!h)
		return NULL;
	h->log2 = log2;
	h->sb = 1u << log2;
	h->buckets = log2 - 1;
	h->sblocks = sblocks;
	h->pages = sblocks - 1;
	h->raw = calloc((size_t)sblocks << log2, 1);
	h->next = calloc(sblocks, sizeof(uint64_t));
	if (!h->raw || !h->next) {
		free(h->raw);
		free(h->next);
		free(h);
		return NULL;
	}
	h->region = h->raw;
	h->head = h->tail = tw_make(0, 1);
	for (s = 1; s < h->pages; s++)
		port_enqueue(h, s);
	return h;
}

void oport_destroy(void *p)
{
	struct port_heap *h = p;
	if (!h)
		return;
	free(h->raw);
	free(h->next);
	free(h);
}

unsigned char *oport_sb_base(void *p) { return ((struct port_heap *)p)->region; }

/* kma.cl:232-273 */
static int64_t port_get_block(struct port_heap *h, uint32_t s, uint32_t slot)
{
	uint32_t abits = 0, slots, slot_orig = slot, it;
	uint32_t *base = (uint32_t *)(sb_ptr(h, s) + h->sb); /* one past the last word */
	uint32_t *ap;
	slots = LOAD(sb_state(h, s)) >> 16;
	for (it = 0; it < PORT_SPIN; it++) {
		ap = base - (slot >> 5);
		if (slot & 0x1f)
			ap--;
		if (slot)
			abits = LOAD(ap);
		abits >>= (slot & 0x1f);
		for (; slot < slots; slot++, abits >>= 1) {
			if ((slot & 0x1f) == 0) {
				ap--;
				abits = LOAD(ap);
			}
			if ((abits & 1) == 0) {
				uint32_t bit = 1u << (slot & 0x1f);
				if ((ATOMIC_OR(ap, bit) & bit) == 0) {
					int64_t off = ((int64_t)s << h->log2) + 12 + (int64_t)slot * LOAD(sb_size(h, s));
					*(uint32_t *)(h->region + off) = slot_orig;
					return off;
				}
			}
		}
		slot = 0;
	}
	return -1;
}

/* kma.cl:150-225 */
static int64_t port_reserve(struct port_heap *h, int block, uint32_t *slot)
{
	uint32_t it;
	if (block < 0 || block >= (int)h->buckets)
		return -1;
	for (it = 0; it < PORT_SPIN; it++) {
		uint64_t cur = ATOMIC_CAS(&h->cls[block], 0, PORT_POISON);
		FENCE();
		if (cur == 0) {
			int64_t s = port_dequeue(h);
			uint32_t size, slots, i, *ap;
			if (s < 0) {
				ATOMIC_XCHG(&h->cls[block], 0);
				return -1;
			}
			size = oport_size_by_sbid(h->log2, block);
			*sb_size(h, (uint32_t)s) = size;
			slots = (uint32_t)oport_slots_by_size(h->log2, size);
			__atomic_store_n(sb_state(h, (uint32_t)s), (slots << 16) | (slots - 1), __ATOMIC_SEQ_CST);
			ap = (uint32_t *)(sb_ptr(h, (uint32_t)s) + h->sb);
			for (i = 0; i < slots; i += 32) {
				ap--;
				*ap = 0;
			}
			FENCE();
			ATOMIC_CAS(&h->cls[block], PORT_POISON, (uint64_t)s + 2);
			*slot = slots - 1;
			return s;
		}
		if (cur > PORT_POISON) {
			uint32_t s = (uint32_t)(cur - 2);
			uint32_t *stp = sb_state(h, s);
			uint32_t old = ATOMIC_ADD(stp, 0), st, nst;
			st = old & 0xffff;
			if (st == 0)
				continue;
			st--;
			*slot = st;
			nst = st | (old & 0xffff0000u);
			if (ATOMIC_CAS(stp, old, nst) != old)
				continue;
			if ((nst & 0xffff) == 0)
				ATOMIC_XCHG(&h->cls[block], 0);
			return s;
		}
	}
	return -1;
}

/* kma.cl:279-303; offsets from the first superblock, -1 = NULL */
int64_t oport_malloc(void *p, uint64_t size)
{
	struct port_heap *h = p;
	uint32_t slot;
	int block = oport_sbid_by_size(h->log2, size);
	int64_t s;
	if (block < 0)
		return -1;
	s = port_reserve(h, block, &slot);
	if (s < 0)
		return -1;
	return port_get_block(h, (uint32_t)s, slot);
}

/* kma.cl:305-373 */
void oport_free(void *p, int64_t off)
{
	struct port_heap *h = p;
	uint32_t s, size, block, slots, old, st, enq = 0, it;
	uint32_t *ap, *b;
	if (off < 0)
		return;
	s = (uint32_t)((uint64_t)off >> h->log2);
	size = LOAD(sb_size(h, s));
	block = (uint32_t)(((uint64_t)off - ((uint64_t)s << h->log2) - 12) / size);
	ap = (uint32_t *)(sb_ptr(h, s) + h->sb) - ((block >> 5) + 1);
	b = (uint32_t *)(h->region + off);
	*b = ATOMIC_AND(ap, ~(1u << (block & 0x1f)));
	for (it = 0; it < PORT_SPIN; it++) {
		FENCE();
		old = ATOMIC_ADD(sb_state(h, s), 0);
		st = old & 0xffff;
		slots = (old & 0xffff0000u) >> 16;
		st++;
		enq = st == slots;
		if (enq)
			st = 0;
		st |= slots << 16;
		if (ATOMIC_CAS(sb_state(h, s), old, st) == old)
			break;
	}
	if (enq) {
		int sbid = oport_sbid_by_size(h->log2, size);
		ATOMIC_CAS(&h->cls[sbid], (uint64_t)s + 2, 0);
		port_enqueue(h, s);
	}
}

/* same op-stream format as oref_kma_replay */
void oport_replay(void *p, const int64_t *ops, int64_t n, int64_t *out)
{
	int64_t i;
	for (i = 0; i < n; i++) {
		int64_t kind = ops[2 * i], arg = ops[2 * i + 1];
		if (kind == 0) {
			out[i] = oport_malloc(p, (uint64_t)arg);
		} else {
			oport_free(p, arg < 0 ? -1 : out[arg]);
			out[i] = 0;
		}
	}
}

/* canonical decode, same contract as oref_kma_decode */
int64_t oport_decode(void *p, int64_t *cls, uint32_t *size, uint32_t *slots, uint32_t *freec,
		int64_t *freelist, int64_t max_list)
{
	struct port_heap *h = p;
	uint32_t b, s, idx;
	int64_t n = 0;
	for (b = 0; b < h->buckets; b++)
		cls[b] = h->cls[b] == 0 ? -1 : h->cls[b] == PORT_POISON ? -2 : (int64_t)h->cls[b] - 2;
	for (s = 0; s < h->sblocks; s++) {
		uint32_t st = *sb_state(h, s);
		size[s] = *sb_size(h, s);
		slots[s] = st >> 16;
		freec[s] = st & 0xffff;
	}
	idx = tw_idx(h->head);
	while (idx != 0) {
		if (n >= max_list)
			return -1;
		freelist[n++] = idx - 1;
		idx = tw_idx(h->next[idx - 1]);
	}
	return n;
}

int oport_run_workload(void *p, int which, uint64_t items, uint32_t rounds, uint64_t seed, int mode,
		unsigned int threads, uint64_t *stats, double *seconds)
{
	struct wl_heap hp = { p, oport_malloc, oport_free, oport_sb_base(p) };
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
