/*
 * kma_structs.cuh -- the lock-free device structures that sit around the
 * KMA heap, and the PMA bump heap (sm_100a, header-only device code).
 *
 *   kma_clqueue      intrusive pointer FIFO        (clQueue.cl:27-118)
 *   kma_iqueue       indexed FIFO over an item array (clIndexedQueue.cl:44-290)
 *   kma_cltree       unique-key binary tree        (clTree.cl:27-74)
 *   kma_clarraylist  page-chained array list       (clArrayList.cl:23-216)
 *   kma_pma          bump heap, free is a no-op    (pma.cl:24-48)
 *
 * One-thread-at-a-time execution gives the reference's results for every
 * structure (the tests replay op streams against the reference built from
 * its own sources).  Under concurrency each structure is safe where the
 * reference is not; the differences are listed at each structure.
 *
 * Every spin is bounded by a spin limit (the reference bounds its queue
 * loops at 2^20 iterations on NVIDIA, clQueue.h:73-78); on expiry an
 * operation fails (0 / NULL) and, when the caller passes an error word,
 * ORs KMA_ERR_TIMEOUT into it.  Nothing traps.
 */
#ifndef KMA_STRUCTS_CUH
#define KMA_STRUCTS_CUH

#include "kma_device.cuh"

#define KMA_STRUCT_SPIN (1u << 20)

namespace kma_detail {

__device__ __forceinline__ unsigned long long cas64_relaxed(unsigned long long *p,
		unsigned long long cmp, unsigned long long val)
{
	unsigned long long old;
	asm volatile("atom.relaxed.gpu.global.cas.b64 %0, [%1], %2, %3;"
		     : "=l"(old) : "l"(p), "l"(cmp), "l"(val) : "memory");
	return old;
}
__device__ __forceinline__ unsigned long long xchg64_acqrel(unsigned long long *p, unsigned long long v)
{
	unsigned long long old;
	asm volatile("atom.acq_rel.gpu.global.exch.b64 %0, [%1], %2;"
		     : "=l"(old) : "l"(p), "l"(v) : "memory");
	return old;
}
/* 16-byte compare-and-swap of two adjacent 64-bit words (sm_90+).
 * Returns true when {lo, hi} held {cmp_lo, cmp_hi} and now holds the new
 * pair; p must be 16-byte aligned. */
__device__ __forceinline__ bool cas128_acqrel(unsigned long long *p, unsigned long long cmp_lo,
		unsigned long long cmp_hi, unsigned long long val_lo, unsigned long long val_hi)
{
	unsigned long long o_lo, o_hi;
	asm volatile("{\n\t"
		     ".reg .b128 d, c, v;\n\t"
		     "mov.b128 c, {%2, %3};\n\t"
		     "mov.b128 v, {%4, %5};\n\t"
		     "atom.acq_rel.gpu.global.cas.b128 d, [%6], c, v;\n\t"
		     "mov.b128 {%0, %1}, d;\n\t"
		     "}"
		     : "=l"(o_lo), "=l"(o_hi)
		     : "l"(cmp_lo), "l"(cmp_hi), "l"(val_lo), "l"(val_hi), "l"(p)
		     : "memory");
	return o_lo == cmp_lo && o_hi == cmp_hi;
}
/* Exclusive prefix and total of v over the calling lanes (any subset of
 * the warp), in lane order. */
__device__ __forceinline__ unsigned long long active_excl_sum(uint32_t active, uint32_t lane,
		unsigned long long v, unsigned long long &total)
{
	unsigned long long excl = 0, tot = 0;
	for (uint32_t m = active; m; m &= m - 1) {
		uint32_t src = __ffs(m) - 1;
		unsigned long long x = __shfl_sync(active, v, src);
		if (src < lane)
			excl += x;
		tot += x;
	}
	total = tot;
	return excl;
}
__device__ __forceinline__ void flag_err(uint32_t *err, uint32_t e)
{
	if (err)
		atomicOr(err, e);
}
/* linear id of the calling thread in the grid */
__device__ __forceinline__ unsigned long long global_thread()
{
	unsigned long long blk = ((unsigned long long)blockIdx.z * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x;
	uint32_t tpb = blockDim.x * blockDim.y * blockDim.z;
	uint32_t t = (threadIdx.z * blockDim.y + threadIdx.y) * blockDim.x + threadIdx.x;
	return blk * tpb + t;
}

} /* namespace kma_detail */

/* ================================================================== */
/* kma_clqueue: intrusive pointer FIFO (clQueue.cl:27-118)             */
/* ================================================================== */
/*
 * Same contract as the reference: an item's first 8 bytes are its link
 * (`next`), enqueue(q, item) appends the item itself, dequeue(q) returns
 * the oldest item or NULL when empty, head/tail are NULL when empty, and
 * the list can be walked from head through the links (clArrayList_get
 * does).  Dequeue locks the head item by swapping its link to POISON (1)
 * as the reference does (clQueue.cl:97), so a removed item keeps POISON in
 * its link until it is enqueued again.
 *
 * Different from the reference, which under concurrency can leave `tail`
 * on an item that was already dequeued (a dequeue of the last item racing
 * an enqueue behind it, clQueue.cl:60-66 vs :106-108), after which every
 * enqueue spins:
 *   - head and tail carry 16-bit tags above a 48-bit pointer, so a stale
 *     CAS on either fails (ABA);
 *   - the empty <-> one-item transitions change head and tail together
 *     with one 16-byte CAS;
 *   - a dequeue that moves head past the item tail points at moves tail
 *     on (helping), so tail never points at a removed item.
 * Items must stay queue items (type-stable memory) while any thread may
 * still hold a pointer to them, as in the reference (clQueue.cl:92-96).
 * Device pointers must be below 2^48 (the tag bits); enqueue refuses
 * others.
 */
struct __align__(16) kma_clqueue {
	unsigned long long head; /* {tag:16 | item ptr:48} */
	unsigned long long tail;
};
struct kma_clqueue_item {
	unsigned long long next; /* item ptr, 0 = end, 1 = POISON */
};

#define KMA_Q_POISON 1ull
#define KMA_PTR_BITS 48
#define KMA_PTR_MASK ((1ull << KMA_PTR_BITS) - 1ull)

namespace kma_detail {
__device__ __forceinline__ unsigned long long qp_ptr(unsigned long long w) { return w & KMA_PTR_MASK; }
__device__ __forceinline__ unsigned long long qp_next(unsigned long long w, unsigned long long ptr)
{
	return (((w >> KMA_PTR_BITS) + 1ull) << KMA_PTR_BITS) | ptr;
}
} /* namespace kma_detail */

/* clQueue_init (clQueue.cl:27-32) */
__device__ __forceinline__ void kma_clqueue_init(kma_clqueue *q)
{
	q->head = 0;
	q->tail = 0;
}

namespace kma_detail {
/* Where an item's 64-bit link lives.  Plain items: their first 8 bytes
 * (the item must be 8-byte aligned).  Blocks of a KMA heap are only 4-byte
 * aligned (12-byte superblock header, sizes multiples of 4) and PMA blocks
 * any-byte aligned, so a block that carries a link keeps it in the first
 * 8-byte aligned word of its first 15 bytes (kma_clarraylist pages). */
struct clq_link_head {
	static __device__ __forceinline__ unsigned long long *at(unsigned long long p)
	{
		return reinterpret_cast<unsigned long long *>(p);
	}
	static __device__ __forceinline__ bool ok(unsigned long long p) { return (p & 7ull) == 0; }
};
struct clq_link_aligned {
	static __device__ __forceinline__ unsigned long long *at(unsigned long long p)
	{
		return reinterpret_cast<unsigned long long *>((p + 7ull) & ~7ull);
	}
	static __device__ __forceinline__ bool ok(unsigned long long) { return true; }
};

#ifndef KMA_CONTEND_MAX_NS
#define KMA_CONTEND_MAX_NS 4096u
#endif
/* After a CAS lost to another thread on a contended word: a randomised
 * exponential wait (__nanosleep(t) sleeps somewhere in [0, 2t]), 64 ns
 * doubling per consecutive loss up to KMA_CONTEND_MAX_NS.  Retrying at
 * once floods the word's L2 slice with requests that queue ahead of the
 * winner's next step; spread out, the retries let one thread through per
 * round trip. */
__device__ __forceinline__ void contend(uint32_t &losses)
{
	uint32_t t = 64u << (losses < 10 ? losses : 10);
	__nanosleep(t < KMA_CONTEND_MAX_NS ? t : KMA_CONTEND_MAX_NS);
	losses++;
}

template <class L>
__device__ inline int clq_enqueue(kma_clqueue *q, unsigned long long it_p, uint32_t *err, uint32_t spin_limit)
{
	if (it_p == 0 || it_p == KMA_Q_POISON || (it_p & ~KMA_PTR_MASK) || !L::ok(it_p))
		return 0;
	st_release64(L::at(it_p), 0ull);
	uint32_t losses = 0;
	for (uint32_t it = 0; it < spin_limit; it++) {
		unsigned long long t = ld_acquire64(&q->tail);
		if (qp_ptr(t) == 0) {
			unsigned long long h = ld_acquire64(&q->head);
			if (qp_ptr(h) == 0 &&
			    cas128_acqrel(&q->head, h, t, qp_next(h, it_p), qp_next(t, it_p)))
				return 1;
			backoff(it);
			continue;
		}
		unsigned long long *tl = L::at(qp_ptr(t));
		unsigned long long n = ld_acquire64(tl);
		if (t != ld_acquire64(&q->tail))
			continue;
		if (n == 0) {
			if (cas64_acqrel(tl, 0ull, it_p) == 0ull) {
				cas64_acqrel(&q->tail, t, qp_next(t, it_p));
				return 1;
			}
			contend(losses);
		} else if (n == KMA_Q_POISON) {
			/* the tail item is being dequeued: it either goes (the
			 * queue empties) or its link comes back */
			backoff(it);
		} else {
			cas64_acqrel(&q->tail, t, qp_next(t, n)); /* help the lagging tail */
		}
	}
	flag_err(err, KMA_ERR_TIMEOUT);
	return 0;
}

template <class L>
__device__ inline unsigned long long clq_dequeue(kma_clqueue *q, uint32_t *err, uint32_t spin_limit)
{
	for (uint32_t it = 0; it < spin_limit; it++) {
		unsigned long long h = ld_acquire64(&q->head);
		unsigned long long hp = qp_ptr(h);
		if (hp == 0)
			return 0;
		unsigned long long *hl = L::at(hp);
		unsigned long long nx = xchg64_acqrel(hl, KMA_Q_POISON);
		if (nx == KMA_Q_POISON) {
			/* another dequeuer holds it, or it was removed already */
			backoff(it);
			continue;
		}
		if (nx != 0) {
			if (cas64_acqrel(&q->head, h, qp_next(h, nx)) == h) {
				unsigned long long t = ld_acquire64(&q->tail);
				if (qp_ptr(t) == hp)
					cas64_acqrel(&q->tail, t, qp_next(t, nx));
				return hp;
			}
		} else {
			/* the last item: head and tail go to NULL together, which
			 * fails if tail has not reached it yet */
			unsigned long long t = ld_acquire64(&q->tail);
			if (qp_ptr(t) == hp && cas128_acqrel(&q->head, h, t, qp_next(h, 0), qp_next(t, 0)))
				return hp;
		}
		/* stale head: put the link back (clQueue.cl:113) */
		cas64_acqrel(hl, KMA_Q_POISON, nx);
		backoff(it);
	}
	flag_err(err, KMA_ERR_TIMEOUT);
	return 0;
}

template <class L>
__device__ __forceinline__ unsigned long long clq_next(unsigned long long p)
{
	unsigned long long n = *(const volatile unsigned long long *)L::at(p);
	return n == KMA_Q_POISON ? 0ull : n;
}
} /* namespace kma_detail */

/* enqueue (clQueue.cl:40-75): 1 on success, 0 on a NULL, misaligned or
 * unaddressable item, or on spin-limit expiry (which also flags *err). */
__device__ __forceinline__ int kma_clqueue_enqueue(kma_clqueue *q, kma_clqueue_item *item,
		uint32_t *err = nullptr, uint32_t spin_limit = KMA_STRUCT_SPIN)
{
	return kma_detail::clq_enqueue<kma_detail::clq_link_head>(q, (unsigned long long)item, err, spin_limit);
}

/* dequeue (clQueue.cl:82-118): the oldest item, NULL when empty or on
 * spin-limit expiry (which also flags *err). */
__device__ __forceinline__ kma_clqueue_item *kma_clqueue_dequeue(kma_clqueue *q, uint32_t *err = nullptr,
		uint32_t spin_limit = KMA_STRUCT_SPIN)
{
	return reinterpret_cast<kma_clqueue_item *>(
		kma_detail::clq_dequeue<kma_detail::clq_link_head>(q, err, spin_limit));
}

/* The first item (NULL when empty), for walks from the head. */
__device__ __forceinline__ kma_clqueue_item *kma_clqueue_first(const kma_clqueue *q)
{
	return reinterpret_cast<kma_clqueue_item *>(
		kma_detail::qp_ptr(*(const volatile unsigned long long *)&q->head));
}
/* The item after `it` in a walk (NULL at the end or on a removed item). */
__device__ __forceinline__ kma_clqueue_item *kma_clqueue_next(const kma_clqueue_item *it)
{
	return reinterpret_cast<kma_clqueue_item *>(
		kma_detail::clq_next<kma_detail::clq_link_head>((unsigned long long)it));
}

/* ================================================================== */
/* kma_iqueue: indexed FIFO (clIndexedQueue.cl:44-290)                 */
/* ================================================================== */
/*
 * Items are addressed by index: item i (1-based) at base + (i-1) << stride.
 * An item's first 8 bytes are its link, a {tag:32 | index:32} word (the
 * reference packs {tag:10 | index:16 | poison:1} into 32 bits,
 * clIndexedQueue.cl:90-92, so it holds at most 65 535 items and wraps its
 * tag every 1024 updates).  Head and tail are tagged the same way, each on
 * its own 128-byte line, and every update increments the tag, so no CAS
 * succeeds on a recycled value.  The algorithm is the Michael-Scott queue
 * with a dummy item, as the reference's: init makes `first` the dummy,
 * dequeue returns the OLD dummy (so `first` comes out first and the last
 * item enqueued always stays behind), NULL when only the dummy is left.
 *
 * Shards (B200 addition, default 1): `nshards` independent queues over
 * the same item array, chosen by global thread id % nshards, so a
 * full-GPU producer/consumer does not serialise on one head.  FIFO order
 * holds per shard; one thread alone always uses shard 0, which is the
 * reference's queue.  Shard k > 0 starts on an internal dummy (index
 * capacity + k) that dequeue consumes silently.
 */
#define KMA_IQ_MAX_SHARDS 4096

struct __align__(128) kma_iqueue {
	unsigned char *base;
	unsigned long long *dummies; /* link words of the internal dummies [nshards-1], then the nil word */
	kma_line64 *ends;            /* shard k: head at ends[2k], tail at ends[2k+1] */
	uint32_t stride_l2;
	uint32_t capacity;   /* user items are 1..capacity */
	uint32_t nshards;
	uint32_t spin_limit;
	uint32_t err;
};

namespace kma_detail {
__device__ __forceinline__ unsigned long long *iq_link(const kma_iqueue *q, uint32_t idx)
{
	/* index 0 (no item) has no link: a read of it sees the nil word (0),
	 * so no state can address outside the item array */
	if (idx == 0)
		return &q->dummies[q->nshards - 1];
	if (idx > q->capacity)
		return &q->dummies[idx - q->capacity - 1];
	return reinterpret_cast<unsigned long long *>(q->base + ((size_t)(idx - 1) << q->stride_l2));
}
/* clIndexedQueue_ptr2idx (clIndexedQueue.cl:44-71): 0 when p is not an
 * item of the array */
__device__ __forceinline__ uint32_t iq_idx(const kma_iqueue *q, const void *p)
{
	unsigned long long a = (unsigned long long)p, b = (unsigned long long)q->base;
	if (a < b)
		return 0;
	unsigned long long d = a - b;
	if (d & ((1ull << q->stride_l2) - 1ull))
		return 0;
	d >>= q->stride_l2;
	if (d >= q->capacity)
		return 0;
	return (uint32_t)d + 1;
}
__device__ __forceinline__ uint32_t iq_shard(const kma_iqueue *q)
{
	return q->nshards > 1 ? (uint32_t)(global_thread() % q->nshards) : 0u;
}
} /* namespace kma_detail */

/* Item pointer of index idx (1-based), NULL for 0. */
__device__ __forceinline__ void *kma_iqueue_item(const kma_iqueue *q, uint32_t idx)
{
	if (idx == 0 || idx > q->capacity)
		return nullptr;
	return q->base + ((size_t)(idx - 1) << q->stride_l2);
}

/* idxd_enqueue (clIndexedQueue.cl:132-196) on the caller's shard: 1 on
 * success, 0 for an item outside the array or on spin-limit expiry. */
__device__ inline int kma_iqueue_enqueue_shard(kma_iqueue *q, void *item, uint32_t shard)
{
	using namespace kma_detail;
	uint32_t idx = iq_idx(q, item);
	if (idx == 0)
		return 0;
	unsigned long long *link = iq_link(q, idx);
	unsigned long long old = *((volatile unsigned long long *)link);
	st_release64(link, tw_make(tw_tag(old) + 1, 0));
	unsigned long long *tailw = &q->ends[2 * shard + 1].v;
	uint32_t lim = q->spin_limit;
	for (uint32_t it = 0; it < lim; it++) {
		unsigned long long t = ld_acquire64(tailw);
		unsigned long long *tl = iq_link(q, tw_idx(t));
		unsigned long long n = ld_acquire64(tl);
		if (t != ld_acquire64(tailw))
			continue;
		if (tw_idx(n) == 0) {
			if (cas64_acqrel(tl, n, tw_make(tw_tag(n) + 1, idx)) == n) {
				cas64_acqrel(tailw, t, tw_make(tw_tag(t) + 1, idx));
				return 1;
			}
		} else {
			cas64_acqrel(tailw, t, tw_make(tw_tag(t) + 1, tw_idx(n)));
		}
		backoff(it);
	}
	atomicOr(&q->err, KMA_ERR_TIMEOUT);
	return 0;
}

/* idxd_dequeue (clIndexedQueue.cl:203-247) on one shard: the old dummy
 * (an item pointer), NULL when only the dummy is left or on spin-limit
 * expiry. */
__device__ inline void *kma_iqueue_dequeue_shard(kma_iqueue *q, uint32_t shard)
{
	using namespace kma_detail;
	unsigned long long *headw = &q->ends[2 * shard].v;
	unsigned long long *tailw = &q->ends[2 * shard + 1].v;
	uint32_t lim = q->spin_limit;
	for (uint32_t it = 0; it < lim; it++) {
		unsigned long long hd = ld_acquire64(headw);
		unsigned long long t = ld_acquire64(tailw);
		unsigned long long n = ld_acquire64(iq_link(q, tw_idx(hd)));
		if (hd != ld_acquire64(headw))
			continue;
		if (tw_idx(hd) == tw_idx(t)) {
			if (tw_idx(n) == 0)
				return nullptr;
			cas64_acqrel(tailw, t, tw_make(tw_tag(t) + 1, tw_idx(n)));
		} else if (cas64_acqrel(headw, hd, tw_make(tw_tag(hd) + 1, tw_idx(n))) == hd) {
			uint32_t idx = tw_idx(hd);
			if (idx > q->capacity)
				continue; /* an internal dummy left the shard: take the next item */
			return kma_iqueue_item(q, idx);
		}
		backoff(it);
	}
	atomicOr(&q->err, KMA_ERR_TIMEOUT);
	return nullptr;
}

__device__ __forceinline__ int kma_iqueue_enqueue(kma_iqueue *q, void *item)
{
	return kma_iqueue_enqueue_shard(q, item, kma_detail::iq_shard(q));
}
__device__ __forceinline__ void *kma_iqueue_dequeue(kma_iqueue *q)
{
	return kma_iqueue_dequeue_shard(q, kma_detail::iq_shard(q));
}

/* ================================================================== */
/* kma_cltree: unique-key binary search tree (clTree.cl:27-74)         */
/* ================================================================== */
/*
 * Node layout as the reference's 64-bit node (clTree.h:24-28: key, left,
 * right, 24 bytes); the 4 bytes of padding after the key hold a state word
 * used by remove, which the reference does not have.  Remove is logical:
 * it marks the node removed (get skips it, add of the same key revives it),
 * so a concurrent get never follows a link into freed memory.
 */
struct kma_cltree_node {
	uint32_t key;
	uint32_t state; /* 0 live, 1 removed */
	unsigned long long left;
	unsigned long long right;
};
struct kma_cltree {
	unsigned long long root;
};

#define KMA_TREE_EXISTS 0
#define KMA_TREE_INSERTED 1
#define KMA_TREE_REVIVED 2

/* clTree_add (clTree.cl:27-53): KMA_TREE_INSERTED when `node` (its key set
 * by the caller) was linked; KMA_TREE_EXISTS when a live node has the key;
 * KMA_TREE_REVIVED when a removed node with the key was made live again
 * (`node` is not linked).  The reference returns 1 / 0 for the first two. */
__device__ inline int kma_cltree_add(kma_cltree *tree, kma_cltree_node *node)
{
	using namespace kma_detail;
	node->left = 0;
	node->right = 0;
	node->state = 0;
	unsigned long long np = (unsigned long long)node;
	unsigned long long *cursor = &tree->root;
	__threadfence();
	for (;;) {
		unsigned long long cur = cas64_acqrel(cursor, 0ull, np);
		if (cur == 0)
			return KMA_TREE_INSERTED;
		kma_cltree_node *c = reinterpret_cast<kma_cltree_node *>(cur);
		uint32_t ck = *(volatile uint32_t *)&c->key;
		if (ck == node->key) {
			if (ld_acquire(&c->state) != 0 && atomicCAS(&c->state, 1u, 0u) == 1u)
				return KMA_TREE_REVIVED;
			return KMA_TREE_EXISTS;
		}
		cursor = node->key < ck ? &c->left : &c->right;
	}
}

/* clTree_get (clTree.cl:56-74): the live node with `key`, or NULL. */
__device__ inline kma_cltree_node *kma_cltree_get(const kma_cltree *tree, uint32_t key)
{
	using namespace kma_detail;
	unsigned long long cur = ld_acquire64(const_cast<unsigned long long *>(&tree->root));
	while (cur) {
		kma_cltree_node *c = reinterpret_cast<kma_cltree_node *>(cur);
		uint32_t ck = *(volatile uint32_t *)&c->key;
		if (ck == key)
			return ld_acquire(&c->state) == 0 ? c : nullptr;
		cur = ld_acquire64(key < ck ? &c->left : &c->right);
	}
	return nullptr;
}

/* Logical remove (no reference counterpart): 1 when a live node with
 * `key` was marked removed, 0 otherwise. */
__device__ inline int kma_cltree_remove(kma_cltree *tree, uint32_t key)
{
	using namespace kma_detail;
	unsigned long long cur = ld_acquire64(&tree->root);
	while (cur) {
		kma_cltree_node *c = reinterpret_cast<kma_cltree_node *>(cur);
		uint32_t ck = *(volatile uint32_t *)&c->key;
		if (ck == key)
			return atomicCAS(&c->state, 0u, 1u) == 0u;
		cur = ld_acquire64(key < ck ? &c->left : &c->right);
	}
	return 0;
}

/* ================================================================== */
/* kma_pma: bump heap (pma.cl:24-48)                                   */
/* ================================================================== */
/*
 * malloc(size) takes [head, head+size) with one fetch-and-add and returns
 * NULL when head+size exceeds `bytes`; free does nothing and head never
 * rolls back.  `bytes` keeps the reference's accounting: the data region
 * plus the reference's 24-byte header (pma.c:31-53 sizes the buffer as
 * sblocks + header, and pma.cl:36 compares against that total from the
 * data base), so the last 24 bytes past the data region are reachable; the
 * host allocates them.  The reference's head is 32 bits and wraps after
 * 4 GiB of requests (handing out memory again); here it is 64 bits.
 */
struct __align__(128) kma_pma {
	unsigned long long bytes; /* data bytes + 24 (the reference's limit) */
	unsigned char *base;
	unsigned long long pad_[14];
	kma_line64 head;
};

#define KMA_PMA_REF_HEADER 24u

__device__ __forceinline__ void *kma_pma_malloc(kma_pma *p, size_t size)
{
	unsigned long long ret = atomicAdd(&p->head.v, (unsigned long long)size);
	if (ret + size > p->bytes)
		return nullptr;
	return p->base + ret;
}
__device__ __forceinline__ void kma_pma_free(kma_pma *, void *) {}

/* Warp-aggregated malloc: one fetch-and-add per warp; lane offsets in
 * lane order.  Any subset of a warp may call it, sizes per lane. */
__device__ inline void *kma_pma_malloc_warp(kma_pma *p, size_t size)
{
	using namespace kma_detail;
	const uint32_t active = __activemask();
	const uint32_t lane = lane_id();
	unsigned long long sz = size, total;
	unsigned long long excl = active_excl_sum(active, lane, sz, total);
	uint32_t first = __ffs(active) - 1;
	unsigned long long base = 0;
	if (lane == first)
		base = atomicAdd(&p->head.v, total);
	base = __shfl_sync(active, base, first);
	unsigned long long ret = base + excl;
	if (ret + sz > p->bytes)
		return nullptr;
	return p->base + ret;
}

/* ================================================================== */
/* kma_clarraylist: page-chained array list (clArrayList.cl:23-216)    */
/* ================================================================== */
/*
 * A page is one heap block: a 24-byte header followed by `count` objects
 * of objSize bytes, so objects start at page + 24 as in the reference; the
 * pages form a kma_clqueue in growth order, and get(i) walks it.  The heap
 * is KMA or PMA, chosen per list (the reference chooses by concatenating
 * the heap's source into the program, test/tb_clArrayList.c:170-173).
 *
 * Header layout.  The reference's header is three 64-bit words {link,
 * count, taken} (clArrayList.h:58-62), but heap blocks are only 4-byte
 * (KMA) or 1-byte (PMA) aligned, so those would be misaligned 64-bit
 * accesses, which a GPU refuses (the reference only ever ran this on
 * hosts that tolerate them).  Here the link is the 8-byte aligned word at
 * align8(page) (inside bytes 0..14), the object count a 32-bit word at
 * align4(page + 15) (inside bytes 15..21); `taken`, which the reference
 * writes and never reads, is not kept.
 */
#define KMA_AL_HEAP_KMA 0u
#define KMA_AL_HEAP_PMA 1u

struct __align__(16) kma_clarraylist {
	kma_clqueue queue;
	unsigned long long obj_size;
	void *heap;         /* kma_heap* or kma_pma* */
	uint32_t heap_kind; /* KMA_AL_HEAP_* */
	uint32_t err;
};
#define KMA_AL_PAGE_HDR 24u

namespace kma_detail {
template <bool WARP>
__device__ __forceinline__ void *al_heap_malloc(kma_clarraylist *l, size_t n)
{
	if (l->heap_kind == KMA_AL_HEAP_PMA)
		return WARP ? kma_pma_malloc_warp((kma_pma *)l->heap, n) : kma_pma_malloc((kma_pma *)l->heap, n);
	return WARP ? kma_malloc_warp((kma_heap *)l->heap, n) : kma_malloc((kma_heap *)l->heap, n);
}
__device__ __forceinline__ void al_heap_free(kma_clarraylist *l, void *p)
{
	if (l->heap_kind == KMA_AL_HEAP_PMA)
		kma_pma_free((kma_pma *)l->heap, p);
	else
		kma_free((kma_heap *)l->heap, p);
}
__device__ __forceinline__ uint32_t *al_page_count(unsigned long long page)
{
	return reinterpret_cast<uint32_t *>((page + 15ull + 3ull) & ~3ull);
}
__device__ __forceinline__ void *al_page_init(kma_clarraylist *l, void *p, uint32_t objs)
{
	unsigned long long page = (unsigned long long)p;
	*al_page_count(page) = objs;
	if (!clq_enqueue<clq_link_aligned>(&l->queue, page, &l->err, KMA_STRUCT_SPIN))
		return nullptr;
	return reinterpret_cast<unsigned char *>(p) + KMA_AL_PAGE_HDR;
}
} /* namespace kma_detail */

/* clArrayList_init (clArrayList.cl:23-30) */
__device__ __forceinline__ void kma_clarraylist_init(kma_clarraylist *l, uint32_t obj_size, void *heap,
		uint32_t heap_kind)
{
	kma_clqueue_init(&l->queue);
	l->obj_size = obj_size;
	l->heap = heap;
	l->heap_kind = heap_kind;
	l->err = 0;
}

/* clArrayList_grow (clArrayList.cl:32-51): room for `objs` objects in a new
 * page, NULL when the heap is exhausted. */
__device__ inline void *kma_clarraylist_grow(kma_clarraylist *l, uint32_t objs)
{
	size_t size = (size_t)objs * l->obj_size + KMA_AL_PAGE_HDR;
	void *p = kma_detail::al_heap_malloc<false>(l, size);
	if (!p)
		return nullptr;
	return kma_detail::al_page_init(l, p, objs);
}

/* Warp form of clArrayList_grow_local (clArrayList.cl:111-176): the calling
 * lanes share one page of sum(objs) objects; lane r gets the slice after
 * the objects of the calling lanes below it.  NULL for lanes with objs 0,
 * and for every lane when the heap is exhausted.  No barrier: any subset
 * of a warp may call it. */
__device__ inline void *kma_clarraylist_grow_warp(kma_clarraylist *l, uint32_t objs)
{
	using namespace kma_detail;
	const uint32_t active = __activemask();
	const uint32_t lane = lane_id();
	unsigned long long total;
	unsigned long long excl = active_excl_sum(active, lane, objs, total);
	uint32_t first = __ffs(active) - 1;
	unsigned long long page = 0;
	if (lane == first)
		page = (unsigned long long)kma_clarraylist_grow(l, (uint32_t)total);
	page = __shfl_sync(active, page, first);
	if (!page || objs == 0)
		return nullptr;
	return reinterpret_cast<unsigned char *>(page) + excl * l->obj_size;
}

/* Block form, the reference's grow_local contract (clArrayList.cl:111-176):
 * every thread of the block calls it (it has barriers); one page of the
 * block's sum(objs) objects, thread t's slice after threads 0..t-1.
 * `smem` is 33 u64 of shared memory supplied by the caller (the
 * reference's rMem[128]). */
__device__ inline void *kma_clarraylist_grow_block(kma_clarraylist *l, uint32_t objs,
		unsigned long long *smem)
{
	using namespace kma_detail;
	const uint32_t tid = (threadIdx.z * blockDim.y + threadIdx.y) * blockDim.x + threadIdx.x;
	const uint32_t nthr = blockDim.x * blockDim.y * blockDim.z;
	const uint32_t lane = tid & 31, warp = tid >> 5, nwarps = (nthr + 31) / 32;
	/* lanes present in this warp: all, or the low ones of a partial last warp */
	const uint32_t wmask = (warp == nwarps - 1 && (nthr & 31)) ? ((1u << (nthr & 31)) - 1u) : 0xffffffffu;
	uint32_t incl = objs;
#pragma unroll
	for (int d = 1; d < 32; d <<= 1) {
		uint32_t v = __shfl_up_sync(wmask, incl, d);
		if (lane >= (uint32_t)d)
			incl += v;
	}
	__syncthreads();
	if (lane == 31 || tid == nthr - 1)
		smem[warp] = incl;
	__syncthreads();
	if (tid == 0) {
		unsigned long long run = 0;
		for (uint32_t w = 0; w < nwarps; w++) {
			unsigned long long v = smem[w];
			smem[w] = run;
			run += v;
		}
		smem[32] = (unsigned long long)kma_clarraylist_grow(l, (uint32_t)run);
	}
	__syncthreads();
	unsigned long long page = smem[32];
	unsigned long long before = smem[warp] + incl - objs;
	__syncthreads();
	if (!page || objs == 0)
		return nullptr;
	return reinterpret_cast<unsigned char *>(page) + before * l->obj_size;
}

/* Each calling lane grows its OWN list (l differs per lane) by `objs`
 * objects; the page mallocs of the warp go to the heap together
 * (kma_malloc_warp / kma_pma_malloc_warp).  Same page layout and result as
 * kma_clarraylist_grow per lane; no counterpart in the reference. */
__device__ inline void *kma_clarraylist_grow_lanes(kma_clarraylist *l, uint32_t objs)
{
	size_t size = (size_t)objs * l->obj_size + KMA_AL_PAGE_HDR;
	void *p = kma_detail::al_heap_malloc<true>(l, size);
	if (!p)
		return nullptr;
	return kma_detail::al_page_init(l, p, objs);
}

/* clArrayList_get (clArrayList.cl:178-200): object i, walking the pages in
 * growth order; NULL past the end (the reference returns an uninitialised
 * value there). */
__device__ inline void *kma_clarraylist_get(kma_clarraylist *l, unsigned long long i)
{
	using namespace kma_detail;
	unsigned long long seen = 0;
	unsigned long long page = qp_ptr(*(const volatile unsigned long long *)&l->queue.head);
	while (page) {
		unsigned long long c = *(volatile uint32_t *)al_page_count(page);
		if (seen + c > i)
			return reinterpret_cast<unsigned char *>(page) + KMA_AL_PAGE_HDR + (i - seen) * l->obj_size;
		seen += c;
		page = clq_next<clq_link_aligned>(page);
	}
	return nullptr;
}

/* clArrayList_clear (clArrayList.cl:206-216): dequeue and free every page;
 * safe to call from many threads at once while nobody uses the list. */
__device__ inline void kma_clarraylist_clear(kma_clarraylist *l)
{
	using namespace kma_detail;
	for (;;) {
		unsigned long long p = clq_dequeue<clq_link_aligned>(&l->queue, &l->err, KMA_STRUCT_SPIN);
		if (!p)
			return;
		al_heap_free(l, reinterpret_cast<void *>(p));
	}
}

/* Each calling lane clears its OWN list; the warp's page frees go to the
 * heap together (kma_free_warp).  Every lane of the warp that calls it
 * must take part until all of their lists are empty. */
__device__ inline void kma_clarraylist_clear_lanes(kma_clarraylist *l)
{
	using namespace kma_detail;
	const uint32_t active = __activemask();
	bool more = true;
	while (__any_sync(active, more)) {
		unsigned long long p = 0;
		if (more) {
			p = clq_dequeue<clq_link_aligned>(&l->queue, &l->err, KMA_STRUCT_SPIN);
			more = p != 0;
		}
		if (l->heap_kind == KMA_AL_HEAP_PMA)
			kma_pma_free((kma_pma *)l->heap, reinterpret_cast<void *>(p));
		else
			kma_free_warp((kma_heap *)l->heap, reinterpret_cast<void *>(p));
	}
}

#endif /* KMA_STRUCTS_CUH */
