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
#include "kma_queue_algo.cuh"

#define KMA_STRUCT_SPIN (1u << 20)
/* Longest back-off of a queue wait (see gpu_ops_t::pause), per call
 * style: waits of per-thread calls, and of the warp and block forms.
 * Config 3 (2^24 payloads by 2^18 threads) measured best at 4 us for
 * per-thread calls over 4096 queues (1923 vs 1622 M ops/s at 512 ns) and
 * at 512 ns for the warp and block forms on one queue (clQueue block form
 * 24.4 vs 23.8, warp form 15.0 vs 13.9 M ops/s at 4 us). */
#ifndef KMA_QUEUE_PAUSE_MAX_NS
#define KMA_QUEUE_PAUSE_MAX_NS 4096u
#endif
#ifndef KMA_QUEUE_GROUP_PAUSE_MAX_NS
#define KMA_QUEUE_GROUP_PAUSE_MAX_NS 512u
#endif

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

/* The atomics policy of the queue algorithms (kma_queue_algo.cuh) on the
 * GPU: gpu-scope acquire/release PTX; CAP is the longest back-off. */
template <uint32_t CAP>
struct gpu_ops_t {
	static __device__ __forceinline__ unsigned long long ld(unsigned long long *p) { return ld_acquire64(p); }
	static __device__ __forceinline__ unsigned long long ld_rlx(unsigned long long *p) { return ld_relaxed64(p); }
	static __device__ __forceinline__ void st(unsigned long long *p, unsigned long long v) { st_release64(p, v); }
	static __device__ __forceinline__ void st_rlx(unsigned long long *p, unsigned long long v) { st_relaxed64(p, v); }
	static __device__ __forceinline__ unsigned long long xchg(unsigned long long *p, unsigned long long v)
	{
		return xchg64_acqrel(p, v);
	}
	static __device__ __forceinline__ unsigned long long cas(unsigned long long *p, unsigned long long c,
			unsigned long long v)
	{
		return cas64_acqrel(p, c, v);
	}
	/* after `it` fruitless tries: a randomised wait (__nanosleep(t) sleeps
	 * somewhere in [0, 2t]) of 64 ns doubling per try, at most CAP, so
	 * that the waiters on one hot word do not flood its L2 slice with
	 * requests queued ahead of the holder's: with thousands of waiters one
	 * of them still looks soon after a release */
	static __device__ __forceinline__ void pause(uint32_t it)
	{
		const uint32_t t = 64u << (it < 12 ? it : 12);
		__nanosleep(t < CAP ? t : CAP);
	}
};
/* per-thread calls */
typedef gpu_ops_t<KMA_QUEUE_PAUSE_MAX_NS> gpu_ops;
/* the warp and block forms */
typedef gpu_ops_t<KMA_QUEUE_GROUP_PAUSE_MAX_NS> gpu_ops_group;

} /* namespace kma_detail */

/* ================================================================== */
/* chain log (optional, for the warp forms of both queues)             */
/* ================================================================== */
/*
 * A log of `mask + 1` records (a power of two), reused round robin.  A
 * warp that appends a chain of its items (kma_clqueue_enqueue_warp: 3 or
 * more items; kma_iqueue_enqueue_warp_shard: 2 or more) writes the items
 * into the next record and marks the chain's first link(s) with the
 * record's number; a warp dequeue that finds a marked chain at the head
 * checks the record against the queue's links with independent loads and
 * takes the chain at once instead of walking it link by link (the
 * algorithm and its checks: kma_queue_algo.cuh).  Records are only hints:
 * a stale or overwritten one fails the check and the dequeue walks.  One
 * log may serve any number of queues of one kind.  No counterpart in the
 * reference.
 */
struct kma_chain_log {
	static constexpr bool enabled = true;
	unsigned long long *rec; /* [mask + 1][32] pointers, or [mask + 1][64] u32 indices (first 32 used) */
	unsigned int *next;      /* record counter, a line of its own */
	uint32_t mask;
	uint32_t pad;

	/* a record's slot; its entries are read with ld (relaxed) */
	__device__ __forceinline__ const unsigned long long *clq_record(uint32_t recno) const
	{
		return &rec[(size_t)(recno & mask) * 32];
	}
	__device__ __forceinline__ const uint32_t *iq_record(uint32_t recno) const
	{
		return reinterpret_cast<const uint32_t *>(&rec[(size_t)(recno & mask) * 32]);
	}
	static __device__ __forceinline__ unsigned long long ld(const unsigned long long *p)
	{
		return kma_detail::ld_relaxed64(p);
	}
	static __device__ __forceinline__ uint32_t ld(const uint32_t *p) { return kma_detail::ld_relaxed(p); }
	__device__ __forceinline__ uint32_t take() { return atomicAdd(next, 1u) & kma_q::LOG_RECNO_MASK; }
	/* chains taken from their records (next[1], a count for reports) */
	__device__ __forceinline__ void taken(uint32_t) const { atomicAdd(next + 1, 1u); }
	__device__ __forceinline__ unsigned long long *clq_slot(uint32_t recno) { return &rec[(size_t)(recno & mask) * 32]; }
	__device__ __forceinline__ uint32_t *iq_slot(uint32_t recno)
	{
		return reinterpret_cast<uint32_t *>(&rec[(size_t)(recno & mask) * 32]);
	}
};

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
 * The algorithm is kma_queue_algo.cuh's (the text its host harness checks):
 *   - enqueue exchanges the tail (always succeeds, one atomic), then links
 *     the previous tail item to the new one; the reference CASes the tail
 *     item's link in a retry loop and then the tail (clQueue.cl:40-75), so
 *     on one hot queue every enqueue but one per round trip retries;
 *   - a warp's items for one queue go in as one chain, one exchange
 *     (kma_clqueue_enqueue_warp), and a warp's dequeues of one queue take
 *     consecutive items under one hold of the head (kma_clqueue_dequeue_warp);
 *   - head carries a 16-bit tag above the 48-bit pointer, so a stale CAS
 *     fails (ABA); the dequeue that empties the queue clears the tail with
 *     a CAS, so an append racing it is never lost -- the reference can
 *     leave `tail` on an already dequeued item there (clQueue.cl:60-66 vs
 *     :106-108), after which every enqueue spins.
 * Items must stay queue items (type-stable memory) while any thread may
 * still hold a pointer to them, as in the reference (clQueue.cl:92-96).
 * Device pointers must be below 2^48 (the tag bits); enqueue refuses
 * others.
 */
struct kma_clqueue {
	unsigned long long head; /* {tag:16 | item ptr:48} */
	unsigned long long tail; /* the last item's pointer, 0 when empty */
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

template <class L>
__device__ __forceinline__ bool clq_item_ok(unsigned long long it_p)
{
	return it_p != 0 && it_p != KMA_Q_POISON && !(it_p & ~KMA_PTR_MASK) && L::ok(it_p);
}

template <class L>
__device__ inline int clq_enqueue(kma_clqueue *q, unsigned long long it_p, uint32_t *err, uint32_t spin_limit)
{
	if (!clq_item_ok<L>(it_p))
		return 0;
	/* the link is published by the exchange (acq_rel) that appends it */
	st_relaxed64(L::at(it_p), 0ull);
	if (kma_q::clq_append<gpu_ops, L>(&q->head, &q->tail, it_p, it_p, spin_limit))
		return 1;
	flag_err(err, KMA_ERR_TIMEOUT);
	return 0;
}

template <class L>
__device__ inline unsigned long long clq_dequeue(kma_clqueue *q, uint32_t *err, uint32_t spin_limit)
{
	unsigned long long out = 0;
	bool timed_out = false;
	if (kma_q::clq_dequeue_n<gpu_ops, L>(&q->head, &q->tail, &out, 1, spin_limit, &timed_out,
					      (const kma_q::no_log *)nullptr))
		return out;
	if (timed_out)
		flag_err(err, KMA_ERR_TIMEOUT);
	return 0;
}

template <class L>
__device__ __forceinline__ unsigned long long clq_next(unsigned long long p)
{
	unsigned long long n = *(const volatile unsigned long long *)L::at(p);
	return n == KMA_Q_POISON ? 0ull : qp_ptr(n); /* a logged chain marks the top bits */
}

/* Lanes grouped by key: this lane's group (lanes with the same key among
 * the `active` lanes), its rank and size, the group's first and last
 * lanes, and the next lane of the group above this one (or this lane). */
struct lane_group {
	uint32_t peers, rank, size, first, last, next;
};
__device__ __forceinline__ lane_group group_by(uint32_t active, uint32_t lane, unsigned long long key)
{
	lane_group gp;
	gp.peers = __match_any_sync(active, key);
	gp.rank = __popc(gp.peers & ((1u << lane) - 1u));
	gp.size = __popc(gp.peers);
	gp.first = __ffs(gp.peers) - 1;
	gp.last = 31 - __clz(gp.peers);
	const uint32_t above = lane == 31 ? 0u : gp.peers & ~((2u << lane) - 1u);
	gp.next = above ? __ffs(above) - 1 : lane;
	return gp;
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

/* Warp form of enqueue: every calling lane appends its own item (NULL: no
 * item) to its own queue (lanes may name different queues).  The items of
 * one queue are linked in lane order and appended as one chain with one
 * exchange of its tail, so they come out in lane order, together; with a
 * chain log, chains of 3 or more items are recorded in it.  Returns what
 * kma_clqueue_enqueue would for the lane's item (1, or 0 for a refused
 * item or an expired wait).  No counterpart in the reference. */
__device__ inline int kma_clqueue_enqueue_warp(kma_clqueue *q, kma_clqueue_item *item, uint32_t *err = nullptr,
		uint32_t spin_limit = KMA_STRUCT_SPIN, kma_chain_log *log = nullptr)
{
	using namespace kma_detail;
	const uint32_t active = __activemask();
	const uint32_t lane = lane_id();
	const unsigned long long ip = (unsigned long long)item;
	const bool ok = q && clq_item_ok<clq_link_head>(ip);
	const lane_group gp = group_by(active, lane, ok ? (unsigned long long)q : ~0ull);
	const unsigned long long nip = __shfl_sync(active, ip, gp.next);
	const unsigned long long lip = __shfl_sync(active, ip, gp.last);
	/* a chain of 3 or more: its record number, taken by the first lane */
	const bool logged = ok && log && gp.size >= 3;
	uint32_t recno = 0;
	if (logged && lane == gp.first)
		recno = log->take();
	recno = __shfl_sync(active, recno, gp.first);
	if (ok) {
		unsigned long long link = gp.next != lane ? nip : 0ull;
		if (logged) {
			log->clq_slot(recno)[gp.rank] = ip;
			link |= gp.rank == 0 ? kma_q::clq_mark_first(recno, gp.size)
					     : (gp.rank == 1 ? kma_q::clq_mark_second(recno) : 0ull);
		}
		st_relaxed64(clq_link_head::at(ip), link);
		/* every lane's link and record entry is visible before the first
		 * lane's exchange publishes the chain */
		__threadfence();
	}
	__syncwarp(active);
	int r = 0;
	if (ok && lane == gp.first) {
		r = kma_q::clq_append<gpu_ops_group, clq_link_head>(&q->head, &q->tail, ip, lip, spin_limit,
								       logged ? kma_q::clq_mark_into(recno) : 0ull);
		if (!r)
			flag_err(err, KMA_ERR_TIMEOUT);
	}
	r = __shfl_sync(active, r, gp.first);
	return ok ? r : 0;
}

/* Warp form of dequeue: every calling lane takes one item from its own
 * queue (NULL q: none).  The lanes of one queue take consecutive items
 * under one hold of its head, in lane order (a logged chain at the head
 * in one step); lanes left over when the queue runs empty get NULL.  No
 * counterpart in the reference. */
__device__ inline kma_clqueue_item *kma_clqueue_dequeue_warp(kma_clqueue *q, uint32_t *err = nullptr,
		uint32_t spin_limit = KMA_STRUCT_SPIN, const kma_chain_log *log = nullptr)
{
	using namespace kma_detail;
	const uint32_t active = __activemask();
	const uint32_t lane = lane_id();
	const lane_group gp = group_by(active, lane, q ? (unsigned long long)q : ~0ull);
	unsigned long long got = 0;
	uint32_t served = 0;
	bool more = q != nullptr;
	/* one batch per turn; a group's turns end when it is served or the
	 * queue is empty */
	for (uint32_t turn = 0; __any_sync(active, more) && turn < 32; turn++) {
		unsigned long long out[32];
		uint32_t r = 0;
		if (more && lane == gp.first) {
			bool timed_out = false;
			r = kma_q::clq_dequeue_n<gpu_ops_group, clq_link_head>(&q->head, &q->tail, out, gp.size - served,
									 spin_limit, &timed_out, log);
			if (timed_out)
				flag_err(err, KMA_ERR_TIMEOUT);
		}
		r = __shfl_sync(active, r, gp.first);
		const uint32_t rmax = __reduce_max_sync(active, more ? r : 0u);
		for (uint32_t j = 0; j < rmax; j++) {
			const unsigned long long v = __shfl_sync(active, lane == gp.first && j < r ? out[j] : 0ull, gp.first);
			if (more && j < r && gp.rank == served + j)
				got = v;
		}
		if (more) {
			served += r;
			if (r == 0 || served >= gp.size)
				more = false;
		}
	}
	return reinterpret_cast<kma_clqueue_item *>(got);
}

namespace kma_detail {
/* Linear thread index of the block. */
__device__ __forceinline__ uint32_t block_tid()
{
	return threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
}
/* Block-wide numbering of the threads with `want` set: every thread of the
 * block calls it.  Returns this thread's number (warps in the order their
 * leaders arrive, lanes in order within a warp) and the count in *total;
 * *cnt is a shared word used as the counter. */
__device__ inline uint32_t block_rank(bool want, unsigned int *cnt, uint32_t *total)
{
	if (block_tid() == 0)
		*cnt = 0;
	__syncthreads();
	const uint32_t active = __activemask();
	const uint32_t b = __ballot_sync(active, want);
	const uint32_t leader = __ffs(active) - 1;
	uint32_t base = 0;
	if (lane_id() == leader && b)
		base = atomicAdd(cnt, (unsigned int)__popc(b));
	base = __shfl_sync(active, base, leader);
	__syncthreads();
	*total = *cnt;
	return base + __popc(b & lanemask_lt());
}
} /* namespace kma_detail */

/* Block form of dequeue: every thread of the block calls it, all with the
 * same q; a thread with `want` false takes nothing (NULL).  One thread
 * serves the block's requests, in turns of one hold of the head each, and
 * a hold takes several logged chains in a row, so a block takes its items
 * in a few more round trips than a warp takes its own instead of one hold
 * per warp.  smem: blockDim + 1 words of shared memory the call may use.
 * Items go to the wanting threads in the order block_rank numbers them;
 * threads left over when the queue runs empty get NULL.  No counterpart in
 * the reference. */
__device__ inline kma_clqueue_item *kma_clqueue_dequeue_block(kma_clqueue *q, bool want, unsigned long long *smem,
		uint32_t *err = nullptr, uint32_t spin_limit = KMA_STRUCT_SPIN, const kma_chain_log *log = nullptr)
{
	using namespace kma_detail;
	unsigned int *w = reinterpret_cast<unsigned int *>(smem);
	uint32_t k = 0;
	const uint32_t rank = block_rank(want && q, &w[0], &k);
	unsigned long long *out = smem + 1;
	if (block_tid() == 0) {
		uint32_t served = 0;
		for (uint32_t turn = 0; q && served < k && turn < k; turn++) {
			bool timed_out = false;
			const uint32_t r = kma_q::clq_dequeue_n<gpu_ops_group, clq_link_head>(&q->head, &q->tail, out + served,
											 k - served, spin_limit, &timed_out, log);
			if (timed_out)
				flag_err(err, KMA_ERR_TIMEOUT);
			if (r == 0)
				break;
			served += r;
		}
		w[1] = served;
	}
	__syncthreads();
	const unsigned long long got = want && q && rank < w[1] ? out[rank] : 0ull;
	__syncthreads();
	return reinterpret_cast<kma_clqueue_item *>(got);
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
 * tag every 1024 updates).  Head is tagged the same way, on its own
 * 128-byte line, and every update increments the tag, so no CAS succeeds
 * on a recycled value; the tail, on its own line, holds the last item's
 * index.  The queue is the Michael-Scott queue with a dummy item, as the
 * reference's: init makes `first` the dummy, dequeue returns the OLD dummy
 * (so `first` comes out first and the last item enqueued always stays
 * behind), NULL when only the dummy is left.  The algorithm is
 * kma_queue_algo.cuh's: enqueue exchanges the tail and links the previous
 * tail item (no retry loop, one atomic on the shared tail, where the
 * reference CASes the link and then the tail, clIndexedQueue.cl:132-196);
 * the warp forms append a warp's items as one chain and take a warp's
 * dequeues with one CAS of the head.
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
	kma_chain_log *log;  /* chain log of the warp forms, or NULL */
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

namespace kma_detail {
/* the item links of q, as the queue algorithms address them */
/* The queue's geometry, read once into registers: the queue algorithms'
 * strong loads and atomics order every later plain load of the queue
 * struct behind them, so computing each link address from the struct
 * would put a round trip of its own in front of every link load. */
struct iq_links {
	unsigned char *base;
	unsigned long long *dummies;
	uint32_t stride_l2, capacity, nshards;
	__device__ __forceinline__ explicit iq_links(const kma_iqueue *q)
	    : base(q->base), dummies(q->dummies), stride_l2(q->stride_l2), capacity(q->capacity), nshards(q->nshards)
	{
	}
	/* iq_link with the geometry in registers */
	__device__ __forceinline__ unsigned long long *link(uint32_t idx) const
	{
		if (idx == 0)
			return &dummies[nshards - 1];
		if (idx > capacity)
			return &dummies[idx - capacity - 1];
		return reinterpret_cast<unsigned long long *>(base + ((size_t)(idx - 1) << stride_l2));
	}
};
} /* namespace kma_detail */

/* idxd_enqueue (clIndexedQueue.cl:132-196) on the caller's shard: 1 on
 * success, 0 for an item outside the array.  Never waits. */
__device__ inline int kma_iqueue_enqueue_shard(kma_iqueue *q, void *item, uint32_t shard)
{
	using namespace kma_detail;
	uint32_t idx = iq_idx(q, item);
	if (idx == 0)
		return 0;
	const iq_links L(q);
	kma_q::iq_set_link<gpu_ops>(L, idx, 0u);
	/* the link is published by the exchange (acq_rel) that appends it */
	kma_q::iq_append<gpu_ops>(L, &q->ends[2 * shard + 1].v, idx, idx);
	return 1;
}

/* idxd_dequeue (clIndexedQueue.cl:203-247) on one shard: the old dummy
 * (an item pointer), NULL when only the dummy is left or on spin-limit
 * expiry.  An internal dummy leaving the shard is skipped. */
__device__ inline void *kma_iqueue_dequeue_shard(kma_iqueue *q, uint32_t shard)
{
	using namespace kma_detail;
	const iq_links L(q);
	for (uint32_t k = 0; k < 2; k++) {
		uint32_t idx = 0;
		bool timed_out = false;
		if (!kma_q::iq_dequeue_n<gpu_ops>(L, &q->ends[2 * shard].v, &idx, 1, q->spin_limit, &timed_out,
						  (const kma_q::no_log *)nullptr)) {
			if (timed_out)
				atomicOr(&q->err, KMA_ERR_TIMEOUT);
			return nullptr;
		}
		if (idx <= q->capacity)
			return kma_iqueue_item(q, idx);
		/* shard k > 0's initial internal dummy: at most once per shard */
	}
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

/* Warp form of enqueue on each lane's shard (NULL item: none): the items
 * of one shard are linked in lane order and appended as one chain with
 * one exchange of its tail (recorded in the queue's chain log, if it has
 * one, from 2 items).  1 per appended item, 0 for an item outside the
 * array.  No counterpart in the reference. */
__device__ inline int kma_iqueue_enqueue_warp_shard(kma_iqueue *q, void *item, uint32_t shard)
{
	using namespace kma_detail;
	const uint32_t active = __activemask();
	const uint32_t lane = lane_id();
	const uint32_t idx = item ? iq_idx(q, item) : 0u;
	const bool ok = idx != 0;
	const lane_group gp = group_by(active, lane, ok ? (unsigned long long)shard : ~0ull);
	const uint32_t nidx = __shfl_sync(active, idx, gp.next);
	const uint32_t lidx = __shfl_sync(active, idx, gp.last);
	const iq_links L(q);
	/* a chain of 2 or more in a queue with a chain log: its record */
	kma_chain_log *log = q->log;
	const bool logged = ok && log && gp.size >= 2;
	uint32_t recno = 0;
	if (logged && lane == gp.first)
		recno = log->take();
	recno = __shfl_sync(active, recno, gp.first);
	if (ok) {
		if (logged)
			log->iq_slot(recno)[gp.rank] = idx;
		kma_q::iq_set_link<gpu_ops>(L, idx, gp.next != lane ? nidx : 0u,
					    logged && gp.rank == 0 ? kma_q::iq_log_tag(recno, gp.size) : 0u);
		/* every lane's link is visible before the first lane's exchange
		 * publishes the chain */
		__threadfence();
	}
	__syncwarp(active);
	if (ok && lane == gp.first)
		kma_q::iq_append<gpu_ops_group>(L, &q->ends[2 * shard + 1].v, idx, lidx);
	return ok ? 1 : 0;
}

/* Warp form of dequeue on each lane's shard (want 0: none): the lanes of
 * one shard take consecutive old dummies with one CAS of its head, in lane
 * order; lanes left over when only the dummy is left get NULL.  No
 * counterpart in the reference. */
__device__ inline void *kma_iqueue_dequeue_warp_shard(kma_iqueue *q, uint32_t shard, bool want = true)
{
	using namespace kma_detail;
	const uint32_t active = __activemask();
	const uint32_t lane = lane_id();
	const lane_group gp = group_by(active, lane, want ? (unsigned long long)shard : ~0ull);
	const iq_links L(q);
	uint32_t got = 0, served = 0;
	bool more = want;
	for (uint32_t turn = 0; __any_sync(active, more) && turn < 33; turn++) {
		uint32_t out[32];
		uint32_t r = 0;
		if (more && lane == gp.first) {
			bool timed_out = false;
			r = kma_q::iq_dequeue_n<gpu_ops_group>(L, &q->ends[2 * shard].v, out, gp.size - served, q->spin_limit,
							 &timed_out, (const kma_chain_log *)q->log);
			if (timed_out)
				atomicOr(&q->err, KMA_ERR_TIMEOUT);
			/* internal dummies leave silently */
			uint32_t k = 0;
			for (uint32_t j = 0; j < r; j++)
				if (out[j] <= q->capacity)
					out[k++] = out[j];
			if (r && !k)
				r = ~0u; /* only an internal dummy left: take again */
			else
				r = k;
		}
		r = __shfl_sync(active, r, gp.first);
		const bool again = r == ~0u;
		if (again)
			r = 0;
		const uint32_t rmax = __reduce_max_sync(active, more ? r : 0u);
		for (uint32_t j = 0; j < rmax; j++) {
			const uint32_t v = __shfl_sync(active, lane == gp.first && j < r ? out[j] : 0u, gp.first);
			if (more && j < r && gp.rank == served + j)
				got = v;
		}
		if (more && !again) {
			served += r;
			if (r == 0 || served >= gp.size)
				more = false;
		}
	}
	return got ? kma_iqueue_item(q, got) : nullptr;
}

/* Block form of dequeue on one shard (see kma_clqueue_dequeue_block):
 * every thread of the block calls it with the same q and shard; smem:
 * blockDim + 1 words.  An internal dummy leaving the shard is skipped.
 * No counterpart in the reference. */
__device__ inline void *kma_iqueue_dequeue_block_shard(kma_iqueue *q, uint32_t shard, bool want,
		unsigned long long *smem)
{
	using namespace kma_detail;
	unsigned int *w = reinterpret_cast<unsigned int *>(smem);
	uint32_t k = 0;
	const uint32_t rank = block_rank(want, &w[0], &k);
	uint32_t *out = reinterpret_cast<uint32_t *>(smem + 1);
	if (block_tid() == 0) {
		const iq_links L(q);
		const uint32_t cap = L.capacity;
		uint32_t served = 0;
		for (uint32_t turn = 0; served < k && turn <= k; turn++) {
			bool timed_out = false;
			const uint32_t r = kma_q::iq_dequeue_n<gpu_ops_group>(L, &q->ends[2 * shard].v, out + served, k - served,
									q->spin_limit, &timed_out,
									(const kma_chain_log *)q->log);
			if (timed_out)
				atomicOr(&q->err, KMA_ERR_TIMEOUT);
			if (r == 0)
				break;
			/* internal dummies leave silently */
			uint32_t kept = 0;
			for (uint32_t j = 0; j < r; j++)
				if (out[served + j] <= cap)
					out[served + kept++] = out[served + j];
			served += kept;
		}
		w[1] = served;
	}
	__syncthreads();
	const uint32_t got = want && rank < w[1] ? out[rank] : 0u;
	__syncthreads();
	return got ? kma_iqueue_item(q, got) : nullptr;
}

/* Block form on shard 0, the reference's queue. */
__device__ __forceinline__ void *kma_iqueue_dequeue_block(kma_iqueue *q, bool want, unsigned long long *smem)
{
	return kma_iqueue_dequeue_block_shard(q, 0, want, smem);
}

__device__ __forceinline__ int kma_iqueue_enqueue_warp(kma_iqueue *q, void *item)
{
	return kma_iqueue_enqueue_warp_shard(q, item, kma_detail::iq_shard(q));
}
__device__ __forceinline__ void *kma_iqueue_dequeue_warp(kma_iqueue *q)
{
	return kma_iqueue_dequeue_warp_shard(q, kma_detail::iq_shard(q));
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
