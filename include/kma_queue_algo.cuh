/*
 * kma_queue_algo.cuh -- the algorithms of the two lock-free FIFOs
 * (kma_clqueue, clQueue.cl:27-118; kma_iqueue, clIndexedQueue.cl:44-290),
 * written once over an atomics policy so that the same text runs on the
 * GPU (kma_structs.cuh binds gpu-scope PTX atomics) and on host threads
 * (oracle/queue_harness.cpp binds GCC atomics), where its concurrency
 * properties are checked before any GPU run.
 *
 * Both queues append with an EXCHANGE on the tail, never a CAS loop:
 *
 *   prev = exchange(tail, last item of the new chain); link prev to the chain
 *
 * so an append of one item or of a whole chain (a warp's items, linked
 * in lane order beforehand) costs one atomic on the shared tail word and
 * always succeeds, and the tail moves straight to the chain's last item.
 * There is no lagging tail for later appends to help forward one link at
 * a time: the Michael-Scott queue of the reference moves the tail with a
 * second CAS after linking, and a chain appended that way leaves the tail
 * on the chain's FIRST item, so every later enqueue first walks it along.
 * Between the exchange and the link the chain is not yet reachable from
 * the head; a dequeuer that meets the end of the linked part meanwhile
 * sees the queue as ending there (the pointer queue waits a bounded time
 * when that end is its last item), the one window in which these queues
 * are not linearizable.  Serially (one operation at a time) both behave
 * exactly as the reference's queues: same results, same head, tail and
 * links.
 *
 * Chain log (optional).  A dequeue that takes k items must learn their
 * addresses, and a linked list gives them one dependent load at a time.
 * With a chain log, an append of a chain of k items (a warp's) also writes
 * the k items into a log record and marks the chain's first link with the
 * record's number and k.  A dequeue that finds a marked link at the head
 * reads the record and checks every link it names with loads that do not
 * depend on one another (one round trip, not k), and takes the whole
 * chain with one move of the head; a dequeue that wants more (the block
 * forms) goes on to the next logged chains under the same hold.  A record
 * is only a hint: records are reused round robin, so a dequeue takes a
 * chain from its record only when the queue's current links say exactly
 * what the record says, and walks otherwise.
 *
 * Log policy `LG` (a null pointer, or the type no_log: no log; `enabled`
 * false compiles the log code out) provides the slot of record `recno`
 * (records are reused modulo the log's size):
 *   iq_record(recno)     32 item indices        clq_record(recno)    32 item pointers
 *   LG::ld(p)            relaxed load of one entry
 *   taken(m)             a chain of m items was taken from a record (a count)
 *
 * Policy `O` provides, on 64-bit words:
 *   ld(p)        acquire load        st(p, v)     release store
 *   ld_rlx(p)    relaxed load        st_rlx(p, v) relaxed store
 *   xchg(p, v)   acq_rel exchange    cas(p, c, v) acq_rel compare-and-swap, returns the old value
 *   pause(it)    back-off after `it` fruitless tries
 * Every wait is bounded by `limit` tries (a dequeue's: tries in which the
 * queue's head did not move, so a waiter is not failed while others make
 * progress; a head that stops moving ends every wait); expiry returns
 * failure and the caller records KMA_ERR_TIMEOUT.
 */
#ifndef KMA_QUEUE_ALGO_CUH
#define KMA_QUEUE_ALGO_CUH

#include <stdint.h>

#if defined(__CUDACC__)
#define KQ_FN __device__ __forceinline__
#define KQ_UNROLL _Pragma("unroll")
#else
#define KQ_FN inline
#define KQ_UNROLL
#endif

namespace kma_q {

typedef unsigned long long u64;

/* ------------------------------------------------------------------ */
/* pointer queue (clQueue)                                             */
/* ------------------------------------------------------------------ */
/* head: {tag:16 | item pointer:48}, the tag bumped by every change, so a
 * stale CAS on it fails; tail: the last item's pointer (0 = empty),
 * changed only by exchange (append) and by the dequeue that empties the
 * queue (CAS last item -> 0).  Item links: next item, 0 = none yet,
 * POISON = held by a dequeuer or removed (the reference's claim,
 * clQueue.cl:97; removed items keep it until enqueued again). */
const u64 POISON = 1ull;
const int PTR_BITS = 48;
const u64 PTR_MASK = (1ull << PTR_BITS) - 1ull;

/* chain log records: numbers of 24 bits, chains of at most 32 items */
const uint32_t LOG_RECNO_MASK = 0xFFFFFFu;
const uint32_t LOG_CHAIN_MAX = 32;

/* The log policy of callers without a log: the log code compiles away. */
struct no_log {
	static constexpr bool enabled = false;
	KQ_FN const u64 *clq_record(uint32_t) const { return nullptr; }
	KQ_FN const uint32_t *iq_record(uint32_t) const { return nullptr; }
	static KQ_FN u64 ld(const u64 *) { return 0; }
	static KQ_FN uint32_t ld(const uint32_t *) { return 0; }
	KQ_FN void taken(uint32_t) const {}
};

KQ_FN u64 qp_ptr(u64 w) { return w & PTR_MASK; }
KQ_FN u64 qp_next(u64 w, u64 ptr) { return (((w >> PTR_BITS) + 1ull) << PTR_BITS) | ptr; }

/* A logged chain (at least 3 items) marks the top 16 bits of its first
 * two links: first = CLQ_LOG | (length - 1) << 10 | record number bits
 * 14..23, second = record number bits 0..13 (its top two bits stay clear,
 * so it never reads as a first or into mark).  The append that links the
 * chain after the previous tail item marks that link too (the link INTO
 * the chain): CLQ_INTO | record number bits 0..13, so that a dequeuer that
 * reaches the chain over that link has its whole record number without
 * loading the second link first.  Every other link has the top bits
 * clear; readers take the pointer with qp_ptr. */
const u64 CLQ_LOG = 0x8000ull << PTR_BITS;
const u64 CLQ_INTO = 0x4000ull << PTR_BITS;
KQ_FN u64 clq_mark_first(uint32_t recno, uint32_t len)
{
	return CLQ_LOG | ((u64)(((len - 1u) << 10) | ((recno >> 14) & 0x3FFu)) << PTR_BITS);
}
KQ_FN u64 clq_mark_second(uint32_t recno) { return (u64)(recno & 0x3FFFu) << PTR_BITS; }
KQ_FN u64 clq_mark_into(uint32_t recno) { return CLQ_INTO | ((u64)(recno & 0x3FFFu) << PTR_BITS); }

/* Up to k items [hp, ...] of the logged chain that starts at hp (its link
 * v), if its record matches the links: fills out[], sets *nh to the item
 * after them, returns how many (0: no usable record).  `into`: the link
 * that leads to hp as read (0 if unknown); *nh_link: the link that leads
 * to *nh when the whole chain was taken, else 0.  Reads only. */
template <class O, class L, class LG>
KQ_FN uint32_t clq_chain_from_log(const LG *log, u64 hp, u64 v, u64 *out, uint32_t k, u64 *nh, u64 into = 0,
		u64 *nh_link = nullptr)
{
	if (nh_link)
		*nh_link = 0;
	if constexpr (!LG::enabled)
		return 0;
	if (!log || !(v & CLQ_LOG) || k == 0)
		return 0;
	const uint32_t mark = (uint32_t)(v >> PTR_BITS);
	const uint32_t len = ((mark >> 10) & 31u) + 1u;
	const u64 second = qp_ptr(v);
	if (len < 3 || second <= POISON)
		return 0;
	/* relaxed loads, issued back to back into registers: an acquire load,
	 * or a store of each value before the next load, would make them one
	 * round trip each, as a walk.  The exchange that took the head
	 * already ordered the chain's contents before these reads.  The low
	 * record-number bits come from the link into hp when it carries them
	 * (then the second link loads with the others), else from the second
	 * link, loaded first. */
	const bool via_into = (into & CLQ_INTO) && !(into & CLQ_LOG) && qp_ptr(into) == hp;
	u64 l1 = via_into ? 0ull : O::ld_rlx(L::at(second));
	const uint32_t recno = ((mark & 0x3FFu) << 14) |
			       ((uint32_t)((via_into ? into : l1) >> PTR_BITS) & 0x3FFFu);
	uint32_t m = len < k ? len : k;
	const u64 *rec = log->clq_record(recno);
	u64 item[LOG_CHAIN_MAX];
KQ_UNROLL
	for (uint32_t j = 0; j < LOG_CHAIN_MAX; j++)
		item[j] = j <= m && j < len ? LG::ld(rec + j) : 0ull;
	if (via_into)
		l1 = O::ld_rlx(L::at(second));
	const u64 after = m < len ? item[m < LOG_CHAIN_MAX ? m : 0] : 0ull;
	if (item[0] != hp || (m > 1 && item[1] != second) || (m > 2 && item[2] != qp_ptr(l1)))
		return 0;
	/* record entries are 0 or item pointers (0 in a slot a chain has not
	 * filled, or is refilling): none may be followed before it is known
	 * to be an item */
	bool ok = true;
KQ_UNROLL
	for (uint32_t j = 2; j < LOG_CHAIN_MAX; j++)
		ok &= !(j < m && item[j] <= POISON);
	if (!ok)
		return 0;
	/* each item's link must name the next item (for the last one taken:
	 * the new head) */
	u64 nxs[LOG_CHAIN_MAX];
KQ_UNROLL
	for (uint32_t j = 2; j < LOG_CHAIN_MAX; j++)
		nxs[j] = j < m ? O::ld_rlx(L::at(item[j])) : 0ull;
	u64 last = m == 1 ? second : (m == 2 ? l1 : 0ull);
KQ_UNROLL
	for (uint32_t j = 2; j < LOG_CHAIN_MAX; j++) {
		if (j + 1 < m)
			ok &= nxs[j] != POISON && qp_ptr(nxs[j]) == item[j + 1];
		else if (j + 1 == m)
			last = nxs[j];
	}
	if (!ok || last == POISON)
		return 0;
	u64 next = qp_ptr(last);
	if (m < len) {
		if (next != after || next == 0)
			return 0;
	} else if (next == 0) {
		/* the chain's last item has no successor yet: it stays, as the head */
		next = item[(m - 1) & (LOG_CHAIN_MAX - 1)];
		m--;
	} else if (nh_link) {
		*nh_link = last;
	}
KQ_UNROLL
	for (uint32_t j = 0; j < LOG_CHAIN_MAX; j++)
		if (j < m)
			out[j] = item[j];
	*nh = next;
	return m;
}

/* Append the chain first..last (its links already set, last's link 0,
 * all of it written before the call).  `into`: mark bits for the link from
 * the previous tail item to `first` (clq_mark_into of a logged chain, or
 * 0).  1, or 0 when a wait expired. */
template <class O, class L>
KQ_FN int clq_append(u64 *headw, u64 *tailw, u64 first, u64 last, uint32_t limit, u64 into = 0)
{
	const u64 prev = O::xchg(tailw, last);
	if (prev == 0) {
		/* the queue was empty: the chain becomes the head.  The dequeue
		 * that emptied the queue may not have cleared the head yet. */
		for (uint32_t it = 0; it < limit; it++) {
			const u64 h = O::ld(headw);
			if (qp_ptr(h) == 0 && O::cas(headw, h, qp_next(h, first)) == h)
				return 1;
			O::pause(it);
		}
		return 0;
	}
	/* link after prev; a dequeuer that holds prev's link (POISON) to see
	 * whether prev is the last item gives it back at once */
	u64 *pl = L::at(prev);
	for (uint32_t it = 0; it < limit; it++) {
		const u64 old = O::cas(pl, 0ull, first | into);
		if (old == 0)
			return 1;
		if (old != POISON)
			return 0; /* prev has a successor already: an item enqueued twice */
		O::pause(it);
	}
	return 0;
}

/* Take the head item and up to k-1 items after it, in FIFO order, into
 * out[].  Returns the number taken; 0 when the queue is empty, and 0 with
 * *timed_out set when a wait expired.  The caller holds nothing after.
 *
 * The head item is claimed by exchanging its link for POISON (as the
 * reference does); while a dequeuer holds it nobody else can move the
 * head, so the items behind it are read without further atomics and the
 * head moves past all of them with one store.  Taken items keep POISON
 * in their links. */
template <class O, class L, class LG>
KQ_FN uint32_t clq_dequeue_n(u64 *headw, u64 *tailw, u64 *out, uint32_t k, uint32_t limit, bool *timed_out,
		const LG *log)
{
	*timed_out = false;
	uint32_t it = 0, idle = 0;
	u64 last = ~0ull;
	for (;;) {
		/* waiters poll with relaxed loads: an acquire load also invalidates
		 * the SM's L1 on the GPU (under contention thousands of waiters
		 * would keep evicting the holder's local data); the exchange that
		 * takes the head item is the acquire */
		const u64 h = O::ld_rlx(headw);
		/* `limit` bounds the tries in which the head did not move: one of
		 * many waiters on a head may wait long while the others take
		 * items, and only a head that stops moving means a stuck queue */
		if (h != last) {
			last = h;
			idle = 0;
		} else if (++idle >= limit) {
			break;
		}
		const u64 hp = qp_ptr(h);
		if (hp == 0)
			return 0;
		u64 *hl = L::at(hp);
		/* look before taking: while another dequeuer holds the head item,
		 * waiters only read its link */
		const u64 seen = O::ld_rlx(hl);
		if (seen == POISON) {
			O::pause(it++);
			continue;
		}
		const u64 nx = O::xchg(hl, POISON);
		if (nx == POISON) {
			/* another dequeuer holds it, or it left the queue already */
			O::pause(it++);
			continue;
		}
		/* hp's link is ours; hp is the head unless the head moved since
		 * it was read (hp taken, then enqueued again elsewhere) */
		if (O::ld(headw) != h) {
			O::st(hl, nx);
			O::pause(it++);
			continue;
		}
		/* a logged chain at the head: its record, checked against the
		 * links while the head is held (the items behind a held head
		 * cannot move), gives the chain without walking it */
		u64 nh = 0, into = 0;
		uint32_t m = clq_chain_from_log<O, L>(log, hp, nx, out, k, &nh, 0ull, &into);
		if (m) {
			log->taken(m);
			/* more whole chains behind it, still under the same hold:
			 * each costs its first link, its record and its links (the
			 * link that led to it carries the rest of its record
			 * number), not a hold of its own */
			while (m < k && nh != 0) {
				u64 nh2 = 0, into2 = 0;
				const uint32_t m2 = clq_chain_from_log<O, L>(log, nh, O::ld_rlx(L::at(nh)), out + m, k - m,
									     &nh2, into, &into2);
				if (!m2)
					break;
				log->taken(m2);
				m += m2;
				nh = nh2;
				into = into2;
			}
			for (uint32_t j = 1; j < m; j++)
				O::st_rlx(L::at(out[j]), POISON);
			O::st(headw, qp_next(h, nh));
			return m;
		}
		if (nx != 0) {
			out[0] = hp;
			uint32_t r = 1;
			u64 cur = qp_ptr(nx);
			while (r < k) {
				const u64 n2 = O::ld(L::at(cur));
				if (n2 == 0 || n2 == POISON)
					break; /* cur is the last linked item: it stays, as the head */
				O::st_rlx(L::at(cur), POISON);
				out[r++] = cur;
				cur = qp_ptr(n2);
			}
			O::st(headw, qp_next(h, cur));
			return r;
		}
		/* hp is the last linked item: the only item when the tail still
		 * names it; otherwise an append has exchanged the tail and is
		 * about to link after hp */
		if (O::cas(tailw, hp, 0ull) == hp) {
			O::st(headw, qp_next(h, 0ull));
			out[0] = hp;
			return 1;
		}
		/* give the link back and wait for the append to land */
		O::st(hl, 0ull);
		while (idle < limit && O::ld(hl) == 0ull && O::ld(headw) == h) {
			O::pause(it++);
			idle++;
		}
	}
	*timed_out = true;
	return 0;
}

/* ------------------------------------------------------------------ */
/* indexed queue (clIndexedQueue)                                      */
/* ------------------------------------------------------------------ */
/* Words {tag:32 | index:32}, index 0 = none.  The Michael-Scott queue
 * with a dummy item, as the reference's: head names the dummy, dequeue
 * moves head to the dummy's successor and returns the OLD dummy, NULL
 * when the dummy has no successor.  Appends exchange the tail and then
 * store the link of the previous tail item, which nobody else writes: a
 * dummy leaves the queue only once its successor is linked, so the
 * previous tail item is still in the queue when its link is stored.
 * A link is written only by the append that links after it (0 -> item)
 * and by its own item's next enqueue (reset to 0). */
KQ_FN uint32_t tw_idx(u64 w) { return (uint32_t)w; }
KQ_FN uint32_t tw_tag(u64 w) { return (uint32_t)(w >> 32); }
KQ_FN u64 tw_make(uint32_t tag, uint32_t idx) { return ((u64)tag << 32) | idx; }

/* Links need no ABA tag (nothing CASes them): a link's tag is 0, or, on
 * the first link of a logged chain, IQ_LOG | record number (24 bits) << 5 |
 * (chain length - 1).  Head keeps a counting tag. */
const uint32_t IQ_LOG = 0x80000000u;
KQ_FN uint32_t iq_log_tag(uint32_t recno, uint32_t len)
{
	return IQ_LOG | ((recno & LOG_RECNO_MASK) << 5) | (len - 1u);
}

/* Q provides u64 *link(uint32_t idx); every index the queue can hold,
 * and 0 (a zero word), has one. */
template <class O, class Q>
KQ_FN void iq_append(const Q &q, u64 *tailw, uint32_t first, uint32_t last)
{
	const u64 prev = O::xchg(tailw, tw_make(0, last));
	O::st(q.link(tw_idx(prev)), tw_make(0, first));
}

/* Set item idx's link (to 0, or to the next item of a chain; tag: 0, or
 * iq_log_tag on a logged chain's first item) before idx is appended. */
template <class O, class Q>
KQ_FN void iq_set_link(const Q &q, uint32_t idx, uint32_t next, uint32_t tag = 0)
{
	O::st_rlx(q.link(idx), tw_make(tag, next));
}

/* Take up to k items [h0 = head, ...] of the logged chain that starts at
 * the head, if its record matches the links: fills out[], sets *nh to the
 * head after them, returns how many (0: no usable record).  l0 = h0's
 * link.  The head is not moved here. */
template <class O, class Q, class LG>
KQ_FN uint32_t iq_chain_from_log(const Q &q, const LG *log, uint32_t h0, u64 l0, uint32_t *out, uint32_t k,
		uint32_t *nh)
{
	if constexpr (!LG::enabled)
		return 0;
	if (!log || k == 0)
		return 0;
	/* The head is a dummy when whole chains were taken before: it is the
	 * last item of the chain before, and the next chain starts at its
	 * successor.  Take the dummy, then up to k-1 items of that chain. */
	uint32_t lead = 0;
	if (!(tw_tag(l0) & IQ_LOG)) {
		const uint32_t n1 = tw_idx(l0);
		if (n1 == 0 || k < 2)
			return 0;
		lead = h0;
		h0 = n1;
		l0 = O::ld_rlx(q.link(n1));
		k--;
		if (!(tw_tag(l0) & IQ_LOG))
			return 0;
	}
	const uint32_t tag = tw_tag(l0);
	const uint32_t len = (tag & 31u) + 1u;
	const uint32_t recno = (tag >> 5) & LOG_RECNO_MASK;
	/* the record's items, and the link after each: item j -> item j+1 must
	 * hold for the items taken and for the one that becomes the head.
	 * Loads into registers, back to back (see clq_chain_from_log). */
	uint32_t m = len < k ? len : k;
	const uint32_t *rec = log->iq_record(recno);
	uint32_t item[LOG_CHAIN_MAX];
KQ_UNROLL
	for (uint32_t j = 0; j < LOG_CHAIN_MAX; j++)
		item[j] = j <= m && j < len ? LG::ld(rec + j) : 0u;
	const uint32_t after = m < len ? item[m < LOG_CHAIN_MAX ? m : 0] : 0u;
	if (item[0] != h0 || (m > 1 && item[1] != tw_idx(l0)) || (m == 1 && len > 1 && after != tw_idx(l0)))
		return 0;
	uint32_t nxs[LOG_CHAIN_MAX];
KQ_UNROLL
	for (uint32_t j = 1; j < LOG_CHAIN_MAX; j++)
		nxs[j] = j < m ? tw_idx(O::ld_rlx(q.link(item[j]))) : 0u;
	bool ok = true;
	uint32_t next = m == 1 ? tw_idx(l0) : 0u;
KQ_UNROLL
	for (uint32_t j = 1; j < LOG_CHAIN_MAX; j++) {
		if (j + 1 < m)
			ok &= nxs[j] == item[j + 1];
		else if (j + 1 == m)
			next = nxs[j];
	}
	if (!ok)
		return 0;
	if (m < len) {
		if (next != after || next == 0)
			return 0;
	} else if (next == 0) {
		/* the chain's last item has no successor yet: it stays, as the head */
		if (m == 1)
			return 0;
		next = item[(m - 1) & (LOG_CHAIN_MAX - 1)];
		m--;
	}
	const uint32_t off = lead ? 1u : 0u;
	if (lead)
		out[0] = lead;
KQ_UNROLL
	for (uint32_t j = 0; j < LOG_CHAIN_MAX; j++)
		if (j < m)
			out[j + off] = item[j];
	*nh = next;
	return m + off;
}

/* Dequeue up to k old dummies into out[] (indices, FIFO order).  Returns
 * the number taken: 0 when the dummy has no successor, or (with
 * *timed_out) when the head stayed held past `limit` tries.
 *
 * A dequeuer holds the head while it takes its items: the head's tag is
 * even when free and odd while held (a CAS to tag+1 takes it, the store
 * of the new head with tag+2 gives it back).  The holder reads the chain
 * behind the head (from the log, or link by link) and moves the head past
 * it; others wait reading the head, so a batch's loads are issued by one
 * dequeuer at a time instead of by every contender.  A holder never waits
 * for anything, so a hold lasts a few round trips. */
KQ_FN bool iq_head_held(u64 hd) { return tw_tag(hd) & 1u; }
template <class O, class Q, class LG>
KQ_FN uint32_t iq_dequeue_n(const Q &q, u64 *headw, uint32_t *out, uint32_t k, uint32_t limit, bool *timed_out,
		const LG *log)
{
	*timed_out = false;
	uint32_t idle = 0;
	u64 last = ~0ull;
	for (uint32_t it = 0;; it++) {
		/* relaxed polling, as in clq_dequeue_n; the CAS that takes the
		 * head is the acquire.  `limit` bounds the tries in which the
		 * head did not move (see clq_dequeue_n). */
		const u64 hd = O::ld_rlx(headw);
		if (hd != last) {
			last = hd;
			idle = 0;
		} else if (++idle >= limit) {
			break;
		}
		if (iq_head_held(hd)) {
			O::pause(it);
			continue;
		}
		uint32_t cur = tw_idx(hd), r = 0;
		const u64 l0 = O::ld_rlx(q.link(cur));
		if (tw_idx(l0) == 0) {
			/* only the dummy: empty, if the head is still this one */
			if (O::ld_rlx(headw) == hd)
				return 0;
			continue;
		}
		if (O::cas(headw, hd, tw_make(tw_tag(hd) + 1u, cur)) != hd) {
			O::pause(it);
			continue;
		}
		/* held: the items behind the head cannot leave the queue */
		uint32_t nh = 0;
		if constexpr (LG::enabled)
			if (log)
				r = iq_chain_from_log<O>(q, log, cur, O::ld(q.link(cur)), out, k, &nh);
		if (r) {
			log->taken(r);
			cur = nh;
			/* more whole chains behind it under the same hold (see
			 * clq_dequeue_n); the head item's link is read with acquire,
			 * as the first one */
			while (r < k) {
				uint32_t nh2 = 0;
				const uint32_t r2 = iq_chain_from_log<O>(q, log, cur, O::ld(q.link(cur)), out + r, k - r, &nh2);
				if (!r2)
					break;
				log->taken(r2);
				r += r2;
				cur = nh2;
			}
		} else {
			while (r < k) {
				const uint32_t nx = tw_idx(O::ld(q.link(cur)));
				if (nx == 0)
					break;
				out[r++] = cur;
				cur = nx;
			}
		}
		O::st(headw, tw_make(tw_tag(hd) + 2u, cur));
		return r;
	}
	*timed_out = true;
	return 0;
}

} /* namespace kma_q */

#endif /* KMA_QUEUE_ALGO_CUH */
