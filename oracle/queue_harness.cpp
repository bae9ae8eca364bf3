/*
 * queue_harness.cpp -- TEST INFRASTRUCTURE: runs the queue algorithms of
 * include/kma_queue_algo.cuh (the text the GPU runs) on host threads, bound
 * to GCC atomics, and checks what the device tests check at scale, plus
 * what a GPU run cannot provoke on purpose:
 *
 *   - conservation: every append is taken exactly once, by a dequeue or
 *     as what is left in the queue at the end (found by walking it);
 *   - FIFO per appender: what one thread appended reaches each consumer
 *     in the order appended (chains and single items alike);
 *   - structure at the end: the walk from head ends at the tail, every
 *     taken pointer-queue item keeps POISON, no wait expired;
 *   - the append window: with probability DELAY_PROB an append sleeps (up
 *     to 200 us) between its exchange of the tail and its link -- the
 *     moment at which its chain is not reachable yet -- while other
 *     threads append behind it and dequeue up to it;
 *   - recycling (ABA): consumers append again, as one chain, each item
 *     they take with probability RECYCLE while it has been appended fewer
 *     than three times, as the reference's queue tests shuffle items
 *     (dequeue -> enqueue), so items leave and re-enter the queue.
 *
 *   - the chain log: with LOG_RECORDS > 0 every chain appended (of 3 or
 *     more items for the pointer queue, 2 or more for the indexed one) is
 *     recorded in a log of that many records, reused round robin (a small
 *     log is overwritten while its chains are still queued, so dequeues
 *     meet stale records), and dequeues take chains from their records.
 *
 *   - stuck queues (`queue_harness stuck`): a dequeuer that died holding
 *     the head, an append that exchanged the tail and never linked, an
 *     indexed head left held: every dequeue must give up within its limit
 *     and report it.
 *
 *   queue_harness clq|iq THREADS CHAINS MAX_CHAIN DEQ_BATCH DELAY_PROB SEED
 *                 [PRODUCERS [RECYCLE [LOG_RECORDS [PHASED]]]]
 *   queue_harness stuck
 *
 * PRODUCERS of the threads (default half) append CHAINS fresh chains of
 * 1..MAX_CHAIN items each; the rest take batches of 1..DEQ_BATCH until
 * the producers are done and the queue is empty (a negative MAX_CHAIN or
 * DEQ_BATCH: exactly that many, as warps append and blocks dequeue).
 * With few producers the queue is mostly empty, so the empty <-> one-item
 * transitions and the append window are met all the time; PHASED 1 holds
 * the consumers back until the producers are done (config 3's order), so
 * batches meet whole logged chains and take several per hold.  Prints one
 * JSON line (with the chains taken from records and the dequeue calls
 * that took items); exits 0 when every check passed.  The reference's own
 * queues are the parity oracle (serial replays against tests/golden);
 * this program checks this build's concurrent behaviour.
 */
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <thread>
#include <vector>

#include "kma_queue_algo.cuh"

using kma_q::u64;

namespace {

u64 *g_tail_word = nullptr; /* the word whose exchange may be delayed */
double g_delay_prob = 0.0;
std::atomic<uint64_t> g_delays{0};

thread_local uint64_t t_rng = 1;
inline uint64_t rnd()
{
	uint64_t z = (t_rng += 0x9E3779B97F4A7C15ull);
	z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
	z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
	return z ^ (z >> 31);
}
inline double unit() { return (double)(rnd() >> 11) * (1.0 / 9007199254740992.0); }

struct HostOps {
	static u64 ld(u64 *p) { return __atomic_load_n(p, __ATOMIC_ACQUIRE); }
	static u64 ld_rlx(u64 *p) { return __atomic_load_n(p, __ATOMIC_RELAXED); }
	static void st(u64 *p, u64 v) { __atomic_store_n(p, v, __ATOMIC_RELEASE); }
	static void st_rlx(u64 *p, u64 v) { __atomic_store_n(p, v, __ATOMIC_RELAXED); }
	static u64 xchg(u64 *p, u64 v)
	{
		u64 old = __atomic_exchange_n(p, v, __ATOMIC_ACQ_REL);
		if (p == g_tail_word && g_delay_prob > 0 && unit() < g_delay_prob) {
			g_delays++;
			std::this_thread::sleep_for(std::chrono::microseconds(rnd() % 200));
		}
		return old;
	}
	static u64 cas(u64 *p, u64 c, u64 v)
	{
		__atomic_compare_exchange_n(p, &c, v, false, __ATOMIC_ACQ_REL, __ATOMIC_ACQUIRE);
		return c;
	}
	static void pause(uint32_t it)
	{
		if (it > 16)
			std::this_thread::yield();
	}
};

/* Who appended an item last (thread, that thread's running count), and
 * how many times it has been appended. */
struct Stamp {
	uint32_t owner, seq, hops;
};
struct Item {
	u64 next;
	Stamp st;
};
struct LinkAtItem {
	static u64 *at(u64 p) { return reinterpret_cast<u64 *>(p); }
};

/* host waits: long enough for any sleeping appender, short enough that a
 * corrupted queue shows as reported timeouts rather than a hang */
const uint32_t LIMIT = 1u << 18;
const uint32_t HOPS = 3;

/* The chain log: records of 32 items, reused modulo the record count. */
struct HostLog {
	static constexpr bool enabled = true;
	std::vector<u64> clq;
	std::vector<uint32_t> iq;
	uint32_t mask = 0;
	std::atomic<uint32_t> next{0};
	const u64 *clq_record(uint32_t recno) const { return &clq[(size_t)(recno & mask) * 32]; }
	const uint32_t *iq_record(uint32_t recno) const { return &iq[(size_t)(recno & mask) * 32]; }
	static u64 ld(const u64 *p) { return __atomic_load_n(p, __ATOMIC_RELAXED); }
	static uint32_t ld(const uint32_t *p) { return __atomic_load_n(p, __ATOMIC_RELAXED); }
	uint32_t take() { return next.fetch_add(1) & kma_q::LOG_RECNO_MASK; }
	mutable std::atomic<uint64_t> chains{0};
	void taken(uint32_t) const { chains++; }
};
HostLog g_log;
const HostLog *log_ptr() { return g_log.mask || !g_log.clq.empty() || !g_log.iq.empty() ? &g_log : nullptr; }

struct Result {
	uint64_t enq = 0, deq = 0, left = 0, bad = 0, order = 0, timeouts = 0, holds = 0;
};

int g_producers = 0;
/* MAX_CHAIN or DEQ_BATCH given negative: every chain / every batch has
 * exactly that many items (a warp's chains, a block's dequeues) */
bool g_fixed_chain = false, g_fixed_batch = false;
/* consumers start when every producer is done (config 3's enqueue-then-
 * dequeue phases: the queue holds whole chains, so batches meet the log) */
bool g_phased = false;

void split(int threads, int &np, int &nc)
{
	np = g_producers > 0 ? g_producers : (threads > 1 ? threads / 2 : 1);
	if (np >= threads)
		np = threads > 1 ? threads - 1 : 1;
	nc = threads > np ? threads - np : 1;
}

/* appends[i] / takes[i]: item i's appends and takes */
struct Book {
	std::vector<uint64_t> appends, takes;
	std::atomic<uint64_t> enq{0}, deq{0}, order_bad{0}, tmo{0}, holds{0};
	uint64_t cap; /* more takes than this: the queue hands items out twice */
	Book(size_t n, uint64_t c) : appends(n, 0), takes(n, 0), cap(c) {}
	/* a fault is already reported: the threads stop rather than wait out
	 * more limits on a queue known to be broken */
	bool runaway() const { return deq.load() > cap || tmo.load() > 0; }
};

/* the last sequence number this consumer saw from each appender */
struct Orders {
	std::vector<int64_t> last;
	explicit Orders(size_t owners) : last(owners, -1) {}
	bool ok(const Stamp &s)
	{
		if ((int64_t)s.seq <= last[s.owner])
			return false;
		last[s.owner] = s.seq;
		return true;
	}
};

/* ---------------------------------------------------------- pointer queue */
void run_clq(int threads, int chains, int maxc, int batch, double recycle, uint64_t seed, Result &R)
{
	int np, nc;
	split(threads, np, nc);
	const uint64_t per = (uint64_t)chains * maxc;
	std::vector<Item> items((size_t)np * per);
	alignas(16) u64 q[2] = {0, 0}; /* head, tail */
	g_tail_word = &q[1];
	std::atomic<int> producing{np};
	Book bk(items.size(), (uint64_t)items.size() * HOPS);
	auto append = [&](Item **v, int len, uint32_t owner, uint32_t &seq) {
		const bool logged = log_ptr() && len >= 3;
		const uint32_t recno = logged ? g_log.take() : 0;
		for (int j = 0; j < len; j++) {
			v[j]->st.owner = owner;
			v[j]->st.seq = seq++;
			v[j]->st.hops++;
			__atomic_fetch_add(&bk.appends[(size_t)(v[j] - items.data())], 1, __ATOMIC_RELAXED);
			u64 link = j + 1 < len ? (u64)v[j + 1] : 0ull;
			if (logged) {
				__atomic_store_n(&g_log.clq[(size_t)(recno & g_log.mask) * 32 + j], (u64)v[j], __ATOMIC_RELAXED);
				link |= j == 0 ? kma_q::clq_mark_first(recno, (uint32_t)len)
					       : (j == 1 ? kma_q::clq_mark_second(recno) : 0ull);
			}
			__atomic_store_n(&v[j]->next, link, __ATOMIC_RELAXED);
		}
		if (!kma_q::clq_append<HostOps, LinkAtItem>(&q[0], &q[1], (u64)v[0], (u64)v[len - 1], LIMIT,
							     logged ? kma_q::clq_mark_into(recno) : 0ull))
			bk.tmo++;
		bk.enq += len;
	};
	auto producer = [&](int p) {
		t_rng = seed * 0x9E3779B97F4A7C15ull + 0x1000u + p;
		Item *mine = &items[(size_t)p * per];
		std::vector<Item *> v(maxc);
		uint32_t seq = 0, used = 0;
		for (int c = 0; c < chains && !bk.runaway(); c++) {
			int len = g_fixed_chain ? maxc : 1 + (int)(rnd() % maxc);
			for (int j = 0; j < len; j++)
				v[j] = &mine[used + j];
			used += len;
			append(v.data(), len, (uint32_t)p, seq);
		}
		producing--;
	};
	auto consumer = [&](int c) {
		t_rng = seed * 0x9E3779B97F4A7C15ull + 0x2000u + c;
		while (g_phased && producing.load() != 0)
			std::this_thread::yield();
		Orders ord((size_t)np + nc);
		std::vector<u64> out(batch);
		std::vector<Item *> back;
		uint32_t seq = 0;
		for (;;) {
			bool done = producing.load() == 0;
			bool to = false;
			uint32_t k = g_fixed_batch ? (uint32_t)batch : 1 + (uint32_t)(rnd() % batch);
			uint32_t r = kma_q::clq_dequeue_n<HostOps, LinkAtItem>(&q[0], &q[1], out.data(), k, LIMIT, &to,
									       log_ptr());
			if (to)
				bk.tmo++;
			back.clear();
			for (uint32_t i = 0; i < r; i++) {
				Item *it = reinterpret_cast<Item *>(out[i]);
				__atomic_fetch_add(&bk.takes[(size_t)(it - items.data())], 1, __ATOMIC_RELAXED);
				if (!ord.ok(it->st))
					bk.order_bad++;
				if (it->st.hops < HOPS && unit() < recycle)
					back.push_back(it);
			}
			bk.deq += r;
			bk.holds += r ? 1 : 0;
			if (!back.empty())
				/* re-appended in chains of at most 32, a warp's */
				for (size_t o = 0; o < back.size(); o += 32)
					append(back.data() + o, (int)std::min<size_t>(32, back.size() - o), (uint32_t)(np + c),
					       seq);
			if (to || bk.runaway())
				break;
			if (r == 0 && done && kma_q::qp_ptr(HostOps::ld(&q[0])) == 0)
				break;
		}
	};
	std::vector<std::thread> ts;
	for (int p = 0; p < np; p++)
		ts.emplace_back(producer, p);
	for (int c = 0; c < nc; c++)
		ts.emplace_back(consumer, c);
	for (auto &t : ts)
		t.join();
	/* what is left: re-appends made after the other consumers stopped */
	uint64_t left = 0, bad = bk.deq.load() > bk.cap ? 1 : 0;
	u64 lastp = 0;
	for (u64 p = kma_q::qp_ptr(q[0]); p && p != kma_q::POISON && left <= items.size();
	     p = kma_q::qp_ptr(reinterpret_cast<Item *>(p)->next)) {
		bk.takes[(size_t)(reinterpret_cast<Item *>(p) - items.data())]++;
		left++;
		lastp = p;
	}
	if (lastp != q[1])
		bad++; /* the walk ends at the tail (both 0 when empty) */
	for (size_t i = 0; i < items.size(); i++)
		if (bk.takes[i] != bk.appends[i])
			bad++;
	if (left == 0)
		for (size_t i = 0; i < items.size(); i++)
			if (bk.appends[i] && items[i].next != kma_q::POISON)
				bad++; /* taken items keep POISON */
	R.enq = bk.enq;
	R.deq = bk.deq;
	R.holds = bk.holds;
	R.left = left;
	R.bad = bad;
	R.order = bk.order_bad;
	R.timeouts = bk.tmo;
}

/* ---------------------------------------------------------- indexed queue */
struct IdxQ {
	std::vector<u64> *links; /* links[0] is the nil word; item i at links[i] */
	u64 *link(uint32_t i) const { return &(*links)[i]; }
};

void run_iq(int threads, int chains, int maxc, int batch, double recycle, uint64_t seed, Result &R)
{
	int np, nc;
	split(threads, np, nc);
	const uint64_t per = (uint64_t)chains * maxc;
	const uint64_t n = (uint64_t)np * per;
	/* index 1 is the initial dummy; producer p owns 2 + p*per ... */
	std::vector<u64> links(n + 2, 0);
	std::vector<Stamp> st(n + 2, Stamp{0, 0, 0});
	IdxQ q{&links};
	alignas(16) u64 ends[2] = {kma_q::tw_make(0, 1), kma_q::tw_make(0, 1)};
	g_tail_word = &ends[1];
	std::atomic<int> producing{np};
	Book bk(n + 2, (n + 1) * HOPS);
	bk.appends[1] = 1; /* the initial dummy counts as appended */
	auto append = [&](const uint32_t *v, int len, uint32_t owner, uint32_t &seq) {
		const bool logged = log_ptr() && len >= 2;
		const uint32_t recno = logged ? g_log.take() : 0;
		for (int j = 0; j < len; j++) {
			st[v[j]].owner = owner;
			st[v[j]].seq = seq++;
			st[v[j]].hops++;
			__atomic_fetch_add(&bk.appends[v[j]], 1, __ATOMIC_RELAXED);
			if (logged)
				__atomic_store_n(&g_log.iq[(size_t)(recno & g_log.mask) * 32 + j], v[j], __ATOMIC_RELAXED);
			kma_q::iq_set_link<HostOps>(q, v[j], j + 1 < len ? v[j + 1] : 0u,
						    logged && j == 0 ? kma_q::iq_log_tag(recno, (uint32_t)len) : 0u);
		}
		kma_q::iq_append<HostOps>(q, &ends[1], v[0], v[len - 1]);
		bk.enq += len;
	};
	auto producer = [&](int p) {
		t_rng = seed * 0x9E3779B97F4A7C15ull + 0x3000u + p;
		const uint32_t base = 2 + (uint32_t)(p * per);
		std::vector<uint32_t> v(maxc);
		uint32_t seq = 0, used = 0;
		for (int c = 0; c < chains && !bk.runaway(); c++) {
			int len = g_fixed_chain ? maxc : 1 + (int)(rnd() % maxc);
			for (int j = 0; j < len; j++)
				v[j] = base + used + j;
			used += len;
			append(v.data(), len, (uint32_t)p, seq);
		}
		producing--;
	};
	auto consumer = [&](int c) {
		t_rng = seed * 0x9E3779B97F4A7C15ull + 0x4000u + c;
		while (g_phased && producing.load() != 0)
			std::this_thread::yield();
		Orders ord((size_t)np + nc);
		std::vector<uint32_t> out(batch), back;
		uint32_t seq = 0;
		for (;;) {
			bool done = producing.load() == 0;
			bool to = false;
			uint32_t k = g_fixed_batch ? (uint32_t)batch : 1 + (uint32_t)(rnd() % batch);
			uint32_t r = kma_q::iq_dequeue_n<HostOps>(q, &ends[0], out.data(), k, LIMIT, &to, log_ptr());
			if (to)
				bk.tmo++;
			back.clear();
			for (uint32_t i = 0; i < r; i++) {
				uint32_t idx = out[i];
				__atomic_fetch_add(&bk.takes[idx], 1, __ATOMIC_RELAXED);
				if (idx >= 2 && !ord.ok(st[idx]))
					bk.order_bad++;
				if (idx >= 2 && st[idx].hops < HOPS && unit() < recycle)
					back.push_back(idx);
			}
			bk.deq += r;
			bk.holds += r ? 1 : 0;
			if (!back.empty())
				/* re-appended in chains of at most 32, a warp's */
				for (size_t o = 0; o < back.size(); o += 32)
					append(back.data() + o, (int)std::min<size_t>(32, back.size() - o), (uint32_t)(np + c),
					       seq);
			if ((r == 0 && done) || to || bk.runaway())
				break;
		}
	};
	std::vector<std::thread> ts;
	for (int p = 0; p < np; p++)
		ts.emplace_back(producer, p);
	for (int c = 0; c < nc; c++)
		ts.emplace_back(consumer, c);
	for (auto &t : ts)
		t.join();
	/* the dummy left behind and anything after it */
	uint64_t left = 0, bad = bk.deq.load() > bk.cap ? 1 : 0;
	uint32_t idx = kma_q::tw_idx(ends[0]), lastidx = idx;
	bk.takes[idx]++;
	for (uint32_t nx = kma_q::tw_idx(links[idx]); nx && left <= n; nx = kma_q::tw_idx(links[nx])) {
		bk.takes[nx]++;
		left++;
		lastidx = nx;
	}
	if (lastidx != kma_q::tw_idx(ends[1]))
		bad++;
	for (uint64_t i = 1; i < n + 2; i++)
		if (bk.takes[i] != bk.appends[i])
			bad++;
	R.enq = bk.enq;
	R.deq = bk.deq;
	R.holds = bk.holds;
	R.left = left;
	R.bad = bad;
	R.order = bk.order_bad;
	R.timeouts = bk.tmo;
}

} /* namespace */

/* Stuck queues (a dequeuer that died holding the head, an append that
 * exchanged the tail and never linked): every wait must end, within
 * `limit` tries in which the head did not move, and report the expiry. */
int run_stuck()
{
	const uint32_t limit = 1000;
	bool ok = true;
	{
		Item a{}, b{};
		u64 q[2] = {(u64)&a, (u64)&b};
		a.next = kma_q::POISON; /* held by a dequeuer that is gone */
		b.next = 0;
		(void)b;
		u64 out[4];
		bool to = false;
		uint32_t r = kma_q::clq_dequeue_n<HostOps, LinkAtItem>(&q[0], &q[1], out, 4, limit, &to,
								      (const HostLog *)nullptr);
		printf("{\"case\": \"clq_head_held\", \"taken\": %u, \"timed_out\": %s}\n", r, to ? "true" : "false");
		ok &= r == 0 && to && a.next == kma_q::POISON;
	}
	{
		Item a{}, b{};
		u64 q[2] = {(u64)&a, (u64)&b}; /* b's append exchanged the tail, never linked */
		a.next = 0;
		u64 out[4];
		bool to = false;
		uint32_t r = kma_q::clq_dequeue_n<HostOps, LinkAtItem>(&q[0], &q[1], out, 4, limit, &to,
								      (const HostLog *)nullptr);
		printf("{\"case\": \"clq_append_unlinked\", \"taken\": %u, \"timed_out\": %s}\n", r, to ? "true" : "false");
		ok &= r == 0 && to && a.next == 0 && q[0] == (u64)&a;
	}
	{
		std::vector<u64> links(4, 0);
		IdxQ iq{&links};
		links[1] = kma_q::tw_make(0, 2); /* dummy 1 -> item 2 */
		u64 ends[2] = {kma_q::tw_make(1, 1), kma_q::tw_make(0, 2)}; /* head held (odd tag) */
		uint32_t out[4];
		bool to = false;
		uint32_t r = kma_q::iq_dequeue_n<HostOps>(iq, &ends[0], out, 4, limit, &to, (const HostLog *)nullptr);
		printf("{\"case\": \"iq_head_held\", \"taken\": %u, \"timed_out\": %s}\n", r, to ? "true" : "false");
		ok &= r == 0 && to && ends[0] == kma_q::tw_make(1, 1);
	}
	printf("{\"stuck_ok\": %s}\n", ok ? "true" : "false");
	return ok ? 0 : 1;
}

int main(int argc, char **argv)
{
	if (argc == 2 && strcmp(argv[1], "stuck") == 0)
		return run_stuck();
	if (argc < 8 || argc > 12) {
		fprintf(stderr, "usage: %s clq|iq THREADS CHAINS MAX_CHAIN DEQ_BATCH DELAY_PROB SEED "
			"[PRODUCERS [RECYCLE [LOG_RECORDS [PHASED]]]]\n       %s stuck\n", argv[0], argv[0]);
		return 2;
	}
	const bool clq = strcmp(argv[1], "clq") == 0;
	const int threads = atoi(argv[2]), chains = atoi(argv[3]);
	int maxc = atoi(argv[4]), batch = atoi(argv[5]);
	if (maxc < 0) {
		g_fixed_chain = true;
		maxc = -maxc;
	}
	if (batch < 0) {
		g_fixed_batch = true;
		batch = -batch;
	}
	g_delay_prob = atof(argv[6]);
	const uint64_t seed = strtoull(argv[7], NULL, 0);
	if (argc >= 9)
		g_producers = atoi(argv[8]);
	const double recycle = argc >= 10 ? atof(argv[9]) : 0.5;
	const uint32_t log_records = argc >= 11 ? (uint32_t)strtoul(argv[10], NULL, 0) : 0u;
	g_phased = argc >= 12 && atoi(argv[11]) != 0;
	if (log_records) {
		if (log_records & (log_records - 1))
			return 2; /* a power of two */
		g_log.mask = log_records - 1;
		g_log.clq.assign((size_t)log_records * 32, 0);
		g_log.iq.assign((size_t)log_records * 32, 0);
	}
	if (threads < 1 || chains < 1 || maxc < 1 || batch < 1)
		return 2;
	Result R;
	auto t0 = std::chrono::steady_clock::now();
	if (clq)
		run_clq(threads, chains, maxc, batch, recycle, seed, R);
	else
		run_iq(threads, chains, maxc, batch, recycle, seed, R);
	double s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
	const bool ok = R.bad == 0 && R.order == 0 && R.timeouts == 0;
	printf("{\"queue\": \"%s\", \"log_records\": %u, \"log_chains\": %llu, \"threads\": %d, \"appended\": %llu, \"taken\": %llu, \"left\": %llu, "
	       "\"conservation_faults\": %llu, \"order_faults\": %llu, \"timeouts\": %llu, \"delays\": %llu, "
	       "\"dequeue_calls\": %llu, \"seconds\": %.3f, \"ok\": %s}\n",
	       clq ? "clq" : "iq", log_records, (unsigned long long)g_log.chains.load(), threads, (unsigned long long)R.enq, (unsigned long long)R.deq,
	       (unsigned long long)R.left, (unsigned long long)R.bad, (unsigned long long)R.order,
	       (unsigned long long)R.timeouts, (unsigned long long)g_delays.load(), (unsigned long long)R.holds, s,
	       ok ? "true" : "false");
	return ok ? 0 : 1;
}
