/*
 * kma_workload.cu -- the stress workloads that drive kma_malloc/kma_free
 * (C ABI kma_wl_* of include/kma.h) and the L2-atomic microbenchmark.
 *
 * The per-work-item programs generalise the reference's test kernels
 * (kma.cl:424-526: malloc, write the item id, free) to the two stress
 * configurations:
 *   C1: per round n = {8,16,32,64,128,256}[draw % 6]: malloc, tag every
 *       32-bit word with the item id, verify, free.
 *   C2: per round malloc(8 << (draw % 9)), tag, keep live; then free each
 *       live block whose bit in a second draw is set (verifying it first).
 * PRNG SplitMix64 seeded seed ^ gid*0x9E3779B97F4A7C15, draw = r >> 32.
 * The same programs, in host C, are the oracle's (oracle/workload.c);
 * serial execution of both yields identical offsets.
 *
 * Concurrent execution: a persistent grid walks the items round by round
 * (k_wl_rounds).  Each lane tags and verifies its own block with 16-byte
 * accesses unrolled by four, so a warp keeps many independent requests in
 * flight (the verify pass is bound by memory latency, not by bandwidth).
 * The per-item state (PRNG, ordered malloc hash, live table) lives in
 * device scratch owned by the kma_wl handle.
 */
#include <string.h>
#include <stdlib.h>
#include <mutex>
#include "kma_internal.h"
#include "kma_wl_common.cuh"

#define WL_CAP 32
/* Counter words behind wl_dev.stats: [0..5] kma_wl_stats counters, [8] the
 * hash XOR of kma_wl_stats_get, [10..13] phase cycles, [16..23] tallies.
 * Every scratch layout reserves this many. */
#define WL_STATS_WORDS 32

struct wl_dev {
	uint64_t items;
	int program;
	uint64_t *rng;
	uint64_t *hash;
	uint32_t *nlive;
	unsigned long long *live_off; /* [WL_CAP * items], offset from sb_base */
	uint32_t *live_size;          /* [WL_CAP * items] */
	unsigned long long *stats;    /* mallocs, frees, nulls, bad_tags, fill, verify bytes */
	uint64_t *seeds;              /* [items] staging for kma_wl_run_host */
};

struct kma_wl_s {
	kma_heap_s *heap;
	wl_dev d;
	void *scratch;
	size_t scratch_bytes;
	unsigned long long *hash_out; /* device u64 for the XOR reduction */
};

namespace {

using namespace kma_wl;

__device__ __forceinline__ uint32_t c1_size(uint64_t d)
{
	const uint32_t r = (uint32_t)((d >> 32) % 6);
	return 8u << r; /* 8,16,32,64,128,256 */
}
__device__ __forceinline__ uint32_t c2_size(uint64_t d) { return 8u << (uint32_t)((d >> 32) % 9); }

/* MODE bit 0: warp-collaborative calls; bit 1 (KMA_MODE_PROFILE): count
 * cycles per phase (malloc, tag fill, verify, free) -- a separate
 * instantiation, so the timed kernels carry none of it. */
template <int MODE>
__device__ __forceinline__ void *wl_malloc(kma_heap *h, size_t n, kma_tally *tl, uint32_t *hint)
{
	return (MODE & KMA_MODE_WARP) ? kma_malloc_warp(h, n, (MODE & KMA_MODE_PROFILE) ? tl : nullptr, hint)
				      : kma_malloc(h, n);
}
template <int MODE>
__device__ __forceinline__ void wl_free(kma_heap *h, void *p)
{
	if (MODE & KMA_MODE_WARP)
		kma_free_warp(h, p);
	else if (p)
		kma_free(h, p);
}

struct wl_counters {
	uint32_t mallocs, frees, nulls, bad, fill, verify;
	unsigned long long cyc[4];
	kma_tally tl;
	uint32_t *hint; /* the warp's kma_malloc_warp hint words (shared memory), or NULL */
};

template <int MODE>
__device__ __forceinline__ void phase(wl_counters &ct, int k, long long &t0)
{
	if (MODE & KMA_MODE_PROFILE) {
		long long t1 = clock64();
		ct.cyc[k] += (unsigned long long)(t1 - t0);
		t0 = t1;
	}
}

/* Per-item state held in registers while an item runs. */
struct wl_item {
	uint64_t rng, hash;
	uint32_t nlive;
};

/* C1 round (every lane in `mask` takes part; act = this lane has an item) */
template <int MODE>
__device__ __forceinline__ void c1_round(kma_heap *h, uint32_t mask, uint32_t lane, bool act, uint64_t g,
		wl_item &it, wl_counters &ct)
{
	uint64_t d = splitmix(it.rng);
	uint32_t n = c1_size(d);
	void *p = NULL;
	if (act) {
		p = wl_malloc<MODE>(h, n, &ct.tl, ct.hint);
		ct.mallocs++;
		it.hash = hash_step(it.hash, p ? (int64_t)((unsigned char *)p - h->sb_base) : -1);
		if (!p)
			ct.nulls++;
	}
	__syncwarp(mask);
	coop_fill(mask, lane, p, n, (uint32_t)g);
	if (coop_verify(mask, lane, p, n, (uint32_t)g))
		ct.bad++;
	wl_free<MODE>(h, p);
	if (p) {
		ct.frees++;
		ct.fill += n;
		ct.verify += n;
	}
}

/* The whole warp's frees of one C2 round (bit i of a lane's fmask: entry
 * i of its live table), packed 32 to a pass (warp_pack); each block is
 * verified against its owner's tag and freed by the lane that takes it. */
template <int MODE>
__device__ __forceinline__ void c2_free_packed(kma_heap *h, const wl_dev &w, uint32_t lane, uint64_t g,
		uint32_t fmask, wl_counters &ct, long long &t0)
{
	const uint32_t full = 0xffffffffu;
	const warp_pack wp = warp_pack_init(lane, fmask);
	for (uint32_t base = 0; base < wp.total; base += 32) {
		uint32_t owner, i;
		const bool mine = warp_pack_slot(wp, lane, base, owner, i);
		const uint64_t o_g = __shfl_sync(full, g, owner);
		void *q = NULL;
		uint32_t qn = 0;
		if (mine) {
			const uint64_t e = (uint64_t)i * w.items + o_g;
			q = h->sb_base + w.live_off[e];
			qn = w.live_size[e];
		}
		if (coop_verify(full, lane, q, qn, (uint32_t)o_g))
			ct.bad++;
		phase<MODE>(ct, 2, t0);
		wl_free<MODE>(h, q);
		phase<MODE>(ct, 3, t0);
		if (q) {
			ct.frees++;
			ct.verify += qn;
		}
	}
	/* other lanes read this lane's live table above; it is compacted next */
	__syncwarp(full);
}

/* C2 round */
template <int MODE>
__device__ __forceinline__ void c2_round(kma_heap *h, const wl_dev &w, uint32_t mask, uint32_t lane, bool act,
		uint64_t g, wl_item &it, wl_counters &ct)
{
	const uint64_t items = w.items;
	long long t0 = (MODE & KMA_MODE_PROFILE) ? clock64() : 0;
	uint64_t d = splitmix(it.rng);
	uint32_t n = c2_size(d);
	uint32_t tag = (uint32_t)g;
	/* table full: retire the oldest entry (never reached in practice) */
	bool full = act && it.nlive == WL_CAP;
	if (__any_sync(mask, full)) {
		void *q = NULL;
		uint32_t qn = 0;
		if (full) {
			q = h->sb_base + w.live_off[g];
			qn = w.live_size[g];
		}
		if (coop_verify(mask, lane, q, qn, tag))
			ct.bad++;
		wl_free<MODE>(h, q);
		if (full) {
			ct.frees++;
			ct.verify += qn;
			for (uint32_t i = 1; i < WL_CAP; i++) {
				w.live_off[(i - 1) * items + g] = w.live_off[i * items + g];
				w.live_size[(i - 1) * items + g] = w.live_size[i * items + g];
			}
			it.nlive--;
		}
	}
	void *p = NULL;
	if (act) {
		p = wl_malloc<MODE>(h, n, &ct.tl, ct.hint);
		ct.mallocs++;
		int64_t off = p ? (int64_t)((unsigned char *)p - h->sb_base) : -1;
		it.hash = hash_step(it.hash, off);
		if (p) {
			w.live_off[(uint64_t)it.nlive * items + g] = (unsigned long long)off;
			w.live_size[(uint64_t)it.nlive * items + g] = n;
			it.nlive++;
			ct.fill += n;
		} else {
			ct.nulls++;
		}
	}
	__syncwarp(mask);
	phase<MODE>(ct, 0, t0);
	coop_fill(mask, lane, p, n, tag);
	phase<MODE>(ct, 1, t0);
	uint64_t bits = splitmix(it.rng);
	uint32_t nl = act ? it.nlive : 0;
	/* live entry i is freed this round when bit i of the draw is set.  A
	 * full warp packs its frees (c2_free_packed); a partial one (the
	 * one-thread serial replay) makes one pass per freed block of its
	 * busiest lane, each lane freeing its entries in increasing i, the
	 * oracle's order */
	uint32_t fmask = nl ? ((uint32_t)bits & (nl >= 32 ? 0xffffffffu : ((1u << nl) - 1u))) : 0u;
	uint32_t npass = mask == 0xffffffffu ? 0u : __reduce_max_sync(mask, (uint32_t)__popc(fmask));
	if (mask == 0xffffffffu)
		c2_free_packed<MODE>(h, w, lane, g, fmask, ct, t0);
	uint32_t rest = fmask;
	for (uint32_t pass = 0; pass < npass; pass++) {
		void *q = NULL;
		uint32_t qn = 0;
		if (rest) {
			uint32_t i = __ffs(rest) - 1;
			rest &= rest - 1;
			q = h->sb_base + w.live_off[(uint64_t)i * items + g];
			qn = w.live_size[(uint64_t)i * items + g];
		}
		if (coop_verify(mask, lane, q, qn, tag))
			ct.bad++;
		phase<MODE>(ct, 2, t0);
		wl_free<MODE>(h, q);
		phase<MODE>(ct, 3, t0);
		if (q) {
			ct.frees++;
			ct.verify += qn;
		}
	}
	if (fmask) {
		/* keep the survivors, in order */
		uint32_t j = 0;
		for (uint32_t i = 0; i < nl; i++) {
			if ((fmask >> i) & 1)
				continue;
			if (j != i) {
				w.live_off[(uint64_t)j * items + g] = w.live_off[(uint64_t)i * items + g];
				w.live_size[(uint64_t)j * items + g] = w.live_size[(uint64_t)i * items + g];
			}
			j++;
		}
		it.nlive = j;
	}
}

template <int MODE>
__device__ __forceinline__ void c2_drain(kma_heap *h, const wl_dev &w, uint32_t mask, uint32_t lane, bool act,
		uint64_t g, wl_item &it, wl_counters &ct)
{
	uint32_t nl = act ? it.nlive : 0;
	uint32_t maxl = __reduce_max_sync(mask, nl);
	for (uint32_t i = 0; i < maxl; i++) {
		void *q = NULL;
		uint32_t qn = 0;
		if (i < nl) {
			q = h->sb_base + w.live_off[(uint64_t)i * w.items + g];
			qn = w.live_size[(uint64_t)i * w.items + g];
		}
		if (coop_verify(mask, lane, q, qn, (uint32_t)g))
			ct.bad++;
		wl_free<MODE>(h, q);
		if (q) {
			ct.frees++;
			ct.verify += qn;
		}
	}
	if (act)
		it.nlive = 0;
}

__device__ __forceinline__ void flush_counters(const wl_dev &w, uint32_t mask, uint32_t lane, const wl_counters &ct)
{
	uint32_t a = __reduce_add_sync(mask, ct.mallocs);
	uint32_t b = __reduce_add_sync(mask, ct.frees);
	uint32_t c = __reduce_add_sync(mask, ct.nulls);
	uint32_t d = __reduce_add_sync(mask, ct.bad);
	unsigned long long e = __reduce_add_sync(mask, ct.fill);
	unsigned long long f = __reduce_add_sync(mask, ct.verify);
	if (lane == (uint32_t)(__ffs(mask) - 1)) {
		for (int k = 0; k < 4; k++)
			if (ct.cyc[k])
				atomicAdd(&w.stats[10 + k], ct.cyc[k]);
	}
	for (int k = 0; k < 8; k++) {
		uint32_t v = __reduce_add_sync(mask, ct.tl.n[k]);
		if (v && lane == (uint32_t)(__ffs(mask) - 1))
			atomicAdd(&w.stats[16 + k], (unsigned long long)v);
	}
	if (lane == (uint32_t)(__ffs(mask) - 1)) {
		if (a) atomicAdd(&w.stats[0], (unsigned long long)a);
		if (b) atomicAdd(&w.stats[1], (unsigned long long)b);
		if (c) atomicAdd(&w.stats[2], (unsigned long long)c);
		if (d) atomicAdd(&w.stats[3], (unsigned long long)d);
		if (e) atomicAdd(&w.stats[4], e);
		if (f) atomicAdd(&w.stats[5], f);
	}
}

/* Persistent, round-major: the grid holds only as many threads as stay
 * resident; when there are more items than threads each thread walks the
 * items g = tid, tid+T, ... inside every round, so every item finishes
 * round r before any starts round r+1 -- as if all of them ran at once.
 * (Launching one thread per item instead lets early waves finish all
 * their rounds and pin their last live blocks while later waves start,
 * which fragments the heap far beyond what concurrent items do.) */
template <int MODE, bool C2>
__global__ void __launch_bounds__(256, 4) k_wl_rounds(kma_heap *h, wl_dev w, uint32_t nrounds, int drain)
{
	const uint32_t mask = 0xffffffffu;
	const uint32_t lane = threadIdx.x & 31;
	const uint64_t T = (uint64_t)gridDim.x * blockDim.x;
	const uint64_t tid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
	__shared__ uint32_t s_hint[256 / 32][KMA_MAX_CLASSES];
	if (lane < KMA_MAX_CLASSES)
		s_hint[threadIdx.x >> 5][lane] = 0;
	__syncwarp();
	wl_counters ct = {0, 0, 0, 0, 0, 0, {0, 0, 0, 0}, {{0, 0, 0, 0, 0, 0, 0, 0}}, s_hint[threadIdx.x >> 5]};
	/* one kernel per program: a kernel carrying both programs' paths
	 * spilled 148 bytes per thread at the 64-register cap, the config-2
	 * one alone 48 */
	const bool c2 = C2;
	{
		for (uint32_t r = 0; r <= nrounds; r++) {
			if (r == nrounds && !(drain && c2))
				break;
			for (uint64_t base = 0; base < w.items; base += T) {
				uint64_t g = base + tid;
				bool act = g < w.items;
				wl_item it;
				it.rng = act ? w.rng[g] : 0;
				it.hash = act ? w.hash[g] : 0;
				it.nlive = act ? w.nlive[g] : 0;
				if (r == nrounds)
					c2_drain<MODE>(h, w, mask, lane, act, g, it, ct);
				else if (c2)
					c2_round<MODE>(h, w, mask, lane, act, g, it, ct);
				else
					c1_round<MODE>(h, mask, lane, act, g, it, ct);
				if (act) {
					w.rng[g] = it.rng;
					w.hash[g] = it.hash;
					w.nlive[g] = it.nlive;
				}
			}
		}
	}
	flush_counters(w, mask, lane, ct);
}

/* The rounds kernel of a call style for a program (config 2, or config 1). */
template <int MODE>
const void *wl_rounds_fn(bool c2)
{
	return c2 ? (const void *)k_wl_rounds<MODE, true> : (const void *)k_wl_rounds<MODE, false>;
}
template <int MODE>
void wl_rounds_launch(bool c2, uint32_t nb, uint32_t bd, cudaStream_t st, kma_heap *h, const wl_dev &d,
		      uint32_t nrounds, int drain)
{
	if (c2)
		k_wl_rounds<MODE, true><<<nb, bd, 0, st>>>(h, d, nrounds, drain);
	else
		k_wl_rounds<MODE, false><<<nb, bd, 0, st>>>(h, d, nrounds, drain);
}

/* One thread runs every item (round_major: round by round). */
template <int MODE>
__global__ void k_wl_serial(kma_heap *h, wl_dev w, uint32_t nrounds, int round_major)
{
	if (blockIdx.x != 0 || threadIdx.x != 0)
		return;
	const uint32_t mask = 1u;
	wl_counters ct = {0, 0, 0, 0, 0, 0, {0, 0, 0, 0}, {{0, 0, 0, 0, 0, 0, 0, 0}}, nullptr};
	if (!round_major) {
		for (uint64_t g = 0; g < w.items; g++) {
			wl_item it = {w.rng[g], w.hash[g], w.nlive[g]};
			for (uint32_t r = 0; r < nrounds; r++) {
				if (w.program == KMA_WL_C1)
					c1_round<MODE>(h, mask, 0, true, g, it, ct);
				else
					c2_round<MODE>(h, w, mask, 0, true, g, it, ct);
			}
			if (w.program == KMA_WL_C2)
				c2_drain<MODE>(h, w, mask, 0, true, g, it, ct);
			w.rng[g] = it.rng;
			w.hash[g] = it.hash;
			w.nlive[g] = it.nlive;
		}
	} else {
		for (uint32_t r = 0; r < nrounds; r++)
			for (uint64_t g = 0; g < w.items; g++) {
				wl_item it = {w.rng[g], w.hash[g], w.nlive[g]};
				if (w.program == KMA_WL_C1)
					c1_round<MODE>(h, mask, 0, true, g, it, ct);
				else
					c2_round<MODE>(h, w, mask, 0, true, g, it, ct);
				w.rng[g] = it.rng;
				w.hash[g] = it.hash;
				w.nlive[g] = it.nlive;
			}
		if (w.program == KMA_WL_C2)
			for (uint64_t g = 0; g < w.items; g++) {
				wl_item it = {w.rng[g], w.hash[g], w.nlive[g]};
				c2_drain<MODE>(h, w, mask, 0, true, g, it, ct);
				w.nlive[g] = it.nlive;
			}
	}
	w.stats[0] += ct.mallocs;
	w.stats[1] += ct.frees;
	w.stats[2] += ct.nulls;
	w.stats[3] += ct.bad;
	w.stats[4] += ct.fill;
	w.stats[5] += ct.verify;
}

__global__ void k_wl_begin(wl_dev w, uint64_t seed, const uint64_t *seeds)
{
	uint64_t g = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (g == 0) {
		for (int i = 0; i < 6; i++)
			w.stats[i] = 0;
		for (int i = 10; i < WL_STATS_WORDS; i++)
			w.stats[i] = 0;
	}
	for (; g < w.items; g += (uint64_t)gridDim.x * blockDim.x) {
		w.rng[g] = seeds ? seeds[g] : (seed ^ (g * 0x9E3779B97F4A7C15ull));
		w.hash[g] = 0;
		w.nlive[g] = 0;
	}
}

__global__ void k_wl_hash_xor(const uint64_t *hash, uint64_t items, unsigned long long *out)
{
	uint64_t x = 0;
	for (uint64_t g = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; g < items;
			g += (uint64_t)gridDim.x * blockDim.x)
		x ^= hash[g];
	uint32_t lo = __reduce_xor_sync(0xffffffffu, (uint32_t)x);
	uint32_t hi = __reduce_xor_sync(0xffffffffu, (uint32_t)(x >> 32));
	if ((threadIdx.x & 31) == 0 && (lo | hi))
		atomicXor(out, ((unsigned long long)hi << 32) | lo);
}

/* atomics microbenchmark: distinct lines or one word */
__global__ void k_atom_distinct(uint32_t *buf, uint64_t lines, uint32_t iters, uint32_t stride, uint32_t *sink)
{
	uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
	uint64_t nt = (uint64_t)gridDim.x * blockDim.x;
	uint32_t acc = 0;
	for (uint32_t i = 0; i < iters; i++) {
		uint64_t line = (t + (uint64_t)i * nt) % lines;
		acc += atomicAdd(buf + line * stride, 1u);
	}
	if (acc == 0x9e3779b9u)
		sink[0] = acc;
}
__global__ void k_atom_same(uint32_t *buf, uint32_t iters, uint32_t *sink)
{
	uint32_t acc = 0;
	for (uint32_t i = 0; i < iters; i++)
		acc += atomicAdd(buf, 1u);
	if (acc == 0x9e3779b9u)
		sink[0] = acc;
}

uint32_t wl_blocks(uint64_t items, uint32_t bd)
{
	uint64_t b = (items + bd - 1) / bd;
	return (uint32_t)(b ? b : 1);
}

} /* namespace */

extern "C" int kma_wl_create(kma_heap_t h, int program, uint64_t items, kma_wl_t *out)
{
	if (!h || !out || items == 0 || (program != KMA_WL_C1 && program != KMA_WL_C2))
		return KMA_EINVAL;
	if (items > (1ull << 32))
		return KMA_EINVAL;
	*out = NULL;
	kma_device_guard g(h->device);
	kma_wl_s *w = (kma_wl_s *)calloc(1, sizeof(*w));
	if (!w)
		return KMA_ENOMEM;
	w->heap = h;
	size_t n = (size_t)items;
	size_t off_rng = 0;
	size_t off_hash = off_rng + 8 * n;
	size_t off_nlive = off_hash + 8 * n;
	size_t off_loff = (off_nlive + 4 * n + 255) & ~(size_t)255;
	size_t off_lsize = off_loff + 8 * n * WL_CAP;
	size_t off_stats = (off_lsize + 4 * n * WL_CAP + 255) & ~(size_t)255;
	size_t off_seeds = off_stats + 8 * WL_STATS_WORDS;
	size_t total = off_seeds + 8 * n;
	if (cudaMalloc(&w->scratch, total) != cudaSuccess) {
		cudaGetLastError();
		free(w);
		return KMA_ENOMEM;
	}
	unsigned char *b = (unsigned char *)w->scratch;
	w->scratch_bytes = total;
	w->d.items = items;
	w->d.program = program;
	w->d.rng = (uint64_t *)(b + off_rng);
	w->d.hash = (uint64_t *)(b + off_hash);
	w->d.nlive = (uint32_t *)(b + off_nlive);
	w->d.live_off = (unsigned long long *)(b + off_loff);
	w->d.live_size = (uint32_t *)(b + off_lsize);
	w->d.stats = (unsigned long long *)(b + off_stats);
	w->d.seeds = (uint64_t *)(b + off_seeds);
	w->hash_out = w->d.stats + 8;
	if (cudaMemset(w->scratch, 0, total) != cudaSuccess) {
		cudaFree(w->scratch);
		free(w);
		return KMA_ECUDA;
	}
	*out = w;
	return KMA_OK;
}

extern "C" int kma_wl_destroy(kma_wl_t w)
{
	if (!w)
		return KMA_EINVAL;
	kma_device_guard g(w->heap->device);
	cudaError_t e = cudaFree(w->scratch);
	free(w);
	return e == cudaSuccess ? KMA_OK : KMA_ECUDA;
}

static int wl_begin(kma_wl_t w, uint64_t seed, const uint64_t *seeds, void *stream)
{
	if (!w)
		return KMA_EINVAL;
	kma_device_guard g(w->heap->device);
	k_wl_begin<<<wl_blocks(w->d.items, 256) < 148 * 8 ? wl_blocks(w->d.items, 256) : 148 * 8, 256, 0,
		kma_stream(stream)>>>(w->d, seed, seeds);
	KMA_CUDA(cudaGetLastError());
	return KMA_OK;
}

extern "C" int kma_wl_begin(kma_wl_t w, uint64_t seed, void *stream) { return wl_begin(w, seed, NULL, stream); }

extern "C" int kma_wl_begin_seeds(kma_wl_t w, const uint64_t *seeds, void *stream)
{
	if (!seeds)
		return KMA_EINVAL;
	return wl_begin(w, 0, seeds, stream);
}

static int wl_launch(kma_wl_t w, uint32_t nrounds, int mode, uint32_t bd, int drain, void *stream)
{
	if (!w || (mode & ~(KMA_MODE_WARP | KMA_MODE_PROFILE)))
		return KMA_EINVAL;
	if (bd == 0)
		bd = 256;
	if (bd % 32 || bd > 256)
		return KMA_EINVAL;
	kma_device_guard g(w->heap->device);
	cudaStream_t st = kma_stream(stream);
	uint32_t nb = wl_blocks(w->d.items, bd);
	/* persistent grid: no more blocks than stay resident on all SMs */
	int per_sm = 0, sms = 0;
	const bool c2 = w->d.program == KMA_WL_C2;
	const void *fns[4] = {wl_rounds_fn<0>(c2), wl_rounds_fn<1>(c2), wl_rounds_fn<2>(c2), wl_rounds_fn<3>(c2)};
	KMA_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fns[mode], (int)bd, 0));
	KMA_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, w->heap->device));
	uint64_t resident = (uint64_t)(per_sm > 0 ? per_sm : 1) * (uint64_t)(sms > 0 ? sms : 1);
	if (nb > resident)
		nb = (uint32_t)resident;
	switch (mode) {
	case 0: wl_rounds_launch<0>(c2, nb, bd, st, w->heap->dh, w->d, nrounds, drain); break;
	case 1: wl_rounds_launch<1>(c2, nb, bd, st, w->heap->dh, w->d, nrounds, drain); break;
	case 2: wl_rounds_launch<2>(c2, nb, bd, st, w->heap->dh, w->d, nrounds, drain); break;
	default: wl_rounds_launch<3>(c2, nb, bd, st, w->heap->dh, w->d, nrounds, drain); break;
	}
	KMA_CUDA(cudaGetLastError());
	return KMA_OK;
}

extern "C" int kma_wl_rounds(kma_wl_t w, uint32_t nrounds, int mode, uint32_t block_dim, void *stream)
{
	return wl_launch(w, nrounds, mode, block_dim, 0, stream);
}

extern "C" int kma_wl_drain(kma_wl_t w, int mode, uint32_t block_dim, void *stream)
{
	if (w && w->d.program != KMA_WL_C2)
		return KMA_OK;
	return wl_launch(w, 0, mode, block_dim, 1, stream);
}

extern "C" int kma_wl_serial(kma_wl_t w, uint32_t nrounds, int round_major, int mode, void *stream)
{
	if (!w || (mode != KMA_MODE_PLAIN && mode != KMA_MODE_WARP))
		return KMA_EINVAL;
	kma_device_guard g(w->heap->device);
	cudaStream_t st = kma_stream(stream);
	if (mode == KMA_MODE_WARP)
		k_wl_serial<KMA_MODE_WARP><<<1, 1, 0, st>>>(w->heap->dh, w->d, nrounds, round_major);
	else
		k_wl_serial<KMA_MODE_PLAIN><<<1, 1, 0, st>>>(w->heap->dh, w->d, nrounds, round_major);
	KMA_CUDA(cudaGetLastError());
	return KMA_OK;
}

extern "C" int kma_wl_stats_get(kma_wl_t w, void *stream, kma_wl_stats *out)
{
	if (!w || !out)
		return KMA_EINVAL;
	kma_device_guard g(w->heap->device);
	cudaStream_t st = kma_stream(stream);
	unsigned long long buf[6], hx = 0;
	KMA_CUDA(cudaMemsetAsync(w->hash_out, 0, 8, st));
	uint32_t nb = wl_blocks(w->d.items, 256);
	k_wl_hash_xor<<<nb < 148 * 4 ? nb : 148 * 4, 256, 0, st>>>(w->d.hash, w->d.items, w->hash_out);
	KMA_CUDA(cudaGetLastError());
	KMA_CUDA(cudaMemcpyAsync(buf, w->d.stats, sizeof(buf), cudaMemcpyDeviceToHost, st));
	KMA_CUDA(cudaMemcpyAsync(&hx, w->hash_out, 8, cudaMemcpyDeviceToHost, st));
	KMA_CUDA(cudaStreamSynchronize(st));
	out->mallocs = buf[0];
	out->frees = buf[1];
	out->nulls = buf[2];
	out->bad_tags = buf[3];
	out->offset_hash = hx;
	out->fill_bytes = buf[4];
	out->verify_bytes = buf[5];
	return KMA_OK;
}

extern "C" int kma_wl_run_host(kma_wl_t w, const uint64_t *seeds_host, uint32_t nrounds, int mode,
		uint64_t *hashes_host, kma_wl_stats *stats, void *stream)
{
	if (!w || !seeds_host)
		return KMA_EINVAL;
	kma_device_guard g(w->heap->device);
	cudaStream_t st = kma_stream(stream);
	int rc = kma_reset(w->heap, stream);
	if (rc != KMA_OK)
		return rc;
	KMA_CUDA(cudaMemcpyAsync(w->d.seeds, seeds_host, (size_t)w->d.items * 8, cudaMemcpyHostToDevice, st));
	rc = wl_begin(w, 0, w->d.seeds, stream);
	if (rc == KMA_OK)
		rc = wl_launch(w, nrounds, mode, 0, 1, stream);
	if (rc != KMA_OK)
		return rc;
	if (hashes_host)
		KMA_CUDA(cudaMemcpyAsync(hashes_host, w->d.hash, (size_t)w->d.items * 8, cudaMemcpyDeviceToHost, st));
	if (stats)
		return kma_wl_stats_get(w, stream, stats);
	KMA_CUDA(cudaStreamSynchronize(st));
	return KMA_OK;
}

extern "C" const uint64_t *kma_wl_item_hashes(kma_wl_t w) { return w ? w->d.hash : NULL; }

extern "C" int kma_wl_live(kma_wl_t w, void *stream, uint32_t *nlive, uint64_t *off, uint32_t *size)
{
	if (!w)
		return KMA_EINVAL;
	kma_device_guard g(w->heap->device);
	cudaStream_t st = kma_stream(stream);
	size_t n = (size_t)w->d.items;
	if (nlive)
		KMA_CUDA(cudaMemcpyAsync(nlive, w->d.nlive, n * 4, cudaMemcpyDeviceToHost, st));
	if (off)
		KMA_CUDA(cudaMemcpyAsync(off, w->d.live_off, n * 8 * WL_CAP, cudaMemcpyDeviceToHost, st));
	if (size)
		KMA_CUDA(cudaMemcpyAsync(size, w->d.live_size, n * 4 * WL_CAP, cudaMemcpyDeviceToHost, st));
	KMA_CUDA(cudaStreamSynchronize(st));
	return KMA_OK;
}

extern "C" int kma_bench_atomics(int distinct, uint64_t threads, uint32_t iters, uint32_t stride_words,
		void *stream, float *ms)
{
	if (!ms || threads == 0 || threads % 256 || iters == 0)
		return KMA_EINVAL;
	if (stride_words == 0)
		stride_words = 32;
	const uint64_t lines = 1ull << 19; /* 512 Ki lines: 64 MiB at 128 B, inside L2 */
	size_t bytes = distinct ? (size_t)(lines * stride_words * 4) : 256;
	uint32_t *buf = NULL;
	cudaStream_t st = kma_stream(stream);
	if (cudaMalloc(&buf, bytes + 256) != cudaSuccess) {
		cudaGetLastError();
		return KMA_ENOMEM;
	}
	cudaEvent_t e0, e1;
	cudaEventCreate(&e0);
	cudaEventCreate(&e1);
	int rc = KMA_OK;
	uint32_t *sink = (uint32_t *)((unsigned char *)buf + bytes);
	if (cudaMemsetAsync(buf, 0, bytes + 256, st) != cudaSuccess)
		rc = KMA_ECUDA;
	unsigned nb = (unsigned)(threads / 256);
	/* warm-up launch, then the timed one */
	for (int rep = 0; rep < 2 && rc == KMA_OK; rep++) {
		if (rep == 1)
			cudaEventRecord(e0, st);
		if (distinct)
			k_atom_distinct<<<nb, 256, 0, st>>>(buf, lines, iters, stride_words, sink);
		else
			k_atom_same<<<nb, 256, 0, st>>>(buf, iters, sink);
		if (rep == 1)
			cudaEventRecord(e1, st);
		if (cudaGetLastError() != cudaSuccess)
			rc = KMA_ECUDA;
	}
	if (rc == KMA_OK && cudaEventSynchronize(e1) != cudaSuccess)
		rc = KMA_ECUDA;
	if (rc == KMA_OK)
		cudaEventElapsedTime(ms, e0, e1);
	cudaEventDestroy(e0);
	cudaEventDestroy(e1);
	cudaFree(buf);
	return rc;
}

/* ------------------------------------------------------------------ */
/* allocation-free workload run (kma_wl_run_noalloc)                   */
/* ------------------------------------------------------------------ */
/* Some hosts cannot call cudaMalloc when they run a batch: cudaMalloc and
 * cudaFree synchronise with the whole device (stalling every other stream
 * a serving loop keeps busy), and a host framework with its own caching
 * allocator (PyTorch's, say) may own the device memory budget so that a
 * private cudaMalloc fails or fragments its pool.  For them this entry
 * point runs the workload on scratch that lives in this file-scope array
 * instead of the kma_wl handle's cudaMalloc'd scratch.  The array is part
 * of the library's device image: every GPU that loads the library holds
 * its 4 MiB until the process exits, and every call shares it. */
static __device__ __align__(256) unsigned char kma_noalloc_scratch[KMA_WL_NOALLOC_SCRATCH_BYTES];

namespace {

/* Device address of kma_noalloc_scratch per device.  In host code the
 * array's name is only a host-side stand-in, so the address comes from
 * cudaGetSymbolAddress, once per device, with that device current. */
struct noalloc_slot {
	void *ptr;
	bool ready;
};
std::mutex g_noalloc_mu;
noalloc_slot g_noalloc[256];

int noalloc_scratch(int dev, unsigned char **out)
{
	if (dev < 0 || dev >= 256)
		return KMA_ENODEV;
	std::lock_guard<std::mutex> lk(g_noalloc_mu);
	if (!g_noalloc[dev].ready) {
		void *p = NULL;
		if (cudaGetSymbolAddress(&p, kma_noalloc_scratch) != cudaSuccess || !p) {
			cudaGetLastError();
			return KMA_ECUDA;
		}
		g_noalloc[dev].ptr = p;
		g_noalloc[dev].ready = true;
	}
	*out = (unsigned char *)g_noalloc[dev].ptr;
	return KMA_OK;
}

size_t up256(size_t x) { return (x + 255) & ~(size_t)255; }

/* Counters and the XOR of the per-item hashes into the caller's
 * kma_wl_stats (one block). */
__global__ void k_noalloc_finish(const unsigned long long *stats, const uint64_t *hash, uint64_t items,
		kma_wl_stats *out)
{
	__shared__ unsigned long long part[32];
	uint64_t x = 0;
	for (uint64_t g = threadIdx.x; g < items; g += blockDim.x)
		x ^= hash[g];
	uint32_t lo = __reduce_xor_sync(0xffffffffu, (uint32_t)x);
	uint32_t hi = __reduce_xor_sync(0xffffffffu, (uint32_t)(x >> 32));
	if ((threadIdx.x & 31) == 0)
		part[threadIdx.x / 32] = ((unsigned long long)hi << 32) | lo;
	__syncthreads();
	if (threadIdx.x == 0) {
		unsigned long long h = 0;
		for (uint32_t i = 0; i < blockDim.x / 32; i++)
			h ^= part[i];
		out->mallocs = stats[0];
		out->frees = stats[1];
		out->nulls = stats[2];
		out->bad_tags = stats[3];
		out->offset_hash = h;
		out->fill_bytes = stats[4];
		out->verify_bytes = stats[5];
	}
}

} /* namespace */

extern "C" int kma_wl_run_noalloc(kma_heap_t h, int program, uint64_t items, const uint64_t *seeds_dev,
		uint32_t nrounds, int mode, int serial, uint64_t *hashes_dev, kma_wl_stats *stats_dev,
		void *stream)
{
	if (!h || !seeds_dev || !hashes_dev || !stats_dev || items == 0)
		return KMA_EINVAL;
	if (items > KMA_WL_NOALLOC_MAX_ITEMS)
		return KMA_EINVAL; /* the fixed scratch holds at most this many items */
	if (program != KMA_WL_C1 && program != KMA_WL_C2)
		return KMA_EINVAL;
	if (mode != KMA_MODE_PLAIN && mode != KMA_MODE_WARP)
		return KMA_EINVAL;
	kma_device_guard g(h->device);
	if (!g.ok)
		return KMA_ENODEV;
	unsigned char *base = NULL;
	int rc = noalloc_scratch(h->device, &base);
	if (rc != KMA_OK)
		return rc;
	size_t n = (size_t)items;
	size_t o_rng = 0;
	size_t o_nlive = up256(o_rng + 8 * n);
	size_t o_loff = up256(o_nlive + 4 * n);
	size_t o_lsize = up256(o_loff + 8 * n * WL_CAP);
	size_t o_stats = up256(o_lsize + 4 * n * WL_CAP);
	if (o_stats + 8 * WL_STATS_WORDS > sizeof(kma_noalloc_scratch))
		return KMA_EINVAL;
	wl_dev d;
	d.items = items;
	d.program = program;
	d.rng = (uint64_t *)(base + o_rng);
	d.hash = hashes_dev; /* the per-item hashes are the caller's output */
	d.nlive = (uint32_t *)(base + o_nlive);
	d.live_off = (unsigned long long *)(base + o_loff);
	d.live_size = (uint32_t *)(base + o_lsize);
	d.stats = (unsigned long long *)(base + o_stats);
	d.seeds = NULL;
	cudaStream_t st = kma_stream(stream);
	rc = kma_reset(h, stream);
	if (rc != KMA_OK)
		return rc;
	/* k_wl_begin clears what must start at zero: each item's hash and live
	 * count and the counters; the array keeps the previous call's data */
	uint32_t bb = wl_blocks(items, 256);
	k_wl_begin<<<bb < 148 * 8 ? bb : 148 * 8, 256, 0, st>>>(d, 0, seeds_dev);
	if (serial) {
		if (mode == KMA_MODE_WARP)
			k_wl_serial<KMA_MODE_WARP><<<1, 1, 0, st>>>(h->dh, d, nrounds, 1);
		else
			k_wl_serial<KMA_MODE_PLAIN><<<1, 1, 0, st>>>(h->dh, d, nrounds, 1);
	} else {
		uint32_t nb = wl_blocks(items, 256);
		int per_sm = 0, sms = 0;
		const bool c2 = d.program == KMA_WL_C2;
		const void *fn = mode == KMA_MODE_WARP ? wl_rounds_fn<KMA_MODE_WARP>(c2) : wl_rounds_fn<KMA_MODE_PLAIN>(c2);
		KMA_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, 256, 0));
		KMA_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, h->device));
		uint64_t resident = (uint64_t)(per_sm > 0 ? per_sm : 1) * (uint64_t)(sms > 0 ? sms : 1);
		if (nb > resident)
			nb = (uint32_t)resident;
		if (mode == KMA_MODE_WARP)
			wl_rounds_launch<KMA_MODE_WARP>(c2, nb, 256, st, h->dh, d, nrounds, 1);
		else
			wl_rounds_launch<KMA_MODE_PLAIN>(c2, nb, 256, st, h->dh, d, nrounds, 1);
	}
	k_noalloc_finish<<<1, 1024, 0, st>>>(d.stats, hashes_dev, items, stats_dev);
	KMA_CUDA(cudaGetLastError());
	return KMA_OK;
}

extern "C" int kma_wl_phase_cycles(kma_wl_t w, void *stream, uint64_t cycles[4])
{
	if (!w || !cycles)
		return KMA_EINVAL;
	kma_device_guard g(w->heap->device);
	cudaStream_t st = kma_stream(stream);
	KMA_CUDA(cudaMemcpyAsync(cycles, w->d.stats + 10, 32, cudaMemcpyDeviceToHost, st));
	KMA_CUDA(cudaStreamSynchronize(st));
	return KMA_OK;
}

extern "C" int kma_wl_tally(kma_wl_t w, void *stream, uint64_t counts[8])
{
	if (!w || !counts)
		return KMA_EINVAL;
	kma_device_guard g(w->heap->device);
	cudaStream_t st = kma_stream(stream);
	KMA_CUDA(cudaMemcpyAsync(counts, w->d.stats + 16, 64, cudaMemcpyDeviceToHost, st));
	KMA_CUDA(cudaStreamSynchronize(st));
	return KMA_OK;
}
