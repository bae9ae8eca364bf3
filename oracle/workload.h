/*
 * workload.h -- the per-work-item stress programs of the KMA workloads, as
 * host C over any heap that exposes malloc/free on offsets.
 *
 * TEST INFRASTRUCTURE ONLY (the oracle side).  The CUDA stress kernels in
 * kma_b200/csrc implement the same programs; under serial execution both
 * must produce the same offsets and the same final heap.
 *
 * Programs (one work-item = one "item" with global id gid):
 *   C1 (kma.cl:424-461 generalised, 16 MiB heap config): per round
 *      n = {8,16,32,64,128,256}[r % 6], malloc(n), write gid into every
 *      32-bit word, verify, free.
 *   C2 (fragmentation config): per round malloc(8 << (r % 9)), tag every
 *      word with gid and keep the block live; then free each live block
 *      whose bit in one 64-bit draw is set (a seeded 50%), verifying its
 *      tags first.  After the last round the live set is drained.
 * PRNG: SplitMix64 seeded with seed ^ (gid * 0x9E3779B97F4A7C15); r below
 * is (draw >> 32).
 */
#ifndef ORACLE_WORKLOAD_H
#define ORACLE_WORKLOAD_H
#include <stdint.h>

typedef int64_t (*wl_malloc_fn)(void *h, uint64_t size);
typedef void (*wl_free_fn)(void *h, int64_t off);

#define WL_LIVE_CAP 32

struct wl_heap {
	void *h;
	wl_malloc_fn malloc_fn;
	wl_free_fn free_fn;
	unsigned char *base;   /* first superblock; payload = base + off */
};

struct wl_stats {
	uint64_t mallocs, frees, nulls, bad_tags;
	uint64_t offset_hash;  /* XOR over items of each item's ordered malloc-result hash */
};

static inline uint64_t wl_splitmix(uint64_t *s)
{
	uint64_t z = (*s += 0x9E3779B97F4A7C15ull);
	z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
	z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
	return z ^ (z >> 31);
}

static inline uint64_t wl_seed(uint64_t seed, uint64_t gid)
{
	return seed ^ (gid * 0x9E3779B97F4A7C15ull);
}

/* Order-dependent fold of one malloc result into the run hash. */
static inline uint64_t wl_hash_step(uint64_t h, int64_t off)
{
	h ^= (uint64_t)off + 0x9E3779B97F4A7C15ull + (h << 6) + (h >> 2);
	return h;
}

/* C1 and C2 size rules */
static inline uint64_t wl_c1_size(uint64_t draw)
{
	static const uint64_t s[6] = { 8, 16, 32, 64, 128, 256 };
	return s[(draw >> 32) % 6];
}
static inline uint64_t wl_c2_size(uint64_t draw)
{
	return 8ull << ((draw >> 32) % 9);
}

#ifdef __cplusplus
extern "C" {
#endif
/* Serial drivers: 0 = item-major (each item runs to completion in gid
 * order), 1 = round-major (every item does round r before any does r+1).
 * Returns 0, or -1 if a scratch allocation failed. */
int wl_run_c1_serial(struct wl_heap *hp, uint64_t items, uint32_t rounds,
		uint64_t seed, int round_major, struct wl_stats *st);
int wl_run_c2_serial(struct wl_heap *hp, uint64_t items, uint32_t rounds,
		uint64_t seed, int round_major, struct wl_stats *st);
/* Threaded driver: items gid = t, t+T, ... on T pthreads, each item to
 * completion (legal: the programs have no barriers).  Wall time of the
 * parallel section in *seconds. */
int wl_run_c2_threads(struct wl_heap *hp, uint64_t items, uint32_t rounds,
		uint64_t seed, unsigned int threads, struct wl_stats *st,
		double *seconds);
int wl_run_c1_threads(struct wl_heap *hp, uint64_t items, uint32_t rounds,
		uint64_t seed, unsigned int threads, struct wl_stats *st,
		double *seconds);
#ifdef __cplusplus
}
#endif
#endif
