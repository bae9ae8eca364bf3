/*
 * workload.c -- serial and pthread drivers of the C1/C2 per-item programs
 * (see workload.h).  TEST INFRASTRUCTURE ONLY.
 */
#include <stdlib.h>
#include <string.h>
#include <pthread.h>
#include <time.h>
#include "workload.h"

struct wl_item {
	uint64_t rng;
	uint64_t hash;
	uint32_t nlive;
	int64_t off[WL_LIVE_CAP];
	uint32_t size[WL_LIVE_CAP];
};

static void wl_fill(struct wl_heap *hp, int64_t off, uint64_t n, uint32_t tag)
{
	uint32_t *w = (uint32_t *)(hp->base + off);
	uint64_t i;
	for (i = 0; i < n / 4; i++)
		w[i] = tag;
}

static int wl_check(struct wl_heap *hp, int64_t off, uint64_t n, uint32_t tag)
{
	const uint32_t *w = (const uint32_t *)(hp->base + off);
	uint64_t i;
	for (i = 0; i < n / 4; i++)
		if (w[i] != tag)
			return 1;
	return 0;
}

static void wl_c1_round(struct wl_heap *hp, uint64_t gid, struct wl_item *it,
		struct wl_stats *st)
{
	uint64_t n = wl_c1_size(wl_splitmix(&it->rng));
	int64_t off = hp->malloc_fn(hp->h, n);
	st->mallocs++;
	it->hash = wl_hash_step(it->hash, off);
	if (off < 0) {
		st->nulls++;
		return;
	}
	wl_fill(hp, off, n, (uint32_t)gid);
	st->bad_tags += wl_check(hp, off, n, (uint32_t)gid);
	hp->free_fn(hp->h, off);
	st->frees++;
}

static void wl_c2_free_at(struct wl_heap *hp, uint64_t gid, struct wl_item *it,
		uint32_t i, struct wl_stats *st)
{
	st->bad_tags += wl_check(hp, it->off[i], it->size[i], (uint32_t)gid);
	hp->free_fn(hp->h, it->off[i]);
	st->frees++;
}

static void wl_c2_round(struct wl_heap *hp, uint64_t gid, struct wl_item *it,
		struct wl_stats *st)
{
	uint64_t n = wl_c2_size(wl_splitmix(&it->rng));
	uint64_t bits;
	uint32_t i, j;
	int64_t off;

	if (it->nlive == WL_LIVE_CAP) {
		/* table full: retire the oldest entry first */
		wl_c2_free_at(hp, gid, it, 0, st);
		memmove(&it->off[0], &it->off[1], (WL_LIVE_CAP - 1) * sizeof(it->off[0]));
		memmove(&it->size[0], &it->size[1], (WL_LIVE_CAP - 1) * sizeof(it->size[0]));
		it->nlive--;
	}
	off = hp->malloc_fn(hp->h, n);
	st->mallocs++;
	it->hash = wl_hash_step(it->hash, off);
	if (off >= 0) {
		wl_fill(hp, off, n, (uint32_t)gid);
		it->off[it->nlive] = off;
		it->size[it->nlive] = (uint32_t)n;
		it->nlive++;
	} else {
		st->nulls++;
	}
	bits = wl_splitmix(&it->rng);
	for (i = 0, j = 0; i < it->nlive; i++) {
		if ((bits >> i) & 1) {
			wl_c2_free_at(hp, gid, it, i, st);
		} else {
			it->off[j] = it->off[i];
			it->size[j] = it->size[i];
			j++;
		}
	}
	it->nlive = j;
}

static void wl_c2_drain(struct wl_heap *hp, uint64_t gid, struct wl_item *it,
		struct wl_stats *st)
{
	uint32_t i;
	for (i = 0; i < it->nlive; i++)
		wl_c2_free_at(hp, gid, it, i, st);
	it->nlive = 0;
}

static int wl_run_serial(struct wl_heap *hp, uint64_t items, uint32_t rounds,
		uint64_t seed, int round_major, struct wl_stats *st, int c2)
{
	uint64_t g;
	uint32_t r;
	memset(st, 0, sizeof(*st));
	if (!round_major) {
		struct wl_item it;
		for (g = 0; g < items; g++) {
			memset(&it, 0, sizeof(it));
			it.rng = wl_seed(seed, g);
			for (r = 0; r < rounds; r++) {
				if (c2)
					wl_c2_round(hp, g, &it, st);
				else
					wl_c1_round(hp, g, &it, st);
			}
			if (c2)
				wl_c2_drain(hp, g, &it, st);
			st->offset_hash ^= it.hash;
		}
		return 0;
	}
	{
		struct wl_item *its = calloc(items ? items : 1, sizeof(*its));
		if (!its)
			return -1;
		for (g = 0; g < items; g++)
			its[g].rng = wl_seed(seed, g);
		for (r = 0; r < rounds; r++)
			for (g = 0; g < items; g++) {
				if (c2)
					wl_c2_round(hp, g, &its[g], st);
				else
					wl_c1_round(hp, g, &its[g], st);
			}
		for (g = 0; g < items; g++) {
			if (c2)
				wl_c2_drain(hp, g, &its[g], st);
			st->offset_hash ^= its[g].hash;
		}
		free(its);
	}
	return 0;
}

int wl_run_c1_serial(struct wl_heap *hp, uint64_t items, uint32_t rounds,
		uint64_t seed, int round_major, struct wl_stats *st)
{
	return wl_run_serial(hp, items, rounds, seed, round_major, st, 0);
}

int wl_run_c2_serial(struct wl_heap *hp, uint64_t items, uint32_t rounds,
		uint64_t seed, int round_major, struct wl_stats *st)
{
	return wl_run_serial(hp, items, rounds, seed, round_major, st, 1);
}

struct wl_thread_arg {
	struct wl_heap *hp;
	uint64_t items, seed;
	uint32_t rounds;
	unsigned int t, nthreads;
	int c2;
	struct wl_stats st;
};

static void *wl_thread_main(void *p)
{
	struct wl_thread_arg *a = p;
	struct wl_item it;
	uint64_t g;
	uint32_t r;
	memset(&a->st, 0, sizeof(a->st));
	for (g = a->t; g < a->items; g += a->nthreads) {
		memset(&it, 0, sizeof(it));
		it.rng = wl_seed(a->seed, g);
		for (r = 0; r < a->rounds; r++) {
			if (a->c2)
				wl_c2_round(a->hp, g, &it, &a->st);
			else
				wl_c1_round(a->hp, g, &it, &a->st);
		}
		if (a->c2)
			wl_c2_drain(a->hp, g, &it, &a->st);
		a->st.offset_hash ^= it.hash;
	}
	return NULL;
}

static double wl_now(void)
{
	struct timespec ts;
	clock_gettime(CLOCK_MONOTONIC, &ts);
	return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}

static int wl_run_threads(struct wl_heap *hp, uint64_t items, uint32_t rounds,
		uint64_t seed, unsigned int threads, struct wl_stats *st,
		double *seconds, int c2)
{
	struct wl_thread_arg *args;
	pthread_t *tid;
	unsigned int t;
	double t0, t1;

	if (threads == 0)
		threads = 1;
	args = calloc(threads, sizeof(*args));
	tid = calloc(threads, sizeof(*tid));
	if (!args || !tid) {
		free(args);
		free(tid);
		return -1;
	}
	for (t = 0; t < threads; t++) {
		args[t].hp = hp;
		args[t].items = items;
		args[t].seed = seed;
		args[t].rounds = rounds;
		args[t].t = t;
		args[t].nthreads = threads;
		args[t].c2 = c2;
	}
	t0 = wl_now();
	for (t = 0; t < threads; t++)
		pthread_create(&tid[t], NULL, wl_thread_main, &args[t]);
	for (t = 0; t < threads; t++)
		pthread_join(tid[t], NULL);
	t1 = wl_now();
	memset(st, 0, sizeof(*st));
	for (t = 0; t < threads; t++) {
		st->mallocs += args[t].st.mallocs;
		st->frees += args[t].st.frees;
		st->nulls += args[t].st.nulls;
		st->bad_tags += args[t].st.bad_tags;
		st->offset_hash ^= args[t].st.offset_hash;
	}
	if (seconds)
		*seconds = t1 - t0;
	free(args);
	free(tid);
	return 0;
}

int wl_run_c2_threads(struct wl_heap *hp, uint64_t items, uint32_t rounds,
		uint64_t seed, unsigned int threads, struct wl_stats *st,
		double *seconds)
{
	return wl_run_threads(hp, items, rounds, seed, threads, st, seconds, 1);
}

int wl_run_c1_threads(struct wl_heap *hp, uint64_t items, uint32_t rounds,
		uint64_t seed, unsigned int threads, struct wl_stats *st,
		double *seconds)
{
	return wl_run_threads(hp, items, rounds, seed, threads, st, seconds, 0);
}
