/*
 * kma_serve.cu -- the served form (include/kma_serve.h): a host request
 * loop over one device-resident heap.  Each slot owns a CUDA stream and a
 * per-vertex list table; a request runs as build / verify / free kernels
 * on its slot's stream, so requests admitted at different times overlap
 * on the device.  Admission is FIFO and waits for a free slot and for the
 * heap room its estimate needs (reserved bytes <= limit * heap bytes);
 * completion times come from CUDA events on the device timeline.
 */
#include <string.h>
#include <stdlib.h>
#include <math.h>
#include <chrono>
#include <deque>
#include <thread>
#include <vector>

#include "kma_internal.h"
#include "kma_serve.h"
#include "kma_structs.cuh"
#include "kma_wl_common.cuh"

#define SV_MAX_SLOTS 64
#define SV_MAX_CHUNKS 16

namespace {

using namespace kma_wl;

struct sv_params {
	uint32_t n;
	uint32_t deg_max;
	uint64_t seed;
	const uint32_t *deg_cdf;  /* [deg_max] cumulative thresholds of 2^32 */
	const uint32_t *chunks;   /* [nchunks] objects of the k-th page of a list */
	uint32_t nchunks;
	kma_heap *heap;
	kma_clarraylist *lists;   /* [n] */
	unsigned long long *acc;  /* checksum, edges, mallocs, frees, nulls, mismatch */
};

__device__ __forceinline__ uint32_t sv_degree(const sv_params &p, uint64_t d)
{
	uint32_t u = (uint32_t)(d >> 32);
	uint32_t lo = 0, hi = p.deg_max - 1;
	while (lo < hi) {
		uint32_t mid = (lo + hi) >> 1;
		if (u <= __ldg(&p.deg_cdf[mid]))
			hi = mid;
		else
			lo = mid + 1;
	}
	return lo + 1;
}
/* uniform in [0, n) by multiply-shift of the draw's high half */
__device__ __forceinline__ uint32_t sv_neighbour(uint64_t d, uint32_t n)
{
	return (uint32_t)(((d >> 32) * (uint64_t)n) >> 32);
}
__device__ __forceinline__ uint64_t sv_rng0(uint64_t seed, uint32_t v)
{
	return seed ^ ((uint64_t)(v + 1) * 0x9E3779B97F4A7C15ull);
}
__device__ __forceinline__ uint64_t sv_hash_init(uint32_t v, uint32_t d)
{
	return ((uint64_t)(v + 1) * 0xD6E8FEB86659FD93ull) ^ d;
}
__device__ __forceinline__ uint64_t sv_hash_step(uint64_t h, uint32_t nb)
{
	h = (h ^ nb) * 0x9E3779B97F4A7C15ull;
	return h ^ (h >> 29);
}
__device__ __forceinline__ void sv_flush(unsigned long long *acc, int k, unsigned long long v)
{
	for (int d = 16; d > 0; d >>= 1)
		v += __shfl_down_sync(0xffffffffu, v, d);
	if ((threadIdx.x & 31) == 0 && v)
		atomicAdd(&acc[k], v);
}

/* WARP: the pages of a warp's vertices come from one warp-collaborative
 * heap call per step (kma_malloc_warp); otherwise every vertex's thread
 * calls kma_malloc itself (the reference's per-work-item calls, the
 * denominator the served form is measured against). */
template <bool WARP>
__global__ void k_sv_build(sv_params p)
{
	uint32_t v = blockIdx.x * blockDim.x + threadIdx.x;
	bool act = v < p.n;
	uint64_t rng = sv_rng0(p.seed, v);
	uint32_t deg = act ? sv_degree(p, splitmix(rng)) : 0;
	kma_clarraylist *l = act ? &p.lists[v] : nullptr;
	if (act)
		kma_clarraylist_init(l, 4, p.heap, KMA_AL_HEAP_KMA);
	uint32_t written = 0, page = 0;
	unsigned long long mallocs = 0, nulls = 0;
	while (__any_sync(0xffffffffu, written < deg)) {
		uint32_t chunk = 0;
		if (written < deg) {
			chunk = __ldg(&p.chunks[page < p.nchunks ? page : p.nchunks - 1]);
			chunk = chunk < deg - written ? chunk : deg - written;
		}
		/* one warp-collaborative heap call for every lane's page */
		const size_t req = (size_t)chunk * 4 + KMA_AL_PAGE_HDR;
		void *blk = WARP ? kma_malloc_warp(p.heap, chunk ? req : ~(size_t)0)
				 : (chunk ? kma_malloc(p.heap, req) : nullptr);
		if (chunk) {
			mallocs++;
			void *objs = blk ? kma_detail::al_page_init(l, blk, chunk) : nullptr;
			if (!objs) {
				nulls++;
				deg = written; /* give up on this vertex; verify reports it */
			} else {
				uint32_t *o = (uint32_t *)objs;
				for (uint32_t j = 0; j < chunk; j++)
					o[j] = sv_neighbour(splitmix(rng), p.n);
				written += chunk;
				page++;
			}
		}
	}
	sv_flush(p.acc, 2, mallocs);
	sv_flush(p.acc, 4, nulls);
}

__global__ void k_sv_verify(sv_params p)
{
	uint32_t v = blockIdx.x * blockDim.x + threadIdx.x;
	unsigned long long sum = 0, edges = 0, bad = 0;
	if (v < p.n) {
		uint64_t rng = sv_rng0(p.seed, v);
		uint32_t deg = sv_degree(p, splitmix(rng));
		uint64_t h = sv_hash_init(v, deg);
		uint32_t seen = 0;
		unsigned long long pg = kma_detail::qp_ptr(p.lists[v].queue.head);
		while (pg && seen <= deg) {
			uint32_t c = *kma_detail::al_page_count(pg);
			const uint32_t *o = (const uint32_t *)(pg + KMA_AL_PAGE_HDR);
			for (uint32_t j = 0; j < c && seen < deg; j++, seen++) {
				uint32_t nb = o[j];
				if (nb != sv_neighbour(splitmix(rng), p.n))
					bad++;
				h = sv_hash_step(h, nb);
			}
			pg = kma_detail::clq_next<kma_detail::clq_link_aligned>(pg);
		}
		if (seen != deg)
			bad++;
		sum = h;
		edges = seen;
	}
	sv_flush(p.acc, 0, sum);
	sv_flush(p.acc, 1, edges);
	sv_flush(p.acc, 5, bad);
}

template <bool WARP>
__global__ void k_sv_free(sv_params p)
{
	uint32_t v = blockIdx.x * blockDim.x + threadIdx.x;
	unsigned long long frees = 0;
	kma_clarraylist *l = v < p.n ? &p.lists[v] : nullptr;
	bool more = l != nullptr;
	while (__any_sync(0xffffffffu, more)) {
		unsigned long long pg = 0;
		if (more) {
			pg = kma_detail::clq_dequeue<kma_detail::clq_link_aligned>(&l->queue, &l->err, KMA_STRUCT_SPIN);
			more = pg != 0;
		}
		if (WARP)
			kma_free_warp(p.heap, reinterpret_cast<void *>(pg));
		else if (pg)
			kma_free(p.heap, reinterpret_cast<void *>(pg));
		if (pg)
			frees++;
	}
	sv_flush(p.acc, 3, frees);
}

struct sv_slot {
	cudaStream_t st;
	cudaEvent_t end;
	kma_clarraylist *lists;
	unsigned long long *acc;   /* device [8] */
	unsigned long long *host;  /* pinned [8]: acc, then [7] = free superblocks after build */
	int req;
	uint64_t reserved;
};

} /* namespace */

struct kma_serve_s {
	kma_heap_s *heap;
	kma_serve_cfg cfg;
	int mode; /* KMA_MODE_WARP (default) or KMA_MODE_PLAIN */
	uint32_t *deg_cdf;
	uint32_t *chunks;
	uint32_t nchunks;
	double bytes_per_vertex;
	sv_slot slot[SV_MAX_SLOTS];
	unsigned long long *host_all; /* pinned, 8 per slot */
};

static void sv_teardown(kma_serve_s *s)
{
	for (uint32_t i = 0; i < s->cfg.slots; i++) {
		sv_slot &sl = s->slot[i];
		if (sl.end)
			cudaEventDestroy(sl.end);
		if (sl.st)
			cudaStreamDestroy(sl.st);
		if (sl.lists)
			cudaFree(sl.lists);
		if (sl.acc)
			cudaFree(sl.acc);
	}
	if (s->host_all)
		cudaFreeHost(s->host_all);
	if (s->deg_cdf)
		cudaFree(s->deg_cdf);
	if (s->chunks)
		cudaFree(s->chunks);
	free(s);
}

extern "C" int kma_serve_create(kma_heap_t h, const kma_serve_cfg *cfg, kma_serve_t *out)
{
	if (!out)
		return KMA_EINVAL;
	*out = NULL;
	if (!h || !cfg || cfg->slots == 0 || cfg->slots > SV_MAX_SLOTS || cfg->max_vertices == 0 ||
	    cfg->max_vertices > (1u << 28) || cfg->deg_max == 0 || cfg->deg_max > 65535 || !(cfg->gamma > 1.0f) ||
	    !(cfg->occupancy_limit > 0.0f) || cfg->occupancy_limit > 1.0f)
		return KMA_EINVAL;
	uint32_t bd = cfg->block_dim ? cfg->block_dim : 256;
	if (bd % 32 || bd > 1024)
		return KMA_EINVAL;
	kma_device_guard g(h->device);
	kma_serve_s *s = (kma_serve_s *)calloc(1, sizeof(*s));
	if (!s)
		return KMA_ENOMEM;
	s->heap = h;
	s->mode = KMA_MODE_WARP;
	s->cfg = *cfg;
	s->cfg.block_dim = bd;
	/* pages fill their size class: objects = (class bytes - header) / 4 */
	std::vector<uint32_t> chunks, chunk_bytes;
	for (uint32_t c = 0; c < h->hh.nclasses; c++) {
		uint32_t sz = h->hh.cls_size[c];
		if (sz < KMA_AL_PAGE_HDR + 8 * 4)
			continue;
		chunks.push_back((sz - KMA_AL_PAGE_HDR) / 4);
		chunk_bytes.push_back(sz);
		if (chunks.size() == SV_MAX_CHUNKS)
			break;
	}
	if (chunks.empty()) {
		free(s);
		return KMA_EINVAL;
	}
	s->nchunks = (uint32_t)chunks.size();
	/* degree law and the expected heap bytes of one vertex */
	std::vector<double> pd(cfg->deg_max);
	double tot = 0;
	for (uint32_t d = 1; d <= cfg->deg_max; d++)
		tot += (pd[d - 1] = pow((double)d, -(double)cfg->gamma));
	std::vector<uint32_t> cdf(cfg->deg_max);
	double run = 0, bpv = 0;
	for (uint32_t d = 1; d <= cfg->deg_max; d++) {
		double p = pd[d - 1] / tot;
		run += p;
		double t = run * 4294967296.0;
		cdf[d - 1] = d == cfg->deg_max ? 0xffffffffu : (uint32_t)(t >= 4294967295.0 ? 4294967295.0 : t);
		uint64_t left = d, bytes = 0;
		for (uint32_t k = 0; left; k++) {
			uint32_t i = k < s->nchunks ? k : s->nchunks - 1;
			left -= left < chunks[i] ? left : chunks[i];
			bytes += chunk_bytes[i];
		}
		bpv += p * (double)bytes;
	}
	s->bytes_per_vertex = bpv;
	int rc = KMA_OK;
	if (cudaMalloc(&s->deg_cdf, cfg->deg_max * 4) != cudaSuccess ||
	    cudaMalloc(&s->chunks, s->nchunks * 4) != cudaSuccess ||
	    cudaMallocHost(&s->host_all, (size_t)cfg->slots * 8 * 8) != cudaSuccess)
		rc = KMA_ENOMEM;
	if (rc == KMA_OK && (cudaMemcpy(s->deg_cdf, cdf.data(), cfg->deg_max * 4, cudaMemcpyHostToDevice) != cudaSuccess ||
			     cudaMemcpy(s->chunks, chunks.data(), s->nchunks * 4, cudaMemcpyHostToDevice) != cudaSuccess))
		rc = KMA_ECUDA;
	for (uint32_t i = 0; i < cfg->slots && rc == KMA_OK; i++) {
		sv_slot &sl = s->slot[i];
		sl.req = -1;
		sl.host = s->host_all + 8 * i;
		if (cudaStreamCreateWithFlags(&sl.st, cudaStreamNonBlocking) != cudaSuccess ||
		    cudaEventCreateWithFlags(&sl.end, cudaEventDefault) != cudaSuccess)
			rc = KMA_ECUDA;
		else if (cudaMalloc(&sl.lists, (size_t)cfg->max_vertices * sizeof(kma_clarraylist)) != cudaSuccess ||
			 cudaMalloc(&sl.acc, 8 * 8) != cudaSuccess)
			rc = KMA_ENOMEM;
	}
	if (rc != KMA_OK) {
		cudaGetLastError();
		sv_teardown(s);
		return rc;
	}
	*out = s;
	return KMA_OK;
}

extern "C" int kma_serve_destroy(kma_serve_t s)
{
	if (!s)
		return KMA_EINVAL;
	kma_device_guard g(s->heap->device);
	for (uint32_t i = 0; i < s->cfg.slots; i++)
		cudaStreamSynchronize(s->slot[i].st);
	sv_teardown(s);
	return KMA_OK;
}

extern "C" int kma_serve_set_mode(kma_serve_t s, int mode)
{
	if (!s || (mode != KMA_MODE_WARP && mode != KMA_MODE_PLAIN))
		return KMA_EINVAL;
	s->mode = mode;
	return KMA_OK;
}

extern "C" uint64_t kma_serve_estimate(kma_serve_t s, uint32_t n)
{
	if (!s)
		return 0;
	/* expected bytes plus 10% for the spread of a request's degree draws */
	return (uint64_t)(s->bytes_per_vertex * (double)n * 1.10) + (64u << 10);
}

extern "C" int kma_serve_run(kma_serve_t s, const kma_serve_req *reqs, uint32_t n, int realtime,
		kma_serve_result *res, kma_serve_summary *sum)
{
	if (!s || (n && (!reqs || !res)) || !sum)
		return KMA_EINVAL;
	for (uint32_t i = 1; i < n; i++)
		if (reqs[i].arrival_s < reqs[i - 1].arrival_s)
			return KMA_EINVAL;
	kma_device_guard g(s->heap->device);
	memset(sum, 0, sizeof(*sum));
	memset(res, 0, sizeof(*res) * n);
	uint32_t pages = s->heap->hh.pages;
	uint64_t heap_bytes = s->heap->hh.region_bytes;
	const uint64_t limit = (uint64_t)((double)s->cfg.occupancy_limit * (double)heap_bytes);
	const bool ring = (s->heap->hh.flags & KMA_HEAP_RING) != 0;
	const uint32_t bd = s->cfg.block_dim;
	cudaEvent_t t0ev;
	KMA_CUDA(cudaEventCreate(&t0ev));
	KMA_CUDA(cudaEventRecord(t0ev, s->slot[0].st));
	KMA_CUDA(cudaEventSynchronize(t0ev));
	auto t0 = std::chrono::steady_clock::now();
	auto now_s = [&]() {
		return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
	};
	std::deque<uint32_t> waiting;
	uint32_t next = 0, done = 0, running = 0;
	uint64_t reserved = 0, max_reserved = 0;
	bool room_wait = false;
	int rc = KMA_OK;
	double last_done = 0;
	while (done < n && rc == KMA_OK) {
		bool progress = false;
		double t = now_s();
		while (next < n && (!realtime || reqs[next].arrival_s <= t))
			waiting.push_back(next++);
		/* completions */
		for (uint32_t i = 0; i < s->cfg.slots; i++) {
			sv_slot &sl = s->slot[i];
			if (sl.req < 0)
				continue;
			cudaError_t q = cudaEventQuery(sl.end);
			if (q == cudaErrorNotReady)
				continue;
			if (q != cudaSuccess) {
				rc = KMA_ECUDA;
				break;
			}
			kma_serve_result &r = res[sl.req];
			float ms = 0;
			cudaEventElapsedTime(&ms, t0ev, sl.end);
			r.done_s = ms / 1e3;
			r.checksum = sl.host[0];
			r.edges = sl.host[1];
			r.mallocs = sl.host[2];
			r.frees = sl.host[3];
			r.nulls = sl.host[4];
			r.status = sl.host[4] ? KMA_SERVE_NOMEM : (sl.host[5] ? KMA_SERVE_MISMATCH : KMA_SERVE_OK);
			if (ring) {
				uint32_t in_use = pages - (uint32_t)sl.host[7];
				if (in_use > sum->max_sb_in_use && (uint32_t)sl.host[7] <= pages)
					sum->max_sb_in_use = in_use;
			}
			sum->ops += r.mallocs + r.frees;
			last_done = r.done_s > last_done ? r.done_s : last_done;
			reserved -= sl.reserved;
			sl.req = -1;
			running--;
			done++;
			progress = true;
		}
		/* admissions, FIFO */
		while (rc == KMA_OK && !waiting.empty()) {
			uint32_t ri = waiting.front();
			const kma_serve_req &q = reqs[ri];
			uint64_t est = kma_serve_estimate(s, q.n_vertices);
			if (q.n_vertices == 0 || q.n_vertices > s->cfg.max_vertices || est > limit) {
				res[ri].status = KMA_SERVE_TOO_BIG;
				res[ri].admit_s = res[ri].done_s = now_s();
				waiting.pop_front();
				done++;
				progress = true;
				continue;
			}
			int free_slot = -1;
			for (uint32_t i = 0; i < s->cfg.slots; i++)
				if (s->slot[i].req < 0) {
					free_slot = (int)i;
					break;
				}
			if (reserved + est > limit) {
				/* counted once per wait: a slot was free, the room was not */
				if (free_slot >= 0 && !room_wait) {
					sum->admit_waits++;
					room_wait = true;
				}
				break;
			}
			room_wait = false;
			if (free_slot < 0)
				break;
			sv_slot &sl = s->slot[free_slot];
			sv_params p;
			p.n = q.n_vertices;
			p.deg_max = s->cfg.deg_max;
			p.seed = q.seed;
			p.deg_cdf = s->deg_cdf;
			p.chunks = s->chunks;
			p.nchunks = s->nchunks;
			p.heap = s->heap->dh;
			p.lists = sl.lists;
			p.acc = sl.acc;
			uint32_t blocks = (q.n_vertices + bd - 1) / bd;
			if (cudaMemsetAsync(sl.acc, 0, 8 * 8, sl.st) != cudaSuccess) {
				rc = KMA_ECUDA;
				break;
			}
			if (s->mode == KMA_MODE_WARP)
				k_sv_build<true><<<blocks, bd, 0, sl.st>>>(p);
			else
				k_sv_build<false><<<blocks, bd, 0, sl.st>>>(p);
			if (ring)
				cudaMemcpyAsync(&sl.host[7], &s->heap->dh->ring_avail.v, 4, cudaMemcpyDeviceToHost, sl.st);
			k_sv_verify<<<blocks, bd, 0, sl.st>>>(p);
			if (s->mode == KMA_MODE_WARP)
				k_sv_free<true><<<blocks, bd, 0, sl.st>>>(p);
			else
				k_sv_free<false><<<blocks, bd, 0, sl.st>>>(p);
			cudaMemcpyAsync(sl.host, sl.acc, 6 * 8, cudaMemcpyDeviceToHost, sl.st);
			if (cudaGetLastError() != cudaSuccess || cudaEventRecord(sl.end, sl.st) != cudaSuccess) {
				rc = KMA_ECUDA;
				break;
			}
			sl.host[7] = 0;
			sl.req = (int)ri;
			sl.reserved = est;
			reserved += est;
			if (reserved > max_reserved)
				max_reserved = reserved;
			res[ri].admit_s = now_s();
			res[ri].slot = (uint32_t)free_slot;
			res[ri].reserved_bytes = est;
			waiting.pop_front();
			running++;
			if (running > sum->max_running)
				sum->max_running = running;
			progress = true;
		}
		if (!progress) {
			if (running == 0 && waiting.empty() && next < n && realtime) {
				double wait = reqs[next].arrival_s - now_s();
				if (wait > 0)
					std::this_thread::sleep_for(std::chrono::duration<double>(wait < 0.001 ? wait : 0.001));
			} else {
				std::this_thread::sleep_for(std::chrono::microseconds(20));
			}
		}
	}
	for (uint32_t i = 0; i < s->cfg.slots; i++)
		cudaStreamSynchronize(s->slot[i].st);
	cudaEventDestroy(t0ev);
	double first = n ? (realtime ? reqs[0].arrival_s : 0.0) : 0.0;
	sum->wall_s = last_done > first ? last_done - first : 0.0;
	sum->max_occupancy = pages ? (double)sum->max_sb_in_use / (double)pages : 0.0;
	sum->max_reserved = heap_bytes ? (double)max_reserved / (double)heap_bytes : 0.0;
	return rc;
}
