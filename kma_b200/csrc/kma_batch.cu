/*
 * kma_batch.cu -- the batched form (include/kma_batch.h): many uneven jobs
 * in one persistent launch on one heap, captured as a CUDA graph, and the
 * autotuner over superblock size x block dim x per-warp cache depth.
 *
 * The persistent kernel walks all jobs' work-items round-major (every item
 * finishes round r before any starts r+1, as if all ran at once; see
 * k_wl_rounds) with every allocation through kma_malloc_warp /
 * kma_free_warp.  A warp's cache keeps up to `depth` freed blocks per size
 * class in shared memory and hands them to the warp's next mallocs of that
 * class; cached blocks stay allocated in the heap, and the warp frees them
 * when the kernel ends.
 *
 * The kernel is a template on the heap (kma_backend.cuh: KMA, or the PMA
 * bump heap, which frees nothing) and on the call style: the
 * warp-collaborative calls, or the plain per-thread malloc / free of the
 * reference on the same job set (the denominator the batched form is
 * measured against).  The warp cache needs the KMA heap's size classes.
 */
#include <string.h>
#include <stdlib.h>
#include <math.h>
#include <vector>

#include "kma_internal.h"
#include "kma_batch.h"
#include "kma_structs.h"
#include "kma_backend.cuh"
#include "kma_wl_common.cuh"

#define BT_CAP 16        /* live blocks a work-item keeps (lifetimes past this retire early) */
#define BT_ZIPF_N 512    /* sizes 8, 16, ..., 4096 */
#define BT_NCLS 16

struct bt_dev {
	uint64_t items;
	uint32_t njobs, rounds;
	const uint64_t *job_first; /* [njobs + 1] first item of each job */
	const uint64_t *job_seed;  /* [njobs] */
	const uint32_t *zipf;      /* [BT_ZIPF_N] cumulative thresholds of 2^32 */
	uint64_t *rng;             /* [items] */
	uint32_t *nlive;           /* [items] */
	uint32_t *off4;            /* [BT_CAP * items] block offset from the heap base / unit (bt_unit) */
	uint32_t *meta;            /* [BT_CAP * items] size/8 | expiry round << 16 */
	unsigned long long *stats; /* kma_batch_stats order */
};

struct kma_batch_s {
	kma_heap_s *heap;  /* KMA heap, or NULL */
	kma_pma_s *pma;    /* PMA heap, or NULL */
	int device;
	int mode;          /* KMA_MODE_WARP (default) or KMA_MODE_PLAIN */
	bt_dev d;
	void *scratch;
	uint64_t items;
	cudaGraph_t graph;
	cudaGraphExec_t exec;
};

namespace {

using namespace kma_wl;

__device__ __forceinline__ uint32_t zipf_size(const uint32_t *cdf, uint64_t d)
{
	uint32_t u = (uint32_t)(d >> 32);
	uint32_t lo = 0, hi = BT_ZIPF_N - 1;
	while (lo < hi) { /* smallest k with u <= cdf[k] */
		uint32_t mid = (lo + hi) >> 1;
		if (u <= __ldg(&cdf[mid]))
			hi = mid;
		else
			lo = mid + 1;
	}
	return 8u * (lo + 1);
}

/* Geometric(1/4) on {1, 2, ...}: the index of the first 2-bit group of a
 * uniform draw that is 00 (each is, with probability 1/4), capped at 32. */
__device__ __forceinline__ uint32_t geom_quarter(uint64_t x)
{
	uint64_t t = ~(x | (x >> 1)) & 0x5555555555555555ull;
	return t ? (uint32_t)(__ffsll((long long)t) - 1) / 2 + 1 : 32u;
}

struct bt_counters {
	uint32_t mallocs, frees, nulls, bad, hits, puts, retired, refused;
	unsigned long long fill, verify;
};

/* per-warp shared memory: cnt[BT_NCLS], hint[BT_NCLS], slot[BT_NCLS][depth] */
struct bt_cache {
	int *cnt;
	uint32_t *slot;
	uint32_t depth;
	uint32_t *hint; /* the warp's kma_malloc_warp hint words */
};

/* Offsets in the live table are 32-bit multiples of the heap's block
 * alignment: 4 bytes (KMA: 16 GiB heaps), 8 (PMA with the jobs' sizes,
 * multiples of 8: 32 GiB). */
template <class B> struct bt_unit;
template <> struct bt_unit<kma_backend_kma> { static constexpr uint32_t shift = 2; };
template <> struct bt_unit<kma_backend_pma> { static constexpr uint32_t shift = 3; };

template <class B>
__device__ __forceinline__ void *bt_block(typename B::heap *h, uint32_t off)
{
	return B::base(h) + ((size_t)off << bt_unit<B>::shift);
}
template <class B>
__device__ __forceinline__ uint32_t bt_off(typename B::heap *h, const void *p)
{
	return (uint32_t)(((const unsigned char *)p - B::base(h)) >> bt_unit<B>::shift);
}
__device__ __forceinline__ uint32_t bt_bytes(uint32_t meta) { return (meta & 0x3ffu) * 8u; }

/* Free q (NULL allowed) of n bytes: into the warp cache when it has room
 * for q's class, else to the heap.  Every lane of the warp calls it. */
template <class B, bool WARP>
__device__ __forceinline__ void bt_free(typename B::heap *h, const bt_cache &cc, uint32_t lane, void *q, uint32_t n,
		bt_counters &ct)
{
	bool keep = false;
	if constexpr (WARP && B::id == KMA_BACKEND_ID_KMA) {
		if (cc.depth && q) {
			int c = kma_class_of(h, n);
			if (c >= 0) {
				int s = atomicAdd(&cc.cnt[c], 1);
				if (s < (int)cc.depth) {
					cc.slot[c * cc.depth + s] = bt_off<B>(h, q);
					keep = true;
					ct.puts++;
				}
			}
		}
		if (cc.depth) {
			__syncwarp();
			if (lane < BT_NCLS && cc.cnt[lane] > (int)cc.depth)
				cc.cnt[lane] = (int)cc.depth;
			__syncwarp();
		}
	}
	if (WARP)
		B::free_block_warp(h, keep ? NULL : q);
	else if (q)
		B::free_block(h, q);
}

/* Malloc n bytes for lanes with `want`: from the warp cache when it holds
 * a block of n's class, else from the heap.  Every lane calls it. */
template <class B, bool WARP>
__device__ __forceinline__ void *bt_malloc(typename B::heap *h, const bt_cache &cc, uint32_t lane, bool want,
		uint32_t n, bt_counters &ct)
{
	void *p = NULL;
	bool need = want;
	if constexpr (WARP && B::id == KMA_BACKEND_ID_KMA) {
		if (cc.depth) {
			if (want) {
				int c = kma_class_of(h, n);
				if (c >= 0) {
					int old = atomicSub(&cc.cnt[c], 1);
					if (old > 0) {
						p = bt_block<B>(h, cc.slot[c * cc.depth + old - 1]);
						need = false;
						ct.hits++;
					}
				}
			}
			__syncwarp();
			if (lane < BT_NCLS && cc.cnt[lane] < 0)
				cc.cnt[lane] = 0;
			__syncwarp();
		}
		void *q = kma_malloc_warp(h, need ? (size_t)n : B::no_request, nullptr, cc.hint);
		return need ? q : p;
	} else if constexpr (WARP) {
		void *q = B::alloc_warp(h, need ? (size_t)n : B::no_request);
		return need ? q : p;
	} else {
		return need ? B::alloc(h, n) : p;
	}
}

/* One round of every lane's item (act = the lane has one). */
template <class B, bool WARP>
__device__ __forceinline__ void bt_round(typename B::heap *h, const bt_dev &w, const bt_cache &cc, uint32_t lane,
		bool act, uint64_t g, uint32_t r, uint64_t &rng, uint32_t &nl, bt_counters &ct)
{
	const uint32_t mask = 0xffffffffu;
	const uint64_t items = w.items;
	const uint32_t tag = (uint32_t)g;
	/* 1. blocks whose lifetime ends now (all of them when r == rounds) */
	uint32_t emask = 0;
	for (uint32_t i = 0; i < (act ? nl : 0u); i++)
		if ((w.meta[(uint64_t)i * items + g] >> 16) <= r || r == w.rounds)
			emask |= 1u << i;
	/* the warp's ending blocks, packed 32 to a pass (warp_pack); each is
	 * verified against its owner's tag by the lane that takes it */
	const warp_pack wp = warp_pack_init(lane, emask);
	for (uint32_t base = 0; base < wp.total; base += 32) {
		uint32_t owner, i;
		const bool mine = warp_pack_slot(wp, lane, base, owner, i);
		const uint64_t o_g = __shfl_sync(mask, g, owner);
		void *q = NULL;
		uint32_t qn = 0;
		if (mine) {
			const uint64_t e = (uint64_t)i * items + o_g;
			q = bt_block<B>(h, w.off4[e]);
			qn = bt_bytes(w.meta[e]);
		}
		if (coop_verify(mask, lane, q, qn, (uint32_t)o_g))
			ct.bad++;
		bt_free<B, WARP>(h, cc, lane, q, qn, ct);
		if (q) {
			ct.frees++;
			ct.verify += qn;
		}
	}
	/* other lanes read this lane's table above; it is compacted next */
	__syncwarp(mask);
	if (emask) {
		uint32_t j = 0;
		for (uint32_t i = 0; i < nl; i++) {
			if ((emask >> i) & 1u)
				continue;
			if (j != i) {
				w.off4[(uint64_t)j * items + g] = w.off4[(uint64_t)i * items + g];
				w.meta[(uint64_t)j * items + g] = w.meta[(uint64_t)i * items + g];
			}
			j++;
		}
		nl = j;
	}
	if (r == w.rounds)
		return;
	/* 2. a full table retires its oldest block */
	bool full = act && nl == BT_CAP;
	if (__any_sync(mask, full)) {
		void *q = NULL;
		uint32_t qn = 0;
		if (full) {
			q = bt_block<B>(h, w.off4[g]);
			qn = bt_bytes(w.meta[g]);
		}
		if (coop_verify(mask, lane, q, qn, tag))
			ct.bad++;
		bt_free<B, WARP>(h, cc, lane, q, qn, ct);
		if (full) {
			ct.frees++;
			ct.retired++;
			ct.verify += qn;
			for (uint32_t i = 1; i < BT_CAP; i++) {
				w.off4[(uint64_t)(i - 1) * items + g] = w.off4[(uint64_t)i * items + g];
				w.meta[(uint64_t)(i - 1) * items + g] = w.meta[(uint64_t)i * items + g];
			}
			nl--;
		}
	}
	/* 3. this round's block */
	uint32_t n = zipf_size(w.zipf, splitmix(rng));
	uint32_t life = geom_quarter(splitmix(rng));
	void *p = bt_malloc<B, WARP>(h, cc, lane, act, n, ct);
	if (act) {
		ct.mallocs++;
		if (p) {
			w.off4[(uint64_t)nl * items + g] = bt_off<B>(h, p);
			w.meta[(uint64_t)nl * items + g] = (n / 8u) | ((r + life) << 16);
			nl++;
			ct.fill += n;
		} else {
			ct.nulls++;
			if (n > B::max_request(h))
				ct.refused++;
		}
	}
	__syncwarp(mask);
	coop_fill(mask, lane, act ? p : NULL, n, tag);
}

template <class B, bool WARP>
__global__ void __launch_bounds__(512, 2) k_bt_rounds(typename B::heap *h, bt_dev w, uint32_t depth)
{
	extern __shared__ int bt_smem[];
	const uint32_t lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
	const uint64_t T = (uint64_t)gridDim.x * blockDim.x;
	const uint64_t tid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
	bt_cache cc;
	cc.depth = depth;
	cc.cnt = bt_smem + wid * (2 * BT_NCLS + BT_NCLS * depth);
	cc.hint = reinterpret_cast<uint32_t *>(cc.cnt + BT_NCLS);
	cc.slot = cc.hint + BT_NCLS;
	if (lane < BT_NCLS) {
		cc.cnt[lane] = 0;
		cc.hint[lane] = 0;
	}
	__syncwarp();
	bt_counters ct = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
	for (uint32_t r = 0; r <= w.rounds; r++) {
		for (uint64_t base = 0; base < w.items; base += T) {
			uint64_t g = base + tid;
			bool act = g < w.items;
			uint64_t rng = act ? w.rng[g] : 0;
			uint32_t nl = act ? w.nlive[g] : 0;
			bt_round<B, WARP>(h, w, cc, lane, act, g, r, rng, nl, ct);
			if (act) {
				w.rng[g] = rng;
				w.nlive[g] = nl;
			}
		}
	}
	/* hand the cached blocks back to the heap */
	if (depth) {
		uint32_t total = BT_NCLS * depth;
		for (uint32_t k0 = 0; k0 < total; k0 += 32) {
			uint32_t k = k0 + lane;
			void *q = NULL;
			if (k < total) {
				uint32_t c = k / depth, s = k % depth;
				if ((int)s < cc.cnt[c])
					q = bt_block<B>(h, cc.slot[c * depth + s]);
			}
			B::free_block_warp(h, q);
		}
	}
	const uint32_t mask = 0xffffffffu;
	unsigned long long v[10] = {__reduce_add_sync(mask, ct.mallocs), __reduce_add_sync(mask, ct.frees),
				    __reduce_add_sync(mask, ct.nulls), __reduce_add_sync(mask, ct.bad), 0, 0,
				    __reduce_add_sync(mask, ct.hits), __reduce_add_sync(mask, ct.puts),
				    __reduce_add_sync(mask, ct.retired), __reduce_add_sync(mask, ct.refused)};
	unsigned long long f = ct.fill, vb = ct.verify;
	for (int d = 16; d > 0; d >>= 1) {
		f += __shfl_down_sync(mask, f, d);
		vb += __shfl_down_sync(mask, vb, d);
	}
	v[4] = f;
	v[5] = vb;
	if (lane == 0)
		for (int k = 0; k < 10; k++)
			if (v[k])
				atomicAdd(&w.stats[k], v[k]);
}

__global__ void k_bt_begin(bt_dev w)
{
	uint64_t T = (uint64_t)gridDim.x * blockDim.x;
	uint64_t tid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (tid < 16)
		w.stats[tid] = 0;
	for (uint64_t g = tid; g < w.items; g += T) {
		uint32_t lo = 0, hi = w.njobs; /* job j: job_first[j] <= g < job_first[j+1] */
		while (hi - lo > 1) {
			uint32_t mid = (lo + hi) >> 1;
			if (w.job_first[mid] <= g)
				lo = mid;
			else
				hi = mid;
		}
		uint64_t local = g - w.job_first[lo];
		w.rng[g] = w.job_seed[lo] ^ (local * 0x9E3779B97F4A7C15ull);
		w.nlive[g] = 0;
	}
}

/* the rounds kernel of b's heap and call style */
const void *bt_kernel(const kma_batch_s *b)
{
	const bool warp = b->mode == KMA_MODE_WARP;
	if (b->pma)
		return warp ? (const void *)k_bt_rounds<kma_backend_pma, true> : (const void *)k_bt_rounds<kma_backend_pma, false>;
	return warp ? (const void *)k_bt_rounds<kma_backend_kma, true> : (const void *)k_bt_rounds<kma_backend_kma, false>;
}

int bt_grid(const kma_batch_s *b, uint32_t bd, uint32_t depth, int device, uint32_t *blocks, size_t *smem)
{
	*smem = (size_t)(bd / 32) * (2 * BT_NCLS + BT_NCLS * depth) * 4;
	int per_sm = 0, sms = 0;
	KMA_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, bt_kernel(b), (int)bd, *smem));
	KMA_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
	*blocks = (uint32_t)((per_sm > 0 ? per_sm : 1) * (sms > 0 ? sms : 1));
	return KMA_OK;
}

int bt_enqueue(kma_batch_t b, uint32_t bd, uint32_t depth, uint32_t blocks, size_t smem, cudaStream_t st)
{
	int rc = b->pma ? kma_pma_reset(b->pma, st) : kma_reset(b->heap, st);
	if (rc != KMA_OK)
		return rc;
	k_bt_begin<<<148 * 4, 256, 0, st>>>(b->d);
	KMA_CUDA(cudaGetLastError());
	const bool warp = b->mode == KMA_MODE_WARP;
	if (b->pma && warp)
		k_bt_rounds<kma_backend_pma, true><<<blocks, bd, smem, st>>>(b->pma->dp, b->d, depth);
	else if (b->pma)
		k_bt_rounds<kma_backend_pma, false><<<blocks, bd, smem, st>>>(b->pma->dp, b->d, depth);
	else if (warp)
		k_bt_rounds<kma_backend_kma, true><<<blocks, bd, smem, st>>>(b->heap->dh, b->d, depth);
	else
		k_bt_rounds<kma_backend_kma, false><<<blocks, bd, smem, st>>>(b->heap->dh, b->d, depth);
	KMA_CUDA(cudaGetLastError());
	return KMA_OK;
}

bool bt_shape_ok(uint32_t bd, uint32_t depth)
{
	return (bd == 128 || bd == 256 || bd == 512) && depth <= KMA_BATCH_MAX_CACHE;
}

bool bt_params_ok(const kma_batch_s *b, uint32_t bd, uint32_t depth)
{
	/* the warp cache keeps blocks by KMA size class */
	if (depth && (b->pma || b->mode != KMA_MODE_WARP))
		return false;
	return bt_shape_ok(bd, depth);
}

int batch_create(kma_heap_s *h, kma_pma_s *pma, const kma_batch_job *jobs, uint32_t njobs, uint32_t rounds,
		kma_batch_t *out);

} /* namespace */

extern "C" int kma_batch_create(kma_heap_t h, const kma_batch_job *jobs, uint32_t njobs, uint32_t rounds,
		kma_batch_t *out)
{
	if (!out)
		return KMA_EINVAL;
	*out = NULL;
	/* block offsets are kept as 32-bit multiples of 4 bytes */
	if (!h || h->hh.region_bytes > (1ull << 34))
		return KMA_EINVAL;
	return batch_create(h, NULL, jobs, njobs, rounds, out);
}

extern "C" int kma_batch_create_pma(kma_pma_t p, const kma_batch_job *jobs, uint32_t njobs, uint32_t rounds,
		kma_batch_t *out)
{
	if (!out)
		return KMA_EINVAL;
	*out = NULL;
	/* 32-bit multiples of 8 bytes (the jobs' sizes keep bump blocks 8-aligned) */
	if (!p || p->bytes > (1ull << 35))
		return KMA_EINVAL;
	return batch_create(NULL, p, jobs, njobs, rounds, out);
}

extern "C" int kma_batch_set_mode(kma_batch_t b, int mode)
{
	if (!b || (mode != KMA_MODE_WARP && mode != KMA_MODE_PLAIN))
		return KMA_EINVAL;
	b->mode = mode;
	return KMA_OK;
}

namespace {
int batch_create(kma_heap_s *h, kma_pma_s *pma, const kma_batch_job *jobs, uint32_t njobs, uint32_t rounds,
		kma_batch_t *out)
{
	if (!jobs || njobs == 0 || njobs > 4096 || rounds == 0 || rounds > 60000)
		return KMA_EINVAL;
	std::vector<uint64_t> first(njobs + 1, 0), seed(njobs);
	for (uint32_t j = 0; j < njobs; j++) {
		first[j + 1] = first[j] + jobs[j].threads;
		seed[j] = jobs[j].seed;
	}
	uint64_t items = first[njobs];
	if (items == 0 || items > (1ull << 31))
		return KMA_EINVAL;
	/* Zipf(1.2) over k = 1..512 (size 8k), cumulative thresholds of 2^32 */
	std::vector<uint32_t> zipf(BT_ZIPF_N);
	{
		double tot = 0, run = 0;
		for (int k = 1; k <= BT_ZIPF_N; k++)
			tot += pow((double)k, -1.2);
		for (int k = 1; k <= BT_ZIPF_N; k++) {
			run += pow((double)k, -1.2);
			double t = run / tot * 4294967296.0;
			zipf[k - 1] = k == BT_ZIPF_N ? 0xffffffffu : (uint32_t)(t >= 4294967295.0 ? 4294967295.0 : t);
		}
	}
	const int device = h ? h->device : pma->device;
	kma_device_guard g(device);
	kma_batch_s *b = (kma_batch_s *)calloc(1, sizeof(*b));
	if (!b)
		return KMA_ENOMEM;
	b->heap = h;
	b->pma = pma;
	b->device = device;
	b->mode = KMA_MODE_WARP;
	b->items = items;
	size_t o_first = 0, o_seed = o_first + (njobs + 1) * 8, o_zipf = o_seed + njobs * 8;
	size_t o_rng = (o_zipf + BT_ZIPF_N * 4 + 255) & ~(size_t)255;
	size_t o_nl = o_rng + items * 8;
	size_t o_off = (o_nl + items * 4 + 255) & ~(size_t)255;
	size_t o_meta = o_off + (size_t)BT_CAP * items * 4;
	size_t o_stats = (o_meta + (size_t)BT_CAP * items * 4 + 255) & ~(size_t)255;
	size_t total = o_stats + 16 * 8;
	if (cudaMalloc(&b->scratch, total) != cudaSuccess) {
		cudaGetLastError();
		free(b);
		return KMA_ENOMEM;
	}
	unsigned char *s = (unsigned char *)b->scratch;
	b->d.items = items;
	b->d.njobs = njobs;
	b->d.rounds = rounds;
	b->d.job_first = (const uint64_t *)(s + o_first);
	b->d.job_seed = (const uint64_t *)(s + o_seed);
	b->d.zipf = (const uint32_t *)(s + o_zipf);
	b->d.rng = (uint64_t *)(s + o_rng);
	b->d.nlive = (uint32_t *)(s + o_nl);
	b->d.off4 = (uint32_t *)(s + o_off);
	b->d.meta = (uint32_t *)(s + o_meta);
	b->d.stats = (unsigned long long *)(s + o_stats);
	if (cudaMemcpy(s + o_first, first.data(), (njobs + 1) * 8, cudaMemcpyHostToDevice) != cudaSuccess ||
	    cudaMemcpy(s + o_seed, seed.data(), njobs * 8, cudaMemcpyHostToDevice) != cudaSuccess ||
	    cudaMemcpy(s + o_zipf, zipf.data(), BT_ZIPF_N * 4, cudaMemcpyHostToDevice) != cudaSuccess ||
	    cudaMemset(s + o_stats, 0, 16 * 8) != cudaSuccess) {
		cudaFree(b->scratch);
		free(b);
		return KMA_ECUDA;
	}
	*out = b;
	return KMA_OK;
}
} /* namespace */

extern "C" int kma_batch_destroy(kma_batch_t b)
{
	if (!b)
		return KMA_EINVAL;
	kma_device_guard g(b->device);
	if (b->exec)
		cudaGraphExecDestroy(b->exec);
	if (b->graph)
		cudaGraphDestroy(b->graph);
	cudaError_t e = cudaFree(b->scratch);
	free(b);
	return e == cudaSuccess ? KMA_OK : KMA_ECUDA;
}

extern "C" uint64_t kma_batch_items(kma_batch_t b) { return b ? b->items : 0; }

extern "C" int kma_batch_run(kma_batch_t b, uint32_t block_dim, uint32_t cache_depth, void *stream)
{
	if (!b)
		return KMA_EINVAL;
	if (block_dim == 0)
		block_dim = 256;
	if (!bt_params_ok(b, block_dim, cache_depth))
		return KMA_EINVAL;
	kma_device_guard g(b->device);
	uint32_t blocks;
	size_t smem;
	int rc = bt_grid(b, block_dim, cache_depth, b->device, &blocks, &smem);
	if (rc != KMA_OK)
		return rc;
	return bt_enqueue(b, block_dim, cache_depth, blocks, smem, kma_stream(stream));
}

extern "C" int kma_batch_capture(kma_batch_t b, uint32_t block_dim, uint32_t cache_depth, void *stream)
{
	if (!b || !stream)
		return KMA_EINVAL;
	if (block_dim == 0)
		block_dim = 256;
	if (!bt_params_ok(b, block_dim, cache_depth))
		return KMA_EINVAL;
	kma_device_guard g(b->device);
	uint32_t blocks;
	size_t smem;
	int rc = bt_grid(b, block_dim, cache_depth, b->device, &blocks, &smem);
	if (rc != KMA_OK)
		return rc;
	if (b->exec) {
		cudaGraphExecDestroy(b->exec);
		b->exec = NULL;
	}
	if (b->graph) {
		cudaGraphDestroy(b->graph);
		b->graph = NULL;
	}
	cudaStream_t st = kma_stream(stream);
	KMA_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
	rc = bt_enqueue(b, block_dim, cache_depth, blocks, smem, st);
	cudaGraph_t graph = NULL;
	cudaError_t e = cudaStreamEndCapture(st, &graph);
	if (rc != KMA_OK || e != cudaSuccess) {
		if (graph)
			cudaGraphDestroy(graph);
		cudaGetLastError();
		return rc != KMA_OK ? rc : KMA_ECUDA;
	}
	if (cudaGraphInstantiate(&b->exec, graph, 0) != cudaSuccess) {
		cudaGraphDestroy(graph);
		cudaGetLastError();
		return KMA_ECUDA;
	}
	b->graph = graph;
	return KMA_OK;
}

extern "C" int kma_batch_launch(kma_batch_t b, void *stream)
{
	if (!b || !b->exec)
		return KMA_EINVAL;
	kma_device_guard g(b->device);
	KMA_CUDA(cudaGraphLaunch(b->exec, kma_stream(stream)));
	return KMA_OK;
}

extern "C" int kma_batch_stats_get(kma_batch_t b, void *stream, kma_batch_stats *out)
{
	if (!b || !out)
		return KMA_EINVAL;
	kma_device_guard g(b->device);
	unsigned long long v[16];
	cudaStream_t st = kma_stream(stream);
	KMA_CUDA(cudaMemcpyAsync(v, b->d.stats, sizeof(v), cudaMemcpyDeviceToHost, st));
	KMA_CUDA(cudaStreamSynchronize(st));
	out->mallocs = v[0];
	out->frees = v[1];
	out->nulls = v[2];
	out->bad_tags = v[3];
	out->fill_bytes = v[4];
	out->verify_bytes = v[5];
	out->cache_hits = v[6];
	out->cache_puts = v[7];
	out->retired = v[8];
	out->refused = v[9];
	return KMA_OK;
}

extern "C" int kma_batch_autotune(const kma_batch_job *jobs, uint32_t njobs, uint32_t rounds, uint64_t heap_bytes,
		uint32_t shards, const uint32_t *sb_log2s, uint32_t n_sb, const uint32_t *block_dims, uint32_t n_bd,
		const uint32_t *depths, uint32_t n_depth, uint32_t warmup, uint32_t reps, int device,
		kma_batch_tune_entry *entries, uint32_t *best)
{
	if (!jobs || !sb_log2s || !block_dims || !depths || !entries || !best || !n_sb || !n_bd || !n_depth ||
	    reps == 0)
		return KMA_EINVAL;
	for (uint32_t i = 0; i < n_sb; i++)
		if (sb_log2s[i] < 12 || sb_log2s[i] > 16 || (heap_bytes >> sb_log2s[i]) == 0 ||
		    (heap_bytes >> sb_log2s[i]) > 0x7fffffffull)
			return KMA_EINVAL;
	for (uint32_t i = 0; i < n_bd; i++)
		for (uint32_t k = 0; k < n_depth; k++)
			if (!bt_shape_ok(block_dims[i], depths[k]))
				return KMA_EINVAL;
	kma_device_guard g(device);
	if (!g.ok)
		return KMA_ENODEV;
	cudaStream_t st;
	KMA_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
	cudaEvent_t e0, e1;
	cudaEventCreate(&e0);
	cudaEventCreate(&e1);
	int rc = KMA_OK;
	uint32_t idx = 0;
	double best_rate = 0;
	*best = 0xffffffffu;
	for (uint32_t i = 0; i < n_sb && rc == KMA_OK; i++) {
		kma_config cfg;
		memset(&cfg, 0, sizeof(cfg));
		cfg.sblocks = (uint32_t)(heap_bytes >> sb_log2s[i]);
		cfg.sb_size_log2 = sb_log2s[i];
		cfg.device = -1;
		cfg.shards = shards;
		kma_heap_t h = NULL;
		rc = kma_create_ex(&cfg, st, &h);
		if (rc != KMA_OK)
			break;
		kma_batch_t b = NULL;
		rc = kma_batch_create(h, jobs, njobs, rounds, &b);
		for (uint32_t j = 0; j < n_bd && rc == KMA_OK; j++) {
			for (uint32_t k = 0; k < n_depth && rc == KMA_OK; k++, idx++) {
				kma_batch_tune_entry *en = &entries[idx];
				memset(en, 0, sizeof(*en));
				en->sb_size_log2 = sb_log2s[i];
				en->block_dim = block_dims[j];
				en->cache_depth = depths[k];
				/* the largest size the jobs draw against the heap's largest request */
				en->serves_all = 8u * BT_ZIPF_N <= h->hh.max_request;
				rc = kma_batch_capture(b, block_dims[j], depths[k], st);
				for (uint32_t w = 0; w < warmup && rc == KMA_OK; w++)
					rc = kma_batch_launch(b, st);
				if (rc != KMA_OK)
					break;
				cudaEventRecord(e0, st);
				for (uint32_t t = 0; t < reps && rc == KMA_OK; t++)
					rc = kma_batch_launch(b, st);
				cudaEventRecord(e1, st);
				if (rc == KMA_OK && cudaEventSynchronize(e1) != cudaSuccess)
					rc = KMA_ECUDA;
				if (rc != KMA_OK)
					break;
				float ms = 0;
				cudaEventElapsedTime(&ms, e0, e1);
				en->ms = ms / reps;
				rc = kma_batch_stats_get(b, st, &en->stats);
				if (rc != KMA_OK)
					break;
				en->mops = (float)((double)(en->stats.mallocs + en->stats.frees) / (en->ms * 1e3));
				uint32_t flags = 0;
				kma_error_flags(h, st, &flags, 1);
				/* rank by successful calls per second: a NULL malloc is
				 * cheap, and a configuration must not win by failing */
				double good = (double)(en->stats.mallocs - en->stats.nulls + en->stats.frees) / en->ms;
				if (en->serves_all && en->stats.bad_tags == 0 && flags == 0 &&
				    (*best == 0xffffffffu || good > best_rate)) {
					*best = idx;
					best_rate = good;
				}
			}
		}
		if (b)
			kma_batch_destroy(b);
		kma_destroy(h);
	}
	cudaEventDestroy(e0);
	cudaEventDestroy(e1);
	cudaStreamDestroy(st);
	return rc;
}
