/*
 * kma_structs.cu -- host side of the lock-free structures and the PMA bump
 * heap: create/destroy (the reference's clQueue_create, clIndexedQueue_create,
 * clArrayList_create, pma_create), one-thread replays for parity, and the
 * config-3 concurrent microbenchmarks.
 */
#include <cuda_runtime.h>
#include <stdlib.h>
#include <string.h>
#include <algorithm>
#include <vector>

#include "kma_internal.h"
#include "kma_structs.h"
#include "kma_structs.cuh"
#include "kma_backend.cuh"

struct kma_clqueue_s {
	int device;
	kma_clqueue *dq;
};
struct kma_iqueue_s {
	int device;
	void *mem;
	kma_iqueue *dq;
};
struct kma_chain_log_s {
	int device;
	void *mem;
	kma_chain_log *dl;
};
struct kma_cltree_s {
	int device;
	kma_cltree *dt;
};
struct kma_clarraylist_s {
	int device;
	kma_clarraylist *dl;
};

namespace {

/* Copy a host-built object to the device and wait for it (creation is not
 * on any hot path, and the source is a stack object). */
int put_sync(void *dst, const void *src, size_t n, cudaStream_t st)
{
	KMA_CUDA(cudaMemcpyAsync(dst, src, n, cudaMemcpyHostToDevice, st));
	KMA_CUDA(cudaStreamSynchronize(st));
	return KMA_OK;
}

/* Temporary device buffers of a host call, freed on every return path. */
struct dev_bufs {
	std::vector<void *> v;
	~dev_bufs()
	{
		for (void *p : v)
			cudaFree(p);
	}
	template <typename T>
	T *alloc(size_t bytes)
	{
		void *p = NULL;
		if (cudaMalloc(&p, bytes ? bytes : 1) != cudaSuccess) {
			cudaGetLastError();
			return NULL;
		}
		v.push_back(p);
		return (T *)p;
	}
};

int current_device()
{
	int d = 0;
	cudaGetDevice(&d);
	return d;
}

} /* namespace */

/* ------------------------------------------------------------------ */
/* PMA                                                                 */
/* ------------------------------------------------------------------ */

extern "C" int kma_pma_create(uint64_t bytes, int device, void *stream, kma_pma_t *out)
{
	if (!out)
		return KMA_EINVAL;
	*out = NULL;
	if (bytes == 0 || bytes > (1ull << 46))
		return KMA_EINVAL;
	kma_device_guard g(device);
	if (!g.ok)
		return KMA_ENODEV;
	kma_pma_s *p = (kma_pma_s *)calloc(1, sizeof(*p));
	if (!p)
		return KMA_ENOMEM;
	p->device = current_device();
	size_t hdr = (sizeof(kma_pma) + 255) & ~(size_t)255;
	/* data + the reference's 24-byte limit slack, rounded to 16 */
	size_t total = hdr + ((bytes + KMA_PMA_REF_HEADER + 15) & ~15ull);
	if (cudaMalloc(&p->mem, total) != cudaSuccess) {
		cudaGetLastError();
		free(p);
		return KMA_ENOMEM;
	}
	p->dp = (kma_pma *)p->mem;
	p->base = (unsigned char *)p->mem + hdr;
	p->bytes = bytes;
	kma_pma hp;
	memset(&hp, 0, sizeof(hp));
	hp.bytes = bytes + KMA_PMA_REF_HEADER;
	hp.base = p->base;
	int rc = put_sync(p->dp, &hp, sizeof(hp), kma_stream(stream));
	if (rc != KMA_OK) {
		cudaFree(p->mem);
		free(p);
		return rc;
	}
	*out = p;
	return KMA_OK;
}

extern "C" int kma_pma_destroy(kma_pma_t p)
{
	if (!p)
		return KMA_EINVAL;
	kma_device_guard g(p->device);
	cudaError_t e = cudaFree(p->mem);
	free(p);
	return e == cudaSuccess ? KMA_OK : KMA_ECUDA;
}

extern "C" struct kma_pma *kma_pma_device_ptr(kma_pma_t p) { return p ? p->dp : NULL; }
extern "C" void *kma_pma_base(kma_pma_t p) { return p ? p->base : NULL; }

extern "C" int kma_pma_reset(kma_pma_t p, void *stream)
{
	if (!p)
		return KMA_EINVAL;
	kma_device_guard g(p->device);
	KMA_CUDA(cudaMemsetAsync(&p->dp->head.v, 0, 8, kma_stream(stream)));
	return KMA_OK;
}

extern "C" int kma_pma_head(kma_pma_t p, void *stream, uint64_t *head)
{
	if (!p || !head)
		return KMA_EINVAL;
	kma_device_guard g(p->device);
	cudaStream_t st = kma_stream(stream);
	KMA_CUDA(cudaMemcpyAsync(head, &p->dp->head.v, 8, cudaMemcpyDeviceToHost, st));
	KMA_CUDA(cudaStreamSynchronize(st));
	return KMA_OK;
}

namespace {
} /* namespace */

/* run a one-thread replay kernel over host op/out arrays */
template <typename F>
static int replay_host(int64_t n, const int64_t *ops, int64_t *out, F launch)
{
	if (n < 0 || (n && (!ops || !out)))
		return KMA_EINVAL;
	dev_bufs b;
	int64_t *dops = b.alloc<int64_t>((size_t)n * 16), *dout = b.alloc<int64_t>((size_t)n * 8);
	if (!dops || !dout)
		return KMA_ENOMEM;
	if (n)
		KMA_CUDA(cudaMemcpy(dops, ops, (size_t)n * 16, cudaMemcpyHostToDevice));
	int rc = launch(dops, dout);
	if (rc != KMA_OK)
		return rc;
	KMA_CUDA(cudaGetLastError());
	KMA_CUDA(cudaDeviceSynchronize());
	if (n)
		KMA_CUDA(cudaMemcpy(out, dout, (size_t)n * 8, cudaMemcpyDeviceToHost));
	return KMA_OK;
}

extern "C" int kma_pma_replay_host(kma_pma_t p, const int64_t *ops, int64_t n, int64_t *out)
{
	if (!p)
		return KMA_EINVAL;
	kma_device_guard g(p->device);
	return replay_host(n, ops, out, [&](const int64_t *dops, int64_t *dout) {
		kma_k_heap_replay<kma_backend_pma><<<1, 1>>>(p->dp, dops, n, dout, 0);
		return KMA_OK;
	});
}

/* ------------------------------------------------------------------ */
/* clQueue                                                             */
/* ------------------------------------------------------------------ */

extern "C" int kma_clqueue_create(int device, void *stream, kma_clqueue_t *out)
{
	if (!out)
		return KMA_EINVAL;
	*out = NULL;
	kma_device_guard g(device);
	if (!g.ok)
		return KMA_ENODEV;
	kma_clqueue_s *q = (kma_clqueue_s *)calloc(1, sizeof(*q));
	if (!q)
		return KMA_ENOMEM;
	q->device = current_device();
	/* a line of its own: head and tail are the contended words */
	if (cudaMalloc(&q->dq, 128) != cudaSuccess) {
		cudaGetLastError();
		free(q);
		return KMA_ENOMEM;
	}
	if (cudaMemsetAsync(q->dq, 0, 128, kma_stream(stream)) != cudaSuccess ||
	    cudaStreamSynchronize(kma_stream(stream)) != cudaSuccess) {
		cudaFree(q->dq);
		free(q);
		return KMA_ECUDA;
	}
	*out = q;
	return KMA_OK;
}

extern "C" int kma_clqueue_destroy(kma_clqueue_t q)
{
	if (!q)
		return KMA_EINVAL;
	kma_device_guard g(q->device);
	cudaError_t e = cudaFree(q->dq);
	free(q);
	return e == cudaSuccess ? KMA_OK : KMA_ECUDA;
}

extern "C" struct kma_clqueue *kma_clqueue_device_ptr(kma_clqueue_t q) { return q ? q->dq : NULL; }

namespace {
constexpr uint32_t QITEM = 16; /* {link u64, payload u32, pad u32} */

__device__ int64_t q_index(const unsigned char *items, unsigned long long p)
{
	if (p == 0)
		return -1;
	if (p == KMA_Q_POISON)
		return -2;
	return (int64_t)((p - (unsigned long long)items) / QITEM);
}

__global__ void k_clq_replay(kma_clqueue *q, unsigned char *items, uint32_t n_items, const int64_t *ops,
		int64_t n, int64_t *out, int64_t *fin, uint32_t *err)
{
	for (int64_t i = 0; i < n; i++) {
		int64_t kind = ops[2 * i], arg = ops[2 * i + 1];
		if (kind == 0) {
			out[i] = (arg >= 0 && arg < n_items)
				? kma_clqueue_enqueue(q, (kma_clqueue_item *)(items + (size_t)arg * QITEM), err)
				: 0;
		} else {
			kma_clqueue_item *p = kma_clqueue_dequeue(q, err);
			out[i] = q_index(items, (unsigned long long)p);
		}
	}
	fin[0] = q_index(items, kma_detail::qp_ptr(q->head));
	fin[1] = q_index(items, kma_detail::qp_ptr(q->tail));
	for (uint32_t k = 0; k < n_items; k++)
		fin[2 + k] = q_index(items, ((kma_clqueue_item *)(items + (size_t)k * QITEM))->next);
}
} /* namespace */

extern "C" int kma_clqueue_replay_host(uint32_t n_items, const int64_t *ops, int64_t n, int64_t *out,
		int64_t *final_state)
{
	if (!final_state || n_items == 0)
		return KMA_EINVAL;
	kma_clqueue_t q;
	int rc = kma_clqueue_create(-1, NULL, &q);
	if (rc != KMA_OK)
		return rc;
	dev_bufs b;
	unsigned char *items = b.alloc<unsigned char>((size_t)n_items * QITEM);
	int64_t *dfin = b.alloc<int64_t>((size_t)(n_items + 2) * 8);
	uint32_t *derr = b.alloc<uint32_t>(4);
	if (!items || !dfin || !derr) {
		kma_clqueue_destroy(q);
		return KMA_ENOMEM;
	}
	cudaMemset(items, 0, (size_t)n_items * QITEM);
	cudaMemset(derr, 0, 4);
	rc = replay_host(n, ops, out, [&](const int64_t *dops, int64_t *dout) {
		k_clq_replay<<<1, 1>>>(q->dq, items, n_items, dops, n, dout, dfin, derr);
		return KMA_OK;
	});
	if (rc == KMA_OK && cudaMemcpy(final_state, dfin, (size_t)(n_items + 2) * 8, cudaMemcpyDeviceToHost) != cudaSuccess)
		rc = KMA_ECUDA;
	uint32_t err = 0;
	if (rc == KMA_OK && cudaMemcpy(&err, derr, 4, cudaMemcpyDeviceToHost) == cudaSuccess && err)
		rc = KMA_ETIMEDOUT;
	kma_clqueue_destroy(q);
	return rc;
}

/* ------------------------------------------------------------------ */
/* clIndexedQueue                                                      */
/* ------------------------------------------------------------------ */

namespace {
__global__ void k_iq_init(kma_iqueue *q, uint32_t first_idx)
{
	uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
	if (s >= q->nshards)
		return;
	/* shard 0 starts on `first`, shard s > 0 on internal dummy capacity + s */
	uint32_t d = s == 0 ? first_idx : q->capacity + s;
	*kma_detail::iq_link(q, d) = 0ull;
	q->ends[2 * s].v = kma_detail::tw_make(0, d);
	q->ends[2 * s + 1].v = kma_detail::tw_make(0, d);
}
} /* namespace */

extern "C" int kma_iqueue_create(void *base, uint32_t stride_l2, uint32_t capacity, void *first,
		uint32_t shards, int device, void *stream, kma_iqueue_t *out)
{
	if (!out)
		return KMA_EINVAL;
	*out = NULL;
	if (!base || stride_l2 < 3 || stride_l2 > 30 || capacity == 0 || capacity > 0x7fffffffu - KMA_IQ_MAX_SHARDS)
		return KMA_EINVAL;
	if (shards == 0 || shards > KMA_IQ_MAX_SHARDS || ((uintptr_t)base & 7))
		return KMA_EINVAL;
	uintptr_t off = (uintptr_t)first - (uintptr_t)base;
	if ((uintptr_t)first < (uintptr_t)base || (off & ((1ull << stride_l2) - 1)) || (off >> stride_l2) >= capacity)
		return KMA_EINVAL;
	kma_device_guard g(device);
	if (!g.ok)
		return KMA_ENODEV;
	kma_iqueue_s *q = (kma_iqueue_s *)calloc(1, sizeof(*q));
	if (!q)
		return KMA_ENOMEM;
	q->device = current_device();
	size_t hdr = (sizeof(kma_iqueue) + 127) & ~(size_t)127;
	size_t ends = (size_t)shards * 2 * sizeof(kma_line64);
	size_t dum = (((size_t)shards * 8) + 127) & ~(size_t)127;
	if (cudaMalloc(&q->mem, hdr + ends + dum) != cudaSuccess) {
		cudaGetLastError();
		free(q);
		return KMA_ENOMEM;
	}
	q->dq = (kma_iqueue *)q->mem;
	kma_iqueue hq;
	memset(&hq, 0, sizeof(hq));
	hq.base = (unsigned char *)base;
	hq.ends = (kma_line64 *)((unsigned char *)q->mem + hdr);
	hq.dummies = (unsigned long long *)((unsigned char *)q->mem + hdr + ends);
	hq.stride_l2 = stride_l2;
	hq.capacity = capacity;
	hq.nshards = shards;
	hq.spin_limit = KMA_STRUCT_SPIN;
	cudaStream_t st = kma_stream(stream);
	int rc = KMA_OK;
	if (cudaMemsetAsync(q->mem, 0, hdr + ends + dum, st) != cudaSuccess ||
	    cudaMemcpyAsync(q->dq, &hq, sizeof(hq), cudaMemcpyHostToDevice, st) != cudaSuccess)
		rc = KMA_ECUDA;
	if (rc == KMA_OK) {
		k_iq_init<<<(shards + 255) / 256, 256, 0, st>>>(q->dq, (uint32_t)(off >> stride_l2) + 1);
		if (cudaGetLastError() != cudaSuccess || cudaStreamSynchronize(st) != cudaSuccess)
			rc = KMA_ECUDA;
	}
	if (rc != KMA_OK) {
		cudaFree(q->mem);
		free(q);
		return rc;
	}
	*out = q;
	return KMA_OK;
}

extern "C" int kma_iqueue_destroy(kma_iqueue_t q)
{
	if (!q)
		return KMA_EINVAL;
	kma_device_guard g(q->device);
	cudaError_t e = cudaFree(q->mem);
	free(q);
	return e == cudaSuccess ? KMA_OK : KMA_ECUDA;
}

extern "C" struct kma_iqueue *kma_iqueue_device_ptr(kma_iqueue_t q) { return q ? q->dq : NULL; }

extern "C" int kma_iqueue_error_flags(kma_iqueue_t q, void *stream, uint32_t *flags, int clear)
{
	if (!q || !flags)
		return KMA_EINVAL;
	kma_device_guard g(q->device);
	cudaStream_t st = kma_stream(stream);
	KMA_CUDA(cudaMemcpyAsync(flags, &q->dq->err, 4, cudaMemcpyDeviceToHost, st));
	if (clear)
		KMA_CUDA(cudaMemsetAsync(&q->dq->err, 0, 4, st));
	KMA_CUDA(cudaStreamSynchronize(st));
	return KMA_OK;
}

namespace {
__device__ int64_t iq_item_index(const kma_iqueue *q, const void *p)
{
	if (!p)
		return -1;
	return (int64_t)(((const unsigned char *)p - q->base) >> q->stride_l2);
}

__global__ void k_iq_replay(kma_iqueue *q, const int64_t *ops, int64_t n, int64_t *out, int64_t *fin)
{
	for (int64_t i = 0; i < n; i++) {
		int64_t kind = ops[2 * i], arg = ops[2 * i + 1];
		if (kind == 0) {
			out[i] = (arg >= 0 && arg < q->capacity)
				? kma_iqueue_enqueue_shard(q, q->base + ((size_t)arg << q->stride_l2), 0)
				: 0;
		} else {
			out[i] = iq_item_index(q, kma_iqueue_dequeue_shard(q, 0));
		}
	}
	fin[0] = (int64_t)kma_detail::tw_idx(q->ends[0].v) - 1;
	fin[1] = (int64_t)kma_detail::tw_idx(q->ends[1].v) - 1;
	for (uint32_t k = 0; k < q->capacity; k++)
		fin[2 + k] = (int64_t)kma_detail::tw_idx(*kma_detail::iq_link(q, k + 1)) - 1;
}
} /* namespace */

namespace {
/* one thread: plant a stuck state, then one dequeue with spin limit `limit` */
__global__ void k_dbg_stuck_clq(int state, uint32_t limit, unsigned long long *items, kma_clqueue *q, int64_t *out,
				uint32_t *err)
{
	if (blockIdx.x != 0 || threadIdx.x != 0)
		return;
	unsigned long long a = (unsigned long long)&items[0], b = (unsigned long long)&items[2];
	items[0] = state == 0 ? KMA_Q_POISON : 0ull; /* a's link */
	items[2] = 0ull;                               /* b's link */
	q->head = a;
	q->tail = b; /* state 1: b's append exchanged the tail and stopped */
	__threadfence();
	*out = kma_detail::clq_dequeue<kma_detail::clq_link_head>(q, err, limit) ? 1 : -1;
}
__global__ void k_dbg_stuck_iq(uint32_t limit, kma_iqueue *q, int64_t *out)
{
	if (blockIdx.x != 0 || threadIdx.x != 0)
		return;
	q->spin_limit = limit;
	const kma_detail::iq_links L(q);
	kma_q::iq_set_link<kma_detail::gpu_ops>(L, 1u, 2u); /* dummy 1 -> item 2 */
	q->ends[0].v = kma_q::tw_make(1u, 1u);              /* hold tag odd: held by nobody */
	__threadfence();
	void *it = kma_iqueue_dequeue_shard(q, 0);
	*out = it ? 1 : -1;
}
} /* namespace */

namespace {
/* one block: warps append 32 items each, in warp order, `calls` times;
 * then `calls` block-form dequeues */
__global__ void __launch_bounds__(512) k_dbg_fifo_clq(kma_clqueue *q, unsigned char *items, uint32_t calls, int64_t *out, uint32_t *err,
			       const kma_chain_log *log)
{
	__shared__ unsigned long long smem[512 + 1];
	const uint32_t tid = threadIdx.x, lane = tid & 31, wid = tid >> 5, nw = blockDim.x >> 5;
	for (uint32_t c = 0; c < calls; c++)
		for (uint32_t w = 0; w < nw; w++) {
			if (wid == w) {
				const size_t i = (size_t)c * blockDim.x + w * 32 + lane;
				kma_clqueue_enqueue_warp(q, (kma_clqueue_item *)(items + i * QITEM), err, KMA_STRUCT_SPIN,
							 const_cast<kma_chain_log *>(log));
			}
			__syncthreads();
		}
	for (uint32_t c = 0; c < calls; c++) {
		kma_clqueue_item *it = kma_clqueue_dequeue_block(q, true, smem, err, KMA_STRUCT_SPIN, log);
		out[(size_t)c * blockDim.x + tid] = it ? (int64_t)(((unsigned char *)it - items) / QITEM) : -1;
	}
}
__global__ void __launch_bounds__(512) k_dbg_fifo_iq(kma_iqueue *q, uint32_t calls, int64_t *out)
{
	__shared__ unsigned long long smem[512 + 1];
	const uint32_t tid = threadIdx.x, lane = tid & 31, wid = tid >> 5, nw = blockDim.x >> 5;
	for (uint32_t c = 0; c < calls; c++)
		for (uint32_t w = 0; w < nw; w++) {
			if (wid == w) {
				/* item i of the enqueue order is array item i + 2 (item 1 is the dummy) */
				const size_t i = (size_t)c * blockDim.x + w * 32 + lane;
				kma_iqueue_enqueue_warp_shard(q, q->base + ((i + 1) << q->stride_l2), 0);
			}
			__syncthreads();
		}
	for (uint32_t c = 0; c < calls; c++) {
		unsigned char *it = (unsigned char *)kma_iqueue_dequeue_block(q, true, smem);
		out[(size_t)c * blockDim.x + tid] =
			!it ? -1 : (it == q->base ? -2 : (int64_t)((it - q->base) >> q->stride_l2) - 1);
	}
}
} /* namespace */

extern "C" int kma_debug_queue_block_fifo(int kind, uint32_t tpb, uint32_t calls, int device, int64_t *out,
		uint32_t *err)
{
	if (!out || !err || tpb == 0 || tpb % 32 || tpb > 512 || calls == 0 || calls > 1024 ||
	    (kind != KMA_C3_CLQUEUE && kind != KMA_C3_IQUEUE))
		return KMA_EINVAL;
	kma_device_guard g(device);
	if (!g.ok)
		return KMA_ENODEV;
	const size_t n = (size_t)tpb * calls;
	dev_bufs b;
	int64_t *dout = b.alloc<int64_t>(n * 8);
	uint32_t *derr = b.alloc<uint32_t>(4);
	unsigned char *items = b.alloc<unsigned char>((n + 2) * QITEM);
	if (!dout || !derr || !items)
		return KMA_ENOMEM;
	KMA_CUDA(cudaMemset(derr, 0, 4));
	KMA_CUDA(cudaMemset(items, 0, (n + 2) * QITEM));
	kma_chain_log_t log = NULL;
	uint32_t rec = 1;
	while (rec < n / 32 + 1)
		rec <<= 1;
	int rc = kma_chain_log_create(rec, -1, NULL, &log);
	if (rc != KMA_OK)
		return rc;
	uint32_t e = 0;
	if (kind == KMA_C3_CLQUEUE) {
		kma_clqueue *q = b.alloc<kma_clqueue>(sizeof(kma_clqueue));
		if (!q) {
			kma_chain_log_destroy(log);
			return KMA_ENOMEM;
		}
		cudaMemset(q, 0, sizeof(kma_clqueue));
		k_dbg_fifo_clq<<<1, tpb>>>(q, items, calls, dout, derr, kma_chain_log_device_ptr(log));
		if (cudaGetLastError() != cudaSuccess || cudaDeviceSynchronize() != cudaSuccess)
			rc = KMA_ECUDA;
		if (rc == KMA_OK && cudaMemcpy(&e, derr, 4, cudaMemcpyDeviceToHost) != cudaSuccess)
			rc = KMA_ECUDA;
	} else {
		kma_iqueue_t q = NULL;
		rc = kma_iqueue_create(items, 4, (uint32_t)n + 1, items, 1, -1, NULL, &q);
		if (rc == KMA_OK)
			rc = kma_iqueue_set_chain_log(q, log, NULL);
		if (rc == KMA_OK) {
			k_dbg_fifo_iq<<<1, tpb>>>(q->dq, calls, dout);
			if (cudaGetLastError() != cudaSuccess || cudaDeviceSynchronize() != cudaSuccess)
				rc = KMA_ECUDA;
		}
		if (rc == KMA_OK)
			rc = kma_iqueue_error_flags(q, NULL, &e, 0);
		if (q)
			kma_iqueue_destroy(q);
	}
	kma_chain_log_destroy(log);
	if (rc != KMA_OK)
		return rc;
	KMA_CUDA(cudaMemcpy(out, dout, n * 8, cudaMemcpyDeviceToHost));
	*err = e;
	return KMA_OK;
}

extern "C" int kma_debug_queue_stuck_dequeue(int kind, int state, uint32_t spin_limit, int device, int64_t *taken,
		uint32_t *flags)
{
	if (!taken || !flags || spin_limit == 0 || !((kind == KMA_C3_CLQUEUE && (state == 0 || state == 1)) ||
						    (kind == KMA_C3_IQUEUE && state == 0)))
		return KMA_EINVAL;
	kma_device_guard g(device);
	if (!g.ok)
		return KMA_ENODEV;
	dev_bufs b;
	int64_t *out = b.alloc<int64_t>(8);
	uint32_t *err = b.alloc<uint32_t>(4);
	unsigned long long *items = b.alloc<unsigned long long>(64); /* 4 items of 16 bytes */
	if (!out || !err || !items)
		return KMA_ENOMEM;
	KMA_CUDA(cudaMemset(err, 0, 4));
	KMA_CUDA(cudaMemset(items, 0, 64));
	uint32_t e = 0;
	if (kind == KMA_C3_CLQUEUE) {
		kma_clqueue *q = b.alloc<kma_clqueue>(sizeof(kma_clqueue));
		if (!q)
			return KMA_ENOMEM;
		k_dbg_stuck_clq<<<1, 1>>>(state, spin_limit, items, q, out, err);
		KMA_CUDA(cudaGetLastError());
		KMA_CUDA(cudaDeviceSynchronize());
		KMA_CUDA(cudaMemcpy(&e, err, 4, cudaMemcpyDeviceToHost));
	} else {
		kma_iqueue_t q = NULL;
		int rc = kma_iqueue_create(items, 4, 3, items, 1, -1, NULL, &q);
		if (rc != KMA_OK)
			return rc;
		k_dbg_stuck_iq<<<1, 1>>>(spin_limit, q->dq, out);
		if (cudaGetLastError() != cudaSuccess || cudaDeviceSynchronize() != cudaSuccess) {
			kma_iqueue_destroy(q);
			return KMA_ECUDA;
		}
		rc = kma_iqueue_error_flags(q, NULL, &e, 0);
		kma_iqueue_destroy(q);
		if (rc != KMA_OK)
			return rc;
	}
	KMA_CUDA(cudaMemcpy(taken, out, 8, cudaMemcpyDeviceToHost));
	*flags = e;
	return KMA_OK;
}

extern "C" int kma_iqueue_replay_host(uint32_t n_items, uint32_t stride_l2, const int64_t *ops, int64_t n,
		int64_t *out, int64_t *final_state)
{
	if (!final_state || n_items == 0 || stride_l2 < 3 || stride_l2 > 16)
		return KMA_EINVAL;
	dev_bufs b;
	unsigned char *items = b.alloc<unsigned char>((size_t)n_items << stride_l2);
	int64_t *dfin = b.alloc<int64_t>((size_t)(n_items + 2) * 8);
	if (!items || !dfin)
		return KMA_ENOMEM;
	cudaMemset(items, 0, (size_t)n_items << stride_l2);
	kma_iqueue_t q;
	int rc = kma_iqueue_create(items, stride_l2, n_items, items, 1, -1, NULL, &q);
	if (rc != KMA_OK)
		return rc;
	rc = replay_host(n, ops, out, [&](const int64_t *dops, int64_t *dout) {
		k_iq_replay<<<1, 1>>>(q->dq, dops, n, dout, dfin);
		return KMA_OK;
	});
	if (rc == KMA_OK && cudaMemcpy(final_state, dfin, (size_t)(n_items + 2) * 8, cudaMemcpyDeviceToHost) != cudaSuccess)
		rc = KMA_ECUDA;
	uint32_t fl = 0;
	if (rc == KMA_OK && kma_iqueue_error_flags(q, NULL, &fl, 0) == KMA_OK && fl)
		rc = KMA_ETIMEDOUT;
	kma_iqueue_destroy(q);
	return rc;
}

/* ------------------------------------------------------------------ */
/* chain log                                                           */
/* ------------------------------------------------------------------ */

extern "C" int kma_chain_log_create(uint32_t records, int device, void *stream, kma_chain_log_t *out)
{
	if (!out)
		return KMA_EINVAL;
	*out = NULL;
	if (records == 0 || (records & (records - 1)) || records > (1u << 24))
		return KMA_EINVAL;
	kma_device_guard g(device);
	if (!g.ok)
		return KMA_ENODEV;
	kma_chain_log_s *l = (kma_chain_log_s *)calloc(1, sizeof(*l));
	if (!l)
		return KMA_ENOMEM;
	l->device = current_device();
	/* header line, counter line, then the records (zeroed: an entry is 0
	 * until a chain fills it) */
	const size_t hdr = 256, bytes = hdr + (size_t)records * 256;
	if (cudaMalloc(&l->mem, bytes) != cudaSuccess) {
		cudaGetLastError();
		free(l);
		return KMA_ENOMEM;
	}
	l->dl = (kma_chain_log *)l->mem;
	kma_chain_log hl;
	memset(&hl, 0, sizeof(hl));
	hl.rec = (unsigned long long *)((unsigned char *)l->mem + hdr);
	hl.next = (unsigned int *)((unsigned char *)l->mem + 128);
	hl.mask = records - 1;
	cudaStream_t st = kma_stream(stream);
	int rc = KMA_OK;
	if (cudaMemsetAsync(l->mem, 0, bytes, st) != cudaSuccess)
		rc = KMA_ECUDA;
	if (rc == KMA_OK)
		rc = put_sync(l->dl, &hl, sizeof(hl), st);
	if (rc != KMA_OK) {
		cudaFree(l->mem);
		free(l);
		return rc;
	}
	*out = l;
	return KMA_OK;
}

extern "C" int kma_chain_log_destroy(kma_chain_log_t l)
{
	if (!l)
		return KMA_EINVAL;
	kma_device_guard g(l->device);
	cudaError_t e = cudaFree(l->mem);
	free(l);
	return e == cudaSuccess ? KMA_OK : KMA_ECUDA;
}

extern "C" struct kma_chain_log *kma_chain_log_device_ptr(kma_chain_log_t l) { return l ? l->dl : NULL; }

extern "C" int kma_iqueue_set_chain_log(kma_iqueue_t q, kma_chain_log_t l, void *stream)
{
	if (!q)
		return KMA_EINVAL;
	kma_device_guard g(q->device);
	kma_chain_log *p = l ? l->dl : NULL;
	return put_sync(&q->dq->log, &p, sizeof(p), kma_stream(stream));
}

/* ------------------------------------------------------------------ */
/* clTree                                                              */
/* ------------------------------------------------------------------ */

extern "C" int kma_cltree_create(int device, void *stream, kma_cltree_t *out)
{
	if (!out)
		return KMA_EINVAL;
	*out = NULL;
	kma_device_guard g(device);
	if (!g.ok)
		return KMA_ENODEV;
	kma_cltree_s *t = (kma_cltree_s *)calloc(1, sizeof(*t));
	if (!t)
		return KMA_ENOMEM;
	t->device = current_device();
	if (cudaMalloc(&t->dt, 128) != cudaSuccess) {
		cudaGetLastError();
		free(t);
		return KMA_ENOMEM;
	}
	if (cudaMemsetAsync(t->dt, 0, 128, kma_stream(stream)) != cudaSuccess ||
	    cudaStreamSynchronize(kma_stream(stream)) != cudaSuccess) {
		cudaFree(t->dt);
		free(t);
		return KMA_ECUDA;
	}
	*out = t;
	return KMA_OK;
}

extern "C" int kma_cltree_destroy(kma_cltree_t t)
{
	if (!t)
		return KMA_EINVAL;
	kma_device_guard g(t->device);
	cudaError_t e = cudaFree(t->dt);
	free(t);
	return e == cudaSuccess ? KMA_OK : KMA_ECUDA;
}

extern "C" struct kma_cltree *kma_cltree_device_ptr(kma_cltree_t t) { return t ? t->dt : NULL; }

namespace {
/* In-order walk of the live keys with an explicit stack of `cap` entries;
 * writes up to cap keys (when keys != NULL) and the summary. */
__global__ void k_tree_walk(const kma_cltree *t, unsigned long long *stack, uint64_t cap, uint32_t *keys,
		unsigned long long *summary /* count, xor, sum, sorted, overflow */)
{
	uint64_t sp = 0, count = 0;
	unsigned long long x = 0, sum = 0;
	uint32_t sorted = 1, overflow = 0;
	long long prev = -1;
	unsigned long long cur = t->root;
	while (cur || sp) {
		while (cur) {
			if (sp >= cap) {
				overflow = 1;
				cur = 0;
				sp = 0;
				break;
			}
			stack[sp++] = cur;
			cur = ((const kma_cltree_node *)cur)->left;
		}
		if (!sp)
			break;
		cur = stack[--sp];
		const kma_cltree_node *nd = (const kma_cltree_node *)cur;
		if (nd->state == 0) {
			if ((long long)nd->key <= prev)
				sorted = 0;
			prev = nd->key;
			if (keys && count < cap)
				keys[count] = nd->key;
			count++;
			x ^= nd->key;
			sum += nd->key;
		}
		cur = nd->right;
	}
	summary[0] = count;
	summary[1] = x;
	summary[2] = sum;
	summary[3] = sorted;
	summary[4] = overflow;
}

__global__ void k_tree_replay(kma_cltree *t, kma_cltree_node *pool, const int64_t *ops, int64_t n, int64_t *out)
{
	for (int64_t i = 0; i < n; i++) {
		int64_t kind = ops[2 * i];
		uint32_t key = (uint32_t)ops[2 * i + 1];
		if (kind == 0) {
			pool[i].key = key;
			out[i] = kma_cltree_add(t, &pool[i]);
		} else if (kind == 1) {
			kma_cltree_node *f = kma_cltree_get(t, key);
			out[i] = f ? (int64_t)(f - pool) : -1;
		} else {
			out[i] = kma_cltree_remove(t, key);
		}
	}
}
} /* namespace */

extern "C" int kma_cltree_replay_host(const int64_t *ops, int64_t n, int64_t *out, uint32_t *keys_out,
		int64_t *n_keys)
{
	if (!keys_out || !n_keys || n <= 0)
		return KMA_EINVAL;
	kma_cltree_t t;
	int rc = kma_cltree_create(-1, NULL, &t);
	if (rc != KMA_OK)
		return rc;
	dev_bufs b;
	kma_cltree_node *pool = b.alloc<kma_cltree_node>((size_t)n * sizeof(kma_cltree_node));
	unsigned long long *stack = b.alloc<unsigned long long>((size_t)n * 8);
	uint32_t *dkeys = b.alloc<uint32_t>((size_t)n * 4);
	unsigned long long *summ = b.alloc<unsigned long long>(5 * 8);
	if (!pool || !stack || !dkeys || !summ) {
		kma_cltree_destroy(t);
		return KMA_ENOMEM;
	}
	rc = replay_host(n, ops, out, [&](const int64_t *dops, int64_t *dout) {
		k_tree_replay<<<1, 1>>>(t->dt, pool, dops, n, dout);
		k_tree_walk<<<1, 1>>>(t->dt, stack, (uint64_t)n, dkeys, summ);
		return KMA_OK;
	});
	unsigned long long s[5] = {0, 0, 0, 0, 0};
	if (rc == KMA_OK && cudaMemcpy(s, summ, sizeof(s), cudaMemcpyDeviceToHost) != cudaSuccess)
		rc = KMA_ECUDA;
	if (rc == KMA_OK && s[4])
		rc = KMA_EFAULT;
	if (rc == KMA_OK) {
		*n_keys = (int64_t)s[0];
		if (s[0] && cudaMemcpy(keys_out, dkeys, s[0] * 4, cudaMemcpyDeviceToHost) != cudaSuccess)
			rc = KMA_ECUDA;
	}
	kma_cltree_destroy(t);
	return rc;
}

/* ------------------------------------------------------------------ */
/* clArrayList                                                         */
/* ------------------------------------------------------------------ */

extern "C" int kma_clarraylist_create(uint32_t obj_size, kma_heap_t kma, kma_pma_t pma, void *stream,
		kma_clarraylist_t *out)
{
	if (!out)
		return KMA_EINVAL;
	*out = NULL;
	if (obj_size == 0 || (!kma == !pma))
		return KMA_EINVAL;
	kma_device_guard g(kma ? kma->device : pma->device);
	if (!g.ok)
		return KMA_ENODEV;
	kma_clarraylist_s *l = (kma_clarraylist_s *)calloc(1, sizeof(*l));
	if (!l)
		return KMA_ENOMEM;
	l->device = current_device();
	if (cudaMalloc(&l->dl, 128) != cudaSuccess) {
		cudaGetLastError();
		free(l);
		return KMA_ENOMEM;
	}
	unsigned char buf[128];
	memset(buf, 0, sizeof(buf));
	kma_clarraylist *hl = (kma_clarraylist *)buf;
	hl->obj_size = obj_size;
	hl->heap = kma ? (void *)kma->dh : (void *)pma->dp;
	hl->heap_kind = kma ? KMA_AL_HEAP_KMA : KMA_AL_HEAP_PMA;
	int rc = put_sync(l->dl, buf, sizeof(buf), kma_stream(stream));
	if (rc != KMA_OK) {
		cudaFree(l->dl);
		free(l);
		return rc;
	}
	*out = l;
	return KMA_OK;
}

extern "C" int kma_clarraylist_destroy(kma_clarraylist_t l)
{
	if (!l)
		return KMA_EINVAL;
	kma_device_guard g(l->device);
	cudaError_t e = cudaFree(l->dl);
	free(l);
	return e == cudaSuccess ? KMA_OK : KMA_ECUDA;
}

extern "C" struct kma_clarraylist *kma_clarraylist_device_ptr(kma_clarraylist_t l) { return l ? l->dl : NULL; }

namespace {
__device__ int64_t al_off(const unsigned char *base, const void *p)
{
	return p ? (int64_t)((const unsigned char *)p - base) : -1;
}

__global__ void k_al_replay(kma_clarraylist *l, const unsigned char *base, const int64_t *ops, int64_t n,
		int64_t *out)
{
	for (int64_t i = 0; i < n; i++) {
		int64_t kind = ops[2 * i], arg = ops[2 * i + 1];
		if (kind == 0)
			out[i] = al_off(base, kma_clarraylist_grow(l, (uint32_t)arg));
		else if (kind == 1)
			out[i] = al_off(base, kma_clarraylist_get(l, (unsigned long long)arg));
		else if (kind == 2) {
			kma_clarraylist_clear(l);
			out[i] = 0;
		} else
			out[i] = al_off(base, kma_clarraylist_grow_warp(l, (uint32_t)arg));
	}
}

__global__ void k_al_group(kma_clarraylist *l, const unsigned char *base, const uint32_t *objs, uint32_t n,
		int mode, int64_t *out)
{
	__shared__ unsigned long long smem[33];
	uint32_t t = threadIdx.x;
	void *p = mode == 0 ? kma_clarraylist_grow_block(l, objs[t], smem) : kma_clarraylist_grow_warp(l, objs[t]);
	out[t] = al_off(base, p);
}
} /* namespace */

static const unsigned char *al_data_base(kma_heap_t kma, kma_pma_t pma)
{
	return kma ? kma->hh.sb_base : pma->base;
}

extern "C" int kma_clarraylist_replay_host(kma_heap_t kma, kma_pma_t pma, uint32_t obj_size,
		const int64_t *ops, int64_t n, int64_t *out)
{
	kma_clarraylist_t l;
	int rc = kma_clarraylist_create(obj_size, kma, pma, NULL, &l);
	if (rc != KMA_OK)
		return rc;
	{
		kma_device_guard g(l->device);
		const unsigned char *base = al_data_base(kma, pma);
		rc = replay_host(n, ops, out, [&](const int64_t *dops, int64_t *dout) {
			k_al_replay<<<1, 1>>>(l->dl, base, dops, n, dout);
			return KMA_OK;
		});
	}
	kma_clarraylist_destroy(l);
	return rc;
}

extern "C" int kma_clarraylist_group_host(kma_heap_t kma, kma_pma_t pma, uint32_t obj_size,
		const uint32_t *objs, uint32_t n, int mode, int64_t *out)
{
	if (!objs || !out || n == 0 || n > 1024 || (mode != 0 && mode != 1))
		return KMA_EINVAL;
	kma_clarraylist_t l;
	int rc = kma_clarraylist_create(obj_size, kma, pma, NULL, &l);
	if (rc != KMA_OK)
		return rc;
	{
		kma_device_guard g(l->device);
		dev_bufs b;
		uint32_t *dobjs = b.alloc<uint32_t>((size_t)n * 4);
		int64_t *dout = b.alloc<int64_t>((size_t)n * 8);
		if (!dobjs || !dout)
			rc = KMA_ENOMEM;
		if (rc == KMA_OK && cudaMemcpy(dobjs, objs, (size_t)n * 4, cudaMemcpyHostToDevice) != cudaSuccess)
			rc = KMA_ECUDA;
		if (rc == KMA_OK) {
			k_al_group<<<1, n>>>(l->dl, al_data_base(kma, pma), dobjs, n, mode, dout);
			if (cudaGetLastError() != cudaSuccess || cudaDeviceSynchronize() != cudaSuccess)
				rc = KMA_ECUDA;
		}
		if (rc == KMA_OK && cudaMemcpy(out, dout, (size_t)n * 8, cudaMemcpyDeviceToHost) != cudaSuccess)
			rc = KMA_ECUDA;
	}
	kma_clarraylist_destroy(l);
	return rc;
}

/* ------------------------------------------------------------------ */
/* config 3: concurrent queues                                         */
/* ------------------------------------------------------------------ */
namespace {

/* A seeded bijection of [0, n): invertible mixing on the next power of
 * two (odd multiply, xor-shift, add), cycle-walked into [0, n). */
__device__ __forceinline__ uint32_t perm_u32(uint32_t i, uint32_t n, uint64_t seed)
{
	uint32_t bits = n <= 1 ? 1 : 32 - __clz(n - 1);
	uint32_t mask = bits >= 32 ? 0xffffffffu : ((1u << bits) - 1u);
	uint32_t k0 = (uint32_t)seed | 1u, k1 = (uint32_t)(seed >> 32);
	uint32_t x = i;
	do {
		for (int r = 0; r < 3; r++) {
			x = (x * (k0 | 1u)) & mask;
			x ^= x >> ((bits + 1) / 2);
			x = (x + k1) & mask;
			k0 = k0 * 0x9E3779B9u + 0x7F4A7C15u;
		}
		k0 = (uint32_t)seed | 1u;
	} while (x >= n);
	return x;
}

struct c3_acc {
	unsigned long long cnt, x, sum;
};
__device__ __forceinline__ void warp_flush(unsigned long long *dst, unsigned long long cnt, unsigned long long x,
		unsigned long long sum)
{
	for (int d = 16; d > 0; d >>= 1) {
		cnt += __shfl_down_sync(0xffffffffu, cnt, d);
		x ^= __shfl_down_sync(0xffffffffu, x, d);
		sum += __shfl_down_sync(0xffffffffu, sum, d);
	}
	if ((threadIdx.x & 31) == 0) {
		if (cnt)
			atomicAdd(&dst[0], cnt);
		if (x)
			atomicXor(&dst[1], x);
		if (sum)
			atomicAdd(&dst[2], sum);
	}
}

/* acc: [0..2] in (count, xor, sum), [3..5] out, [6] empty, [7] remaining,
 * [8] walk failures */
template <bool WARP>
__global__ void k_c3_clq_enq(unsigned char *qs, uint32_t shards, unsigned char *items, uint32_t per_thread,
		uint32_t n, uint64_t seed, unsigned long long *acc, uint32_t *err, kma_chain_log *log)
{
	uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
	unsigned long long c = 0, x = 0, s = 0;
	kma_clqueue *q = (kma_clqueue *)(qs + (size_t)(t % shards) * 128);
	for (uint32_t k = 0; k < per_thread; k++) {
		uint32_t i = t * per_thread + k;
		/* the warp form keeps every lane in the loop (NULL: no item) */
		if (!WARP && i >= n)
			break;
		unsigned char *it = i < n ? items + (size_t)i * QITEM : nullptr;
		uint32_t pay = i < n ? perm_u32(i, n, seed) : 0u;
		if (it)
			*(uint32_t *)(it + 8) = pay;
		int ok = WARP ? kma_clqueue_enqueue_warp(q, (kma_clqueue_item *)it, err, KMA_STRUCT_SPIN, log)
			      : kma_clqueue_enqueue(q, (kma_clqueue_item *)it, err);
		if (ok) {
			c++;
			x ^= pay;
			s += pay;
		}
	}
	warp_flush(acc, c, x, s);
}

template <bool WARP>
__global__ void k_c3_clq_deq(unsigned char *qs, uint32_t shards, uint32_t per_thread, uint32_t threads,
		unsigned long long *acc, uint32_t *err, const kma_chain_log *log)
{
	uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
	unsigned long long c = 0, x = 0, s = 0, e = 0;
	if (WARP || t < threads) {
		kma_clqueue *q = t < threads ? (kma_clqueue *)(qs + (size_t)(t % shards) * 128) : nullptr;
		for (uint32_t k = 0; k < per_thread; k++) {
			kma_clqueue_item *it = WARP ? kma_clqueue_dequeue_warp(q, err, KMA_STRUCT_SPIN, log)
						    : kma_clqueue_dequeue(q, err);
			if (!q)
				continue;
			if (!it) {
				e++;
				continue;
			}
			uint32_t pay = *(volatile uint32_t *)((unsigned char *)it + 8);
			c++;
			x ^= pay;
			s += pay;
		}
	}
	warp_flush(acc + 3, c, x, s);
	for (int d = 16; d > 0; d >>= 1)
		e += __shfl_down_sync(0xffffffffu, e, d);
	if ((threadIdx.x & 31) == 0 && e)
		atomicAdd(&acc[6], e);
}

/* the block form on one queue: every thread of every block calls it */
__global__ void __launch_bounds__(256) k_c3_clq_deq_block(kma_clqueue *q, uint32_t per_thread, uint32_t threads,
		unsigned long long *acc, uint32_t *err, const kma_chain_log *log)
{
	__shared__ unsigned long long smem[256 + 1];
	const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
	unsigned long long c = 0, x = 0, s = 0, e = 0;
	for (uint32_t k = 0; k < per_thread; k++) {
		kma_clqueue_item *it = kma_clqueue_dequeue_block(q, t < threads, smem, err, KMA_STRUCT_SPIN, log);
		if (t >= threads)
			continue;
		if (!it) {
			e++;
			continue;
		}
		uint32_t pay = *(volatile uint32_t *)((unsigned char *)it + 8);
		c++;
		x ^= pay;
		s += pay;
	}
	warp_flush(acc + 3, c, x, s);
	for (int d = 16; d > 0; d >>= 1)
		e += __shfl_down_sync(0xffffffffu, e, d);
	if ((threadIdx.x & 31) == 0 && e)
		atomicAdd(&acc[6], e);
}

/* one thread per shard: walk what is left; it counts as "out" too */
__global__ void k_c3_clq_walk(unsigned char *qs, uint32_t shards, uint64_t n, unsigned long long *acc)
{
	uint32_t sh = blockIdx.x * blockDim.x + threadIdx.x;
	if (sh >= shards)
		return;
	kma_clqueue *q = (kma_clqueue *)(qs + (size_t)sh * 128);
	unsigned long long c = 0, x = 0, s = 0;
	kma_clqueue_item *it = kma_clqueue_first(q), *last = NULL;
	uint64_t steps = 0;
	while (it && steps <= n) {
		uint32_t pay = *(uint32_t *)((unsigned char *)it + 8);
		c++;
		x ^= pay;
		s += pay;
		last = it;
		it = kma_clqueue_next(it);
		steps++;
	}
	bool ok = steps <= n && (unsigned long long)last == kma_detail::qp_ptr(q->tail);
	if (c) {
		atomicAdd(&acc[3], c);
		atomicXor(&acc[4], x);
		atomicAdd(&acc[5], s);
		atomicAdd(&acc[7], c);
	}
	if (!ok)
		atomicAdd(&acc[8], 1ull);
}

/* indexed queue: item 0 is shard 0's initial dummy (payload excluded) */
template <bool WARP>
__global__ void k_c3_iq_enq(kma_iqueue *q, uint32_t per_thread, uint32_t n, uint64_t seed, unsigned long long *acc)
{
	uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
	unsigned long long c = 0, x = 0, s = 0;
	uint32_t shard = t % q->nshards;
	for (uint32_t k = 0; k < per_thread; k++) {
		uint32_t i = t * per_thread + k;
		if (!WARP && i >= n)
			break;
		unsigned char *it = i < n ? q->base + ((size_t)(i + 1) << q->stride_l2) : nullptr;
		uint32_t pay = i < n ? perm_u32(i, n, seed) : 0u;
		if (it)
			*(uint32_t *)(it + 8) = pay;
		if (WARP ? kma_iqueue_enqueue_warp_shard(q, it, shard) : kma_iqueue_enqueue_shard(q, it, shard)) {
			c++;
			x ^= pay;
			s += pay;
		}
	}
	warp_flush(acc, c, x, s);
}

template <bool WARP>
__global__ void k_c3_iq_deq(kma_iqueue *q, uint32_t per_thread, uint32_t threads, unsigned long long *acc)
{
	uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
	unsigned long long c = 0, x = 0, s = 0, e = 0, d0 = 0;
	if (WARP || t < threads) {
		uint32_t shard = t % q->nshards;
		for (uint32_t k = 0; k < per_thread; k++) {
			unsigned char *it = WARP ? (unsigned char *)kma_iqueue_dequeue_warp_shard(q, shard, t < threads)
						 : (unsigned char *)kma_iqueue_dequeue_shard(q, shard);
			if (t >= threads)
				continue;
			if (!it) {
				e++;
				continue;
			}
			if (it == q->base) {
				d0++; /* the initial dummy carries no payload */
				continue;
			}
			uint32_t pay = *(volatile uint32_t *)(it + 8);
			c++;
			x ^= pay;
			s += pay;
		}
	}
	warp_flush(acc + 3, c, x, s);
	for (int d = 16; d > 0; d >>= 1) {
		e += __shfl_down_sync(0xffffffffu, e, d);
		d0 += __shfl_down_sync(0xffffffffu, d0, d);
	}
	if ((threadIdx.x & 31) == 0) {
		if (e)
			atomicAdd(&acc[6], e);
		if (d0)
			atomicAdd(&acc[9], d0);
	}
}

/* the block form on shard 0 (one queue): every thread of every block calls it */
__global__ void __launch_bounds__(256) k_c3_iq_deq_block(kma_iqueue *q, uint32_t per_thread, uint32_t threads,
		unsigned long long *acc)
{
	__shared__ unsigned long long smem[256 + 1];
	const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
	unsigned long long c = 0, x = 0, s = 0, e = 0, d0 = 0;
	for (uint32_t k = 0; k < per_thread; k++) {
		unsigned char *it = (unsigned char *)kma_iqueue_dequeue_block(q, t < threads, smem);
		if (t >= threads)
			continue;
		if (!it) {
			e++;
			continue;
		}
		if (it == q->base) {
			d0++; /* the initial dummy carries no payload */
			continue;
		}
		uint32_t pay = *(volatile uint32_t *)(it + 8);
		c++;
		x ^= pay;
		s += pay;
	}
	warp_flush(acc + 3, c, x, s);
	for (int d = 16; d > 0; d >>= 1) {
		e += __shfl_down_sync(0xffffffffu, e, d);
		d0 += __shfl_down_sync(0xffffffffu, d0, d);
	}
	if ((threadIdx.x & 31) == 0) {
		if (e)
			atomicAdd(&acc[6], e);
		if (d0)
			atomicAdd(&acc[9], d0);
	}
}

__global__ void k_c3_iq_walk(kma_iqueue *q, uint64_t n, unsigned long long *acc)
{
	uint32_t sh = blockIdx.x * blockDim.x + threadIdx.x;
	if (sh >= q->nshards)
		return;
	unsigned long long c = 0, x = 0, s = 0;
	uint32_t idx = kma_detail::tw_idx(q->ends[2 * sh].v), last = 0;
	uint64_t steps = 0;
	while (idx && steps <= n + q->nshards) {
		if (idx > 1 && idx <= q->capacity) { /* user items carry payloads */
			uint32_t pay = *(uint32_t *)(q->base + ((size_t)(idx - 1) << q->stride_l2) + 8);
			c++;
			x ^= pay;
			s += pay;
		}
		last = idx;
		idx = kma_detail::tw_idx(*kma_detail::iq_link(q, idx));
		steps++;
	}
	bool ok = steps <= n + q->nshards && last == kma_detail::tw_idx(q->ends[2 * sh + 1].v);
	if (c) {
		atomicAdd(&acc[3], c);
		atomicXor(&acc[4], x);
		atomicAdd(&acc[5], s);
		atomicAdd(&acc[7], c);
	}
	if (!ok)
		atomicAdd(&acc[8], 1ull);
}

} /* namespace */

extern "C" int kma_c3_queue_run(int kind, uint32_t threads, uint32_t per_thread, uint32_t shards, uint64_t seed,
		int device, kma_c3_queue_stats *st)
{
	const bool block = kind & KMA_C3_BLOCK;
	const bool warp = (kind & KMA_C3_WARP) || block;
	kind &= ~(KMA_C3_WARP | KMA_C3_BLOCK);
	if (!st || threads == 0 || per_thread == 0 || shards == 0 || shards > KMA_IQ_MAX_SHARDS ||
	    (kind != KMA_C3_CLQUEUE && kind != KMA_C3_IQUEUE) || (block && shards != 1))
		return KMA_EINVAL;
	uint64_t n64 = (uint64_t)threads * per_thread;
	if (n64 >= 0x7fffffffull)
		return KMA_EINVAL;
	uint32_t n = (uint32_t)n64;
	kma_device_guard g(device);
	if (!g.ok)
		return KMA_ENODEV;
	memset(st, 0, sizeof(*st));
	dev_bufs b;
	unsigned long long *acc = b.alloc<unsigned long long>(16 * 8);
	uint32_t *err = b.alloc<uint32_t>(4);
	unsigned char *items = b.alloc<unsigned char>((size_t)(n + 1) * QITEM);
	if (!acc || !err || !items)
		return KMA_ENOMEM;
	KMA_CUDA(cudaMemset(acc, 0, 16 * 8));
	KMA_CUDA(cudaMemset(err, 0, 4));
	KMA_CUDA(cudaMemset(items, 0, (size_t)(n + 1) * QITEM));
	cudaEvent_t e0, e1, e2;
	cudaEventCreate(&e0);
	cudaEventCreate(&e1);
	cudaEventCreate(&e2);
	uint32_t blocks = (threads + 255) / 256;
	int rc = KMA_OK;
	kma_iqueue_t iq = NULL;
	/* warp forms: a chain log of one record per 16 payloads (every chain
	 * of this run keeps its record: chains hold up to 32 payloads) */
	kma_chain_log_t log = NULL;
	if (warp) {
		uint32_t rec = 1;
		while (rec < n / 16 && rec < (1u << 24))
			rec <<= 1;
		rc = kma_chain_log_create(rec, -1, NULL, &log);
	}
	if (rc != KMA_OK) {
		/* no log: nothing ran */
	} else if (kind == KMA_C3_CLQUEUE) {
		unsigned char *qs = b.alloc<unsigned char>((size_t)shards * 128);
		if (!qs)
			rc = KMA_ENOMEM;
		if (rc == KMA_OK) {
			cudaMemset(qs, 0, (size_t)shards * 128);
			cudaEventRecord(e0);
			kma_chain_log *dl = kma_chain_log_device_ptr(log);
			if (warp)
				k_c3_clq_enq<true><<<blocks, 256>>>(qs, shards, items, per_thread, n, seed, acc, err, dl);
			else
				k_c3_clq_enq<false><<<blocks, 256>>>(qs, shards, items, per_thread, n, seed, acc, err, dl);
			cudaEventRecord(e1);
			if (block)
				k_c3_clq_deq_block<<<blocks, 256>>>((kma_clqueue *)qs, per_thread, threads, acc, err, dl);
			else if (warp)
				k_c3_clq_deq<true><<<blocks, 256>>>(qs, shards, per_thread, threads, acc, err, dl);
			else
				k_c3_clq_deq<false><<<blocks, 256>>>(qs, shards, per_thread, threads, acc, err, dl);
			cudaEventRecord(e2);
			k_c3_clq_walk<<<(shards + 127) / 128, 128>>>(qs, shards, n, acc);
		}
	} else {
		rc = kma_iqueue_create(items, 4, n + 1, items, shards, -1, NULL, &iq);
		if (rc == KMA_OK && log)
			rc = kma_iqueue_set_chain_log(iq, log, NULL);
		if (rc == KMA_OK) {
			cudaEventRecord(e0);
			if (warp)
				k_c3_iq_enq<true><<<blocks, 256>>>(iq->dq, per_thread, n, seed, acc);
			else
				k_c3_iq_enq<false><<<blocks, 256>>>(iq->dq, per_thread, n, seed, acc);
			cudaEventRecord(e1);
			if (block)
				k_c3_iq_deq_block<<<blocks, 256>>>(iq->dq, per_thread, threads, acc);
			else if (warp)
				k_c3_iq_deq<true><<<blocks, 256>>>(iq->dq, per_thread, threads, acc);
			else
				k_c3_iq_deq<false><<<blocks, 256>>>(iq->dq, per_thread, threads, acc);
			cudaEventRecord(e2);
			k_c3_iq_walk<<<(shards + 127) / 128, 128>>>(iq->dq, n, acc);
		}
	}
	if (rc == KMA_OK && (cudaGetLastError() != cudaSuccess || cudaDeviceSynchronize() != cudaSuccess))
		rc = KMA_ECUDA;
	unsigned long long h[16];
	if (rc == KMA_OK && cudaMemcpy(h, acc, sizeof(h), cudaMemcpyDeviceToHost) != cudaSuccess)
		rc = KMA_ECUDA;
	uint32_t e = 0;
	if (rc == KMA_OK) {
		if (kind == KMA_C3_CLQUEUE)
			cudaMemcpy(&e, err, 4, cudaMemcpyDeviceToHost);
		else
			kma_iqueue_error_flags(iq, NULL, &e, 0);
		st->enqueued = h[0];
		st->in_xor = h[1];
		st->in_sum = h[2];
		st->out_count = h[3];
		st->out_xor = h[4];
		st->out_sum = h[5];
		st->empty = h[6];
		st->remaining = h[7];
		st->dequeued = h[3] - h[7] + h[9];
		st->walk_ok = h[8] == 0;
		st->err = e;
		cudaEventElapsedTime(&st->enqueue_ms, e0, e1);
		cudaEventElapsedTime(&st->dequeue_ms, e1, e2);
		if (log) {
			kma_chain_log hl;
			unsigned int cnt[2] = {0, 0};
			if (cudaMemcpy(&hl, log->dl, sizeof(hl), cudaMemcpyDeviceToHost) == cudaSuccess &&
			    cudaMemcpy(cnt, hl.next, sizeof(cnt), cudaMemcpyDeviceToHost) == cudaSuccess)
				st->log_chains = cnt[1];
		}
	}
	if (iq)
		kma_iqueue_destroy(iq);
	if (log)
		kma_chain_log_destroy(log);
	cudaEventDestroy(e0);
	cudaEventDestroy(e1);
	cudaEventDestroy(e2);
	return rc;
}

/* ------------------------------------------------------------------ */
/* config 3: concurrent tree                                           */
/* ------------------------------------------------------------------ */
namespace {
__global__ void k_c3_tree(kma_cltree *t, kma_cltree_node *pool, const uint8_t *kinds, const uint32_t *keys,
		const uint32_t *order, const uint64_t *offs, uint32_t threads, int8_t *res)
{
	uint32_t th = blockIdx.x * blockDim.x + threadIdx.x;
	if (th >= threads)
		return;
	for (uint64_t k = offs[th]; k < offs[th + 1]; k++) {
		uint32_t j = order[k];
		uint32_t key = keys[j];
		int r;
		if (kinds[j] == 0) {
			pool[j].key = key;
			r = kma_cltree_add(t, &pool[j]);
		} else if (kinds[j] == 1) {
			r = kma_cltree_get(t, key) != nullptr;
		} else {
			r = kma_cltree_remove(t, key);
		}
		res[j] = (int8_t)r;
	}
}
} /* namespace */

extern "C" int kma_c3_tree_run(const uint8_t *kinds, const uint32_t *keys, uint64_t n_ops, uint32_t threads,
		int device, int8_t *results, kma_c3_tree_stats *st)
{
	if (!kinds || !keys || !results || !st || n_ops == 0 || n_ops >= 0xffffffffull || threads == 0)
		return KMA_EINVAL;
	kma_device_guard g(device);
	if (!g.ok)
		return KMA_ENODEV;
	memset(st, 0, sizeof(*st));
	/* per-key ownership: ops grouped by owner thread, op order kept */
	std::vector<uint64_t> offs((size_t)threads + 1, 0);
	for (uint64_t j = 0; j < n_ops; j++)
		offs[keys[j] % threads + 1]++;
	for (uint32_t i = 0; i < threads; i++)
		offs[i + 1] += offs[i];
	std::vector<uint32_t> order(n_ops);
	{
		std::vector<uint64_t> pos(offs.begin(), offs.end() - 1);
		for (uint64_t j = 0; j < n_ops; j++)
			order[pos[keys[j] % threads]++] = (uint32_t)j;
	}
	kma_cltree_t t;
	int rc = kma_cltree_create(-1, NULL, &t);
	if (rc != KMA_OK)
		return rc;
	{
		dev_bufs b;
		kma_cltree_node *pool = b.alloc<kma_cltree_node>(n_ops * sizeof(kma_cltree_node));
		uint8_t *dk = b.alloc<uint8_t>(n_ops);
		uint32_t *dkeys = b.alloc<uint32_t>(n_ops * 4);
		uint32_t *dord = b.alloc<uint32_t>(n_ops * 4);
		uint64_t *doffs = b.alloc<uint64_t>(((size_t)threads + 1) * 8);
		int8_t *dres = b.alloc<int8_t>(n_ops);
		unsigned long long *stack = b.alloc<unsigned long long>(n_ops * 8);
		unsigned long long *summ = b.alloc<unsigned long long>(5 * 8);
		if (!pool || !dk || !dkeys || !dord || !doffs || !dres || !stack || !summ)
			rc = KMA_ENOMEM;
		if (rc == KMA_OK &&
		    (cudaMemcpy(dk, kinds, n_ops, cudaMemcpyHostToDevice) != cudaSuccess ||
		     cudaMemcpy(dkeys, keys, n_ops * 4, cudaMemcpyHostToDevice) != cudaSuccess ||
		     cudaMemcpy(dord, order.data(), n_ops * 4, cudaMemcpyHostToDevice) != cudaSuccess ||
		     cudaMemcpy(doffs, offs.data(), ((size_t)threads + 1) * 8, cudaMemcpyHostToDevice) != cudaSuccess))
			rc = KMA_ECUDA;
		if (rc == KMA_OK) {
			cudaEvent_t e0, e1;
			cudaEventCreate(&e0);
			cudaEventCreate(&e1);
			cudaEventRecord(e0);
			k_c3_tree<<<(threads + 255) / 256, 256>>>(t->dt, pool, dk, dkeys, dord, doffs, threads, dres);
			cudaEventRecord(e1);
			k_tree_walk<<<1, 1>>>(t->dt, stack, n_ops, NULL, summ);
			if (cudaGetLastError() != cudaSuccess || cudaDeviceSynchronize() != cudaSuccess)
				rc = KMA_ECUDA;
			cudaEventElapsedTime(&st->ms, e0, e1);
			cudaEventDestroy(e0);
			cudaEventDestroy(e1);
		}
		unsigned long long s[5];
		if (rc == KMA_OK && (cudaMemcpy(s, summ, sizeof(s), cudaMemcpyDeviceToHost) != cudaSuccess ||
				     cudaMemcpy(results, dres, n_ops, cudaMemcpyDeviceToHost) != cudaSuccess))
			rc = KMA_ECUDA;
		if (rc == KMA_OK) {
			st->live_keys = s[0];
			st->keys_xor = s[1];
			st->keys_sum = s[2];
			st->sorted = (uint32_t)s[3];
			st->err = s[4] ? 1u : 0u;
		}
	}
	kma_cltree_destroy(t);
	return rc;
}
