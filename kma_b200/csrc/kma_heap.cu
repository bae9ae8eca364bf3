/*
 * kma_heap.cu -- heap lifetime, bulk init/reset, snapshot and serial replay
 * (C ABI of include/kma.h).
 *
 * Replaces kma.c:31-127 (kma_create: buffer + one-work-item clheap_init)
 * and kma.cl:27-52 (clheap_init: empty class table, then pages-1 serial
 * idxd_enqueue calls).  Here the free list is written directly as the
 * state those enqueues produce (superblock 0 at the head as the dummy,
 * then 1..pages-1 in order) by a grid-stride kernel with 16-byte stores.
 */
#include <string.h>
#include <stdlib.h>
#include <vector>
#include "kma_internal.h"
#include "kma_backend.cuh"

/* ------------------------------------------------------------------ */
/* class tables                                                        */
/* ------------------------------------------------------------------ */

/* kma.cl:55-90 */
extern "C" uint32_t kma_size_by_sbid(uint32_t sb_log2, int block)
{
	if (sb_log2 < 4 || sb_log2 > 30)
		return 0;
	int buckets = (int)sb_log2 - 1;
	uint64_t sbsz = 1ull << sb_log2;
	/* kma.cl:61 admits block == buckets, which divides by zero at :87 */
	if (block >= buckets || block < 0)
		return 0;
	block += 2;
	if (block <= (int)(sb_log2 >> 1))
		return 1u << block;
	uint64_t bytes = 1ull << block;
	uint64_t items = sbsz / bytes;
	uint64_t alloc_bytes = items >> 3;
	alloc_bytes += (items & 0x7) ? 1 : 0;
	alloc_bytes += (alloc_bytes & 0x3) ? (4 - (alloc_bytes & 0x3)) : 0;
	uint64_t total = sbsz - (12 + alloc_bytes);
	uint64_t size = total / items;
	return (uint32_t)(size & ~0x3ull);
}

/* kma.cl:95-113 */
extern "C" int kma_slots_by_size(uint32_t sb_log2, uint64_t size)
{
	if (size == 0 || sb_log2 < 4 || sb_log2 > 30)
		return 0;
	uint64_t space = (1ull << sb_log2) - 12;
	int64_t slots = (int64_t)(space / size);
	if (slots & 0x1f)
		slots += 32;
	slots >>= 3;
	slots &= ~0x3;
	space -= (uint64_t)slots;
	return (int)(space / size);
}

/* kma.cl:119-148.  The reference approximates the class from the MSB of
 * size/4 and only ever walks upward from there, so it returns the
 * smallest class whose block size is >= size; -1 above SB-16. */
extern "C" int kma_sbid_by_size(uint32_t sb_log2, uint64_t size)
{
	if (sb_log2 < 4 || sb_log2 > 30)
		return -1;
	if (size > (1ull << sb_log2) - 16)
		return -1;
	int buckets = (int)sb_log2 - 1;
	for (int c = 0; c < buckets; c++)
		if (kma_size_by_sbid(sb_log2, c) >= size)
			return c;
	return -1;
}

int kma_fill_class_tables(uint32_t sb_log2, kma_heap *hh)
{
	uint32_t n = sb_log2 - 1;
	if (n > KMA_MAX_CLASSES)
		return KMA_EINVAL;
	hh->nclasses = n;
	hh->max_request = (1u << sb_log2) - 16;
	for (uint32_t c = 0; c < KMA_MAX_CLASSES; c++) {
		uint32_t sz = c < n ? kma_size_by_sbid(sb_log2, (int)c) : 0;
		uint32_t sl = sz ? (uint32_t)kma_slots_by_size(sb_log2, sz) : 0;
		hh->cls_size[c] = sz;
		hh->cls_slots[c] = sl;
		hh->cls_magic[c] = sz ? (uint32_t)((1ull << 32) / sz + 1) : 0;
		hh->cls_words[c] = (sl + 31) / 32;
		if (sl > KMA_ST_FREE_MASK)
			return KMA_EINVAL;
	}
	if (hh->cls_size[n - 1] != hh->max_request)
		return KMA_EINVAL;
	return KMA_OK;
}

/* ------------------------------------------------------------------ */
/* kernels                                                             */
/* ------------------------------------------------------------------ */

/* Bulk (re)initialisation: sb_state[] = 0; the free list holds superblocks
 * 0..n-1 in order (n = max(pages, 1): superblock 0 is the dummy even when
 * no other page exists, kma.cl:48); class tables empty; flags clear.  Four
 * superblocks per thread with 16-byte stores. */
__global__ void kma_k_reset(kma_heap *h, uint32_t nsb, uint32_t nfree)
{
	using namespace kma_detail;
	uint64_t tid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
	uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
	uint32_t *state = h->sb_state;
	const bool ring = h->flags & KMA_HEAP_RING;
	unsigned long long *w = ring ? h->ring : h->sb_next;
	uint64_t nquad = nsb / 4;
	for (uint64_t q = tid; q < nquad; q += stride)
		reinterpret_cast<uint4 *>(state)[q] = make_uint4(0, 0, 0, 0);
	for (uint64_t s = nquad * 4 + tid; s < nsb; s += stride)
		state[s] = 0;
	/* ring: slot i filled by ticket i ({seq i+1 | sb i}); MS queue: link
	 * i -> i+1, the last link null */
	uint64_t nw = ring ? h->ring_cap : nsb;
	uint64_t npair = nw / 2;
	for (uint64_t q = tid; q < npair; q += stride) {
		unsigned long long l[2];
#pragma unroll
		for (int i = 0; i < 2; i++) {
			uint32_t s = (uint32_t)(2 * q + i);
			if (ring)
				l[i] = s < nfree ? (((unsigned long long)(s + 1) << 32) | s)
						 : ((unsigned long long)s << 32);
			else
				l[i] = (s + 1 < nfree) ? tw_make(0, s + 2) : 0ull;
		}
		reinterpret_cast<ulonglong2 *>(w)[q] = make_ulonglong2(l[0], l[1]);
	}
	for (uint64_t i = npair * 2 + tid; i < nw; i += stride) {
		uint32_t s = (uint32_t)i;
		if (ring)
			w[i] = s < nfree ? (((unsigned long long)(s + 1) << 32) | s) : ((unsigned long long)s << 32);
		else
			w[i] = (s + 1 < nfree) ? tw_make(0, s + 2) : 0ull;
	}
	for (uint64_t i = tid; i < h->cls_lines; i += stride)
		h->cls[i].v = 0;
	if (tid == 0) {
		if (ring) {
			h->free_head.v = 0;
			h->free_tail.v = nfree;
			h->ring_avail.v = nfree;
		} else {
			h->free_head.v = tw_make(0, 1);
			h->free_tail.v = tw_make(0, nfree);
			h->ring_avail.v = 0;
		}
		h->err.v = 0;
	}
}

__global__ void kma_k_gather_bitmaps(kma_heap *h, uint32_t *dst, uint32_t words)
{
	uint64_t tid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
	uint64_t n = (uint64_t)h->nsb * words;
	for (uint64_t i = tid; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
		uint32_t s = (uint32_t)(i / words), k = (uint32_t)(i % words);
		dst[i] = *kma_detail::bitmap_word(h, kma_detail::sb_addr(h, s), k);
	}
}

/* ------------------------------------------------------------------ */
/* C ABI                                                               */
/* ------------------------------------------------------------------ */

static size_t kma_align_up(size_t x, size_t a) { return (x + a - 1) & ~(a - 1); }

static uint32_t kma_nfree(const kma_heap &hh) { return hh.pages > 1 ? hh.pages : 1; }

static int kma_launch_reset(kma_heap_s *k, cudaStream_t st)
{
	uint64_t work = ((uint64_t)k->hh.nsb + 3) / 4;
	uint32_t threads = 256;
	uint64_t blocks = (work + threads - 1) / threads;
	if (blocks < 4)
		blocks = 4; /* enough threads for the class-table lines */
	if (blocks > 148 * 16)
		blocks = 148 * 16;
	kma_k_reset<<<(unsigned)blocks, threads, 0, st>>>(k->dh, k->hh.nsb, kma_nfree(k->hh));
	KMA_CUDA(cudaGetLastError());
	return KMA_OK;
}

extern "C" int kma_create_ex(const kma_config *cfg, void *stream, kma_heap_t *out)
{
	if (!cfg || !out)
		return KMA_EINVAL;
	*out = NULL;
	if (cfg->sblocks == 0 || cfg->sb_size_log2 < 12 || cfg->sb_size_log2 > 16)
		return KMA_EINVAL;
	if (cfg->sblocks > 0x7fffffffu || cfg->shards > KMA_MAX_SHARDS)
		return KMA_EINVAL;
	if (cfg->flags & ~KMA_CFG_COMPAT)
		return KMA_EINVAL;
	kma_device_guard g(cfg->device);
	if (!g.ok)
		return KMA_ENODEV;
	int dev;
	KMA_CUDA(cudaGetDevice(&dev));

	kma_heap_s *k = (kma_heap_s *)calloc(1, sizeof(*k));
	if (!k)
		return KMA_ENOMEM;
	k->device = dev;
	memset(&k->hh, 0, sizeof(k->hh));
	if (kma_fill_class_tables(cfg->sb_size_log2, &k->hh) != KMA_OK) {
		free(k);
		return KMA_EINVAL;
	}
	uint64_t nsb = cfg->sblocks;
	/* kma.cl:42: pages = (bytes >> LOG2) - 1 where bytes also counts the
	 * header, i.e. sblocks - 1 superblocks enter the free list */
	k->hh.pages = (uint32_t)nsb - 1;
	const bool compat = cfg->flags & KMA_CFG_COMPAT;
	/* shards per class.  Every reservation of a class CASes its shard's
	 * current superblock state, so each class needs enough shards to
	 * spread the warps: a base of pages/32, capped at cfg->shards
	 * (default KMA_MAX_SHARDS).  Measured on the config-2 workload (65535
	 * pages, 9 classes in use): caps of 1024 / 2048 / 4096 gave 3.87 /
	 * 4.11 / 4.02 G ops/s, the last with NULL returns (too many
	 * superblocks pinned as shards' current ones); 2048 also cut the
	 * claims that find their bits taken from 25% to 9%. */
	uint32_t cap = compat ? 1u : (cfg->shards ? cfg->shards : KMA_MAX_SHARDS);
	uint32_t base_sh = k->hh.pages / 32;
	uint32_t lines = 0;
	for (uint32_t c = 0; c < KMA_MAX_CLASSES; c++) {
		uint32_t n = 0;
		if (c < k->hh.nclasses)
			n = base_sh < 1 ? 1 : base_sh > cap ? cap : base_sh;
		k->hh.cls_nsh[c] = n;
		k->hh.cls_base[c] = lines;
		lines += n;
	}
	k->hh.cls_lines = lines;
	k->hh.flags = compat ? 0u : KMA_HEAP_RING;
	k->hh.ring_cap = kma_nfree(k->hh);

	size_t hdr = kma_align_up(sizeof(kma_heap), 4096);
	size_t st_bytes = kma_align_up(nsb * 4, 4096);
	size_t home_bytes = kma_align_up(nsb * 2, 4096);
	size_t fl_bytes = kma_align_up((compat ? nsb : k->hh.ring_cap) * 8, 4096);
	size_t region = (size_t)nsb << cfg->sb_size_log2;
	size_t total = hdr + st_bytes + home_bytes + fl_bytes + region;
	if (cudaMalloc(&k->dev_mem, total) != cudaSuccess) {
		cudaGetLastError();
		free(k);
		return KMA_ENOMEM;
	}
	k->dev_bytes = total;
	unsigned char *base = (unsigned char *)k->dev_mem;
	k->dh = (kma_heap *)base;
	size_t o = hdr;
	k->hh.sb_state = (uint32_t *)(base + o);
	o += st_bytes;
	k->hh.sb_home = (uint16_t *)(base + o);
	o += home_bytes;
	if (compat)
		k->hh.sb_next = (unsigned long long *)(base + o);
	else
		k->hh.ring = (unsigned long long *)(base + o);
	o += fl_bytes;
	k->hh.sb_base = base + o;
	k->hh.region_bytes = region;
	k->hh.sb_log2 = cfg->sb_size_log2;
	k->hh.sb_size = 1u << cfg->sb_size_log2;
	k->hh.nsb = (uint32_t)nsb;
	k->hh.spin_limit = cfg->spin_limit ? cfg->spin_limit : KMA_DEFAULT_SPIN;
	cudaStream_t st = kma_stream(stream);
	int rc = KMA_OK;
	/* the geometry part of the header (everything before the hot lines) */
	if (cudaMemcpyAsync(k->dh, &k->hh, offsetof(kma_heap, free_head), cudaMemcpyHostToDevice, st) !=
			cudaSuccess)
		rc = KMA_ECUDA;
	if (rc == KMA_OK)
		rc = kma_launch_reset(k, st);
	if (rc == KMA_OK && cudaStreamSynchronize(st) != cudaSuccess)
		rc = KMA_ECUDA;
	if (rc != KMA_OK) {
		cudaFree(k->dev_mem);
		free(k);
		return rc;
	}
	*out = k;
	return KMA_OK;
}

extern "C" kma_heap_t kma_create(int device, void *stream, unsigned int sblocks)
{
	kma_config cfg;
	kma_heap_t h = NULL;
	if (sblocks == 0)
		return NULL;
	memset(&cfg, 0, sizeof(cfg));
	cfg.sblocks = sblocks;
	cfg.sb_size_log2 = 12;
	cfg.device = device;
	if (kma_create_ex(&cfg, stream, &h) != KMA_OK)
		return NULL;
	return h;
}

extern "C" int kma_destroy(kma_heap_t h)
{
	if (!h)
		return KMA_EINVAL;
	kma_device_guard g(h->device);
	cudaError_t e = cudaFree(h->dev_mem);
	free(h);
	return e == cudaSuccess ? KMA_OK : KMA_ECUDA;
}

extern "C" int kma_reset(kma_heap_t h, void *stream)
{
	if (!h)
		return KMA_EINVAL;
	kma_device_guard g(h->device);
	return kma_launch_reset(h, kma_stream(stream));
}

extern "C" struct kma_heap *kma_heap_device_ptr(kma_heap_t h) { return h ? h->dh : NULL; }

extern "C" int kma_get_info(kma_heap_t h, kma_info *o)
{
	if (!h || !o)
		return KMA_EINVAL;
	memset(o, 0, sizeof(*o));
	o->region_bytes = h->hh.region_bytes;
	o->device_bytes = h->dev_bytes;
	o->sblocks = h->hh.nsb;
	o->pages = h->hh.pages;
	o->sb_size_log2 = h->hh.sb_log2;
	o->nclasses = h->hh.nclasses;
	o->max_request = h->hh.max_request;
	for (int c = 0; c < 16; c++) {
		o->cls_size[c] = h->hh.cls_size[c];
		o->cls_slots[c] = h->hh.cls_slots[c];
	}
	for (int c = 0; c < 16; c++)
		o->cls_shards[c] = h->hh.cls_nsh[c];
	o->cls_lines = h->hh.cls_lines;
	o->flags = (h->hh.flags & KMA_HEAP_RING) ? 0u : KMA_CFG_COMPAT;
	return KMA_OK;
}

extern "C" int kma_error_flags(kma_heap_t h, void *stream, uint32_t *flags, int clear)
{
	if (!h || !flags)
		return KMA_EINVAL;
	kma_device_guard g(h->device);
	cudaStream_t st = kma_stream(stream);
	KMA_CUDA(cudaMemcpyAsync(flags, &h->dh->err.v, 4, cudaMemcpyDeviceToHost, st));
	if (clear)
		KMA_CUDA(cudaMemsetAsync(&h->dh->err.v, 0, 4, st));
	KMA_CUDA(cudaStreamSynchronize(st));
	return KMA_OK;
}

extern "C" int kma_error_flags_async(kma_heap_t h, void *stream, uint32_t *dst)
{
	if (!h || !dst)
		return KMA_EINVAL;
	kma_device_guard g(h->device);
	KMA_CUDA(cudaMemcpyAsync(dst, &h->dh->err.v, 4, cudaMemcpyDefault, kma_stream(stream)));
	return KMA_OK;
}

extern "C" const char *kma_strerror(int err)
{
	switch (err) {
	case KMA_OK: return "ok";
	case KMA_EINVAL: return "invalid argument";
	case KMA_ENOMEM: return "out of device memory";
	case KMA_ECUDA: return "CUDA error";
	case KMA_ETIMEDOUT: return "bounded device wait expired";
	case KMA_ENODEV: return "no such CUDA device";
	case KMA_EFAULT: return "invariant check failed";
	default: return "unknown error";
	}
}

extern "C" const char *kma_version(void) { return "kma_b200 1.1 sm_100a"; }

extern "C" int kma_snapshot(kma_heap_t h, void *stream, uint32_t *cls, uint32_t *state,
		uint32_t *freelist, uint64_t *freelist_len, uint64_t region_off, uint64_t region_len,
		void *region_dst)
{
	if (!h)
		return KMA_EINVAL;
	if (region_dst && (region_off > h->hh.region_bytes || region_len > h->hh.region_bytes - region_off))
		return KMA_EINVAL;
	kma_device_guard g(h->device);
	cudaStream_t st = kma_stream(stream);
	kma_heap *tmp = (kma_heap *)malloc(sizeof(kma_heap));
	if (!tmp)
		return KMA_ENOMEM;
	const bool ring = h->hh.flags & KMA_HEAP_RING;
	size_t nw = ring ? h->hh.ring_cap : h->hh.nsb;
	std::vector<unsigned long long> words;
	int rc = KMA_OK;
	if (cudaMemcpyAsync(tmp, h->dh, sizeof(kma_heap), cudaMemcpyDeviceToHost, st) != cudaSuccess)
		rc = KMA_ECUDA;
	if (rc == KMA_OK && state &&
			cudaMemcpyAsync(state, h->hh.sb_state, (size_t)h->hh.nsb * 4, cudaMemcpyDeviceToHost, st) !=
				cudaSuccess)
		rc = KMA_ECUDA;
	if (rc == KMA_OK && freelist) {
		words.resize(nw);
		if (cudaMemcpyAsync(words.data(), ring ? h->hh.ring : h->hh.sb_next, nw * 8,
				    cudaMemcpyDeviceToHost, st) != cudaSuccess)
			rc = KMA_ECUDA;
	}
	if (rc == KMA_OK && region_dst && region_len &&
			cudaMemcpyAsync(region_dst, h->hh.sb_base + region_off, region_len, cudaMemcpyDeviceToHost,
				st) != cudaSuccess)
		rc = KMA_ECUDA;
	if (rc == KMA_OK && cudaStreamSynchronize(st) != cudaSuccess)
		rc = KMA_ECUDA;
	if (rc == KMA_OK && cls)
		for (uint32_t i = 0; i < h->hh.cls_lines; i++)
			cls[i] = tmp->cls[i].v;
	if (rc == KMA_OK && freelist) {
		uint64_t n = 0;
		if (ring) {
			uint64_t hd = tmp->free_head.v, tl = tmp->free_tail.v;
			for (uint64_t p = hd; p < tl && n < h->hh.nsb; p++)
				freelist[n++] = (uint32_t)words[p % nw];
			if (tl - hd > h->hh.nsb)
				n = UINT64_MAX;
		} else {
			uint32_t idx = (uint32_t)tmp->free_head.v;
			while (idx != 0) {
				if (n >= h->hh.nsb || idx > nw) {
					n = UINT64_MAX;
					break;
				}
				freelist[n++] = idx - 1;
				idx = (uint32_t)words[idx - 1];
			}
		}
		if (freelist_len)
			*freelist_len = n;
	}
	free(tmp);
	return rc;
}

extern "C" int kma_gather_bitmaps(kma_heap_t h, void *stream, uint32_t *dst, uint32_t words)
{
	if (!h || !dst || words == 0)
		return KMA_EINVAL;
	if ((uint64_t)words * 4 > h->hh.sb_size)
		return KMA_EINVAL;
	kma_device_guard g(h->device);
	kma_k_gather_bitmaps<<<148 * 8, 256, 0, kma_stream(stream)>>>(h->dh, dst, words);
	KMA_CUDA(cudaGetLastError());
	return KMA_OK;
}

extern "C" int kma_replay(kma_heap_t h, const int64_t *ops, int64_t n, int64_t *out, int mode,
		void *stream)
{
	if (!h || n < 0 || (n && (!ops || !out)))
		return KMA_EINVAL;
	if (mode != KMA_MODE_PLAIN && mode != KMA_MODE_WARP)
		return KMA_EINVAL;
	kma_device_guard g(h->device);
	if (n == 0)
		return KMA_OK;
	kma_k_heap_replay<kma_backend_kma><<<1, 1, 0, kma_stream(stream)>>>(h->dh, ops, n, out, mode == KMA_MODE_WARP);
	KMA_CUDA(cudaGetLastError());
	return KMA_OK;
}

extern "C" int kma_replay_host(kma_heap_t h, const int64_t *ops, int64_t n, int64_t *out, int mode)
{
	if (!h || n < 0 || (n && (!ops || !out)))
		return KMA_EINVAL;
	if (n == 0)
		return KMA_OK;
	kma_device_guard g(h->device);
	int64_t *dops = NULL, *dout = NULL;
	int rc = KMA_OK;
	if (cudaMalloc(&dops, (size_t)n * 16) != cudaSuccess || cudaMalloc(&dout, (size_t)n * 8) != cudaSuccess) {
		cudaGetLastError();
		rc = KMA_ENOMEM;
	}
	if (rc == KMA_OK && cudaMemcpy(dops, ops, (size_t)n * 16, cudaMemcpyHostToDevice) != cudaSuccess)
		rc = KMA_ECUDA;
	if (rc == KMA_OK)
		rc = kma_replay(h, dops, n, dout, mode, NULL);
	if (rc == KMA_OK && cudaMemcpy(out, dout, (size_t)n * 8, cudaMemcpyDeviceToHost) != cudaSuccess)
		rc = KMA_ECUDA;
	if (dops)
		cudaFree(dops);
	if (dout)
		cudaFree(dout);
	return rc;
}

extern "C" int kma_debug_set_class_word(kma_heap_t h, uint32_t cls, uint32_t value, void *stream)
{
	if (!h || cls >= h->hh.nclasses)
		return KMA_EINVAL;
	kma_device_guard g(h->device);
	cudaStream_t st = kma_stream(stream);
	/* every shard's word of the class, so any calling SM sees it */
	for (uint32_t s = 0; s < h->hh.cls_nsh[cls]; s++)
		KMA_CUDA(cudaMemcpyAsync(&h->dh->cls[h->hh.cls_base[cls] + s].v, &value, 4,
					 cudaMemcpyHostToDevice, st));
	KMA_CUDA(cudaStreamSynchronize(st));
	return KMA_OK;
}

/* ------------------------------------------------------------------ */
/* heap images (kma.h): save and restore                               */
/* ------------------------------------------------------------------ */
namespace {

const uint64_t KMA_IMG_ALIGN = 256;
static_assert(sizeof(kma_image_header) == 184, "kma_image_header is packed, 184 bytes");

/* The image layout of heap geometry hh (sections 256-byte aligned). */
void kma_image_layout(const kma_heap &hh, kma_image_header &hdr)
{
	memset(&hdr, 0, sizeof(hdr));
	memcpy(hdr.magic, KMA_IMAGE_MAGIC, 8);
	hdr.version = KMA_IMAGE_VERSION;
	hdr.header_bytes = sizeof(kma_image_header);
	hdr.sb_log2 = hh.sb_log2;
	hdr.sblocks = hh.nsb;
	hdr.pages = hh.pages;
	hdr.ring = (hh.flags & KMA_HEAP_RING) ? 1u : 0u;
	hdr.nclasses = hh.nclasses;
	hdr.cls_lines = hh.cls_lines;
	hdr.flist_words = hdr.ring ? hh.ring_cap : hh.nsb;
	for (uint32_t c = 0; c < hh.nclasses && c < 16; c++)
		hdr.cls_shards[c] = hh.cls_nsh[c];
	uint64_t o = kma_align_up(sizeof(kma_image_header), KMA_IMG_ALIGN);
	hdr.off_cls = o;
	o = kma_align_up(o + (uint64_t)hdr.cls_lines * 4, KMA_IMG_ALIGN);
	hdr.off_state = o;
	o = kma_align_up(o + (uint64_t)hdr.sblocks * 4, KMA_IMG_ALIGN);
	hdr.off_home = o;
	o = kma_align_up(o + (uint64_t)hdr.sblocks * 2, KMA_IMG_ALIGN);
	hdr.off_flist = o;
	o = kma_align_up(o + (uint64_t)hdr.flist_words * 8, KMA_IMG_ALIGN);
	hdr.off_region = o;
	hdr.total_bytes = o + hh.region_bytes;
}

/* Every metadata word of an image stays inside the heap: what a kernel
 * would index with it (sb_state, sb_next, ring slots, class lines) is in
 * range.  Region bytes need no check: bitmap bits only select slots below
 * a class's slot count. */
bool kma_image_valid(const kma_heap &hh, const kma_image_header &hdr, const uint32_t *cls,
		const uint32_t *state, const uint16_t *home, const unsigned long long *fl)
{
	const uint32_t nsb = hh.nsb;
	for (uint32_t i = 0; i < hdr.cls_lines; i++)
		if (cls[i] == KMA_POISON || (cls[i] >= KMA_CLS_BASE && cls[i] - KMA_CLS_BASE >= nsb))
			return false;
	for (uint32_t s = 0; s < nsb; s++) {
		uint32_t st = state[s];
		if (st == 0)
			continue;
		uint32_t c = st >> KMA_ST_CLASS_SHIFT;
		uint32_t slots = (st >> KMA_ST_SLOTS_SHIFT) & KMA_ST_FREE_MASK;
		uint32_t fr = st & KMA_ST_FREE_MASK;
		if (c >= hh.nclasses || slots != hh.cls_slots[c] || fr > slots || home[s] >= hh.cls_nsh[c])
			return false;
	}
	/* The free list must be one a quiescent heap can hold: every queued
	 * superblock once (a second entry would be handed out twice), each
	 * with free count 0 (detaching for the free list zeroes it; a live
	 * superblock on the list would be reformatted under its blocks). */
	std::vector<unsigned char> queued(nsb, 0);
	auto take = [&](uint32_t s) {
		if (s >= nsb || queued[s] || (state[s] & KMA_ST_FREE_MASK) != 0)
			return false;
		queued[s] = 1;
		return true;
	};
	if (hdr.ring) {
		const uint64_t head = hdr.free_head, tail = hdr.free_tail, cap = hh.ring_cap;
		if (tail < head || tail - head > cap || hdr.flist_words != cap)
			return false;
		/* completed enqueues not yet claimed: the queued count exactly */
		if ((int64_t)(int32_t)hdr.ring_avail != (int64_t)(tail - head))
			return false;
		/* slot of ticket p: {seq p+1 | sb} when filled (head <= p < tail),
		 * {seq p | -} when free for the enqueue with ticket p */
		for (uint64_t p = head; p < head + cap; p++) {
			const unsigned long long w = fl[p % cap];
			const uint32_t seq = (uint32_t)(w >> 32);
			if (p < tail) {
				if (seq != (uint32_t)(p + 1) || !take((uint32_t)w))
					return false;
			} else if (seq != (uint32_t)p) {
				return false;
			}
		}
	} else {
		/* MS queue over superblock indices (idx = s + 1): the chain from
		 * the head (the dummy) must end at the tail with a null link, with
		 * no superblock twice (a cycle never ends) */
		uint32_t hi = (uint32_t)hdr.free_head, ti = (uint32_t)hdr.free_tail;
		if (hi == 0 || hi > nsb || ti == 0 || ti > nsb)
			return false;
		for (uint32_t i = 0; i < hdr.flist_words; i++)
			if ((uint32_t)fl[i] > nsb)
				return false;
		uint32_t idx = hi;
		for (;;) {
			if (!take(idx - 1))
				return false;
			uint32_t nx = (uint32_t)fl[idx - 1];
			if (nx == 0)
				break;
			idx = nx;
		}
		if (idx != ti)
			return false;
	}
	return true;
}

} /* namespace */

extern "C" int kma_image_bytes(kma_heap_t h, uint64_t *bytes)
{
	if (!h || !bytes)
		return KMA_EINVAL;
	kma_image_header hdr;
	kma_image_layout(h->hh, hdr);
	*bytes = hdr.total_bytes;
	return KMA_OK;
}

extern "C" int kma_image_save(kma_heap_t h, void *stream, void *dst, uint64_t dst_bytes)
{
	if (!h || !dst)
		return KMA_EINVAL;
	kma_image_header hdr;
	kma_image_layout(h->hh, hdr);
	if (dst_bytes < hdr.total_bytes)
		return KMA_EINVAL;
	kma_device_guard g(h->device);
	if (!g.ok)
		return KMA_ENODEV;
	cudaStream_t st = kma_stream(stream);
	/* the hot words and the class lines live in the device header */
	std::vector<unsigned char> dev_hdr(sizeof(kma_heap));
	kma_heap *tmp = reinterpret_cast<kma_heap *>(dev_hdr.data());
	KMA_CUDA(cudaMemcpyAsync(tmp, h->dh, sizeof(kma_heap), cudaMemcpyDeviceToHost, st));
	KMA_CUDA(cudaStreamSynchronize(st));
	hdr.free_head = tmp->free_head.v;
	hdr.free_tail = tmp->free_tail.v;
	hdr.ring_avail = tmp->ring_avail.v;
	hdr.err = tmp->err.v;
	std::vector<uint32_t> cls(hdr.cls_lines);
	for (uint32_t i = 0; i < hdr.cls_lines; i++)
		cls[i] = tmp->cls[i].v;
	unsigned char *d = static_cast<unsigned char *>(dst);
	const unsigned long long *fl = hdr.ring ? h->hh.ring : h->hh.sb_next;
	KMA_CUDA(cudaMemcpyAsync(d, &hdr, sizeof(hdr), cudaMemcpyDefault, st));
	KMA_CUDA(cudaMemcpyAsync(d + hdr.off_cls, cls.data(), (size_t)hdr.cls_lines * 4, cudaMemcpyDefault, st));
	KMA_CUDA(cudaMemcpyAsync(d + hdr.off_state, h->hh.sb_state, (size_t)hdr.sblocks * 4, cudaMemcpyDefault, st));
	KMA_CUDA(cudaMemcpyAsync(d + hdr.off_home, h->hh.sb_home, (size_t)hdr.sblocks * 2, cudaMemcpyDefault, st));
	KMA_CUDA(cudaMemcpyAsync(d + hdr.off_flist, fl, (size_t)hdr.flist_words * 8, cudaMemcpyDefault, st));
	KMA_CUDA(cudaMemcpyAsync(d + hdr.off_region, h->hh.sb_base, h->hh.region_bytes, cudaMemcpyDefault, st));
	KMA_CUDA(cudaStreamSynchronize(st)); /* the staged header and class words */
	return KMA_OK;
}

extern "C" int kma_image_load(kma_heap_t h, void *stream, const void *src, uint64_t src_bytes)
{
	if (!h || !src)
		return KMA_EINVAL;
	kma_image_header want;
	kma_image_layout(h->hh, want);
	if (src_bytes < sizeof(kma_image_header))
		return KMA_EINVAL;
	kma_device_guard g(h->device);
	if (!g.ok)
		return KMA_ENODEV;
	cudaStream_t st = kma_stream(stream);
	const unsigned char *s = static_cast<const unsigned char *>(src);
	kma_image_header hdr;
	KMA_CUDA(cudaMemcpyAsync(&hdr, s, sizeof(hdr), cudaMemcpyDefault, st));
	KMA_CUDA(cudaStreamSynchronize(st));
	/* same format and geometry: every section offset then matches too */
	if (memcmp(hdr.magic, want.magic, 8) || hdr.version != want.version ||
			hdr.header_bytes != want.header_bytes || hdr.sb_log2 != want.sb_log2 ||
			hdr.sblocks != want.sblocks || hdr.pages != want.pages || hdr.ring != want.ring ||
			hdr.nclasses != want.nclasses || hdr.cls_lines != want.cls_lines ||
			hdr.flist_words != want.flist_words ||
			memcmp(hdr.cls_shards, want.cls_shards, sizeof(want.cls_shards)) ||
			hdr.off_cls != want.off_cls || hdr.off_state != want.off_state ||
			hdr.off_home != want.off_home || hdr.off_flist != want.off_flist ||
			hdr.off_region != want.off_region || hdr.total_bytes != want.total_bytes ||
			src_bytes < hdr.total_bytes)
		return KMA_EINVAL;
	/* the metadata comes to the host for checking before any of it reaches
	 * the device */
	std::vector<uint32_t> cls(hdr.cls_lines), state(hdr.sblocks);
	std::vector<uint16_t> home(hdr.sblocks);
	std::vector<unsigned long long> fl(hdr.flist_words);
	KMA_CUDA(cudaMemcpyAsync(cls.data(), s + hdr.off_cls, cls.size() * 4, cudaMemcpyDefault, st));
	KMA_CUDA(cudaMemcpyAsync(state.data(), s + hdr.off_state, state.size() * 4, cudaMemcpyDefault, st));
	KMA_CUDA(cudaMemcpyAsync(home.data(), s + hdr.off_home, home.size() * 2, cudaMemcpyDefault, st));
	KMA_CUDA(cudaMemcpyAsync(fl.data(), s + hdr.off_flist, fl.size() * 8, cudaMemcpyDefault, st));
	std::vector<unsigned char> dev_hdr(sizeof(kma_heap));
	kma_heap *tmp = reinterpret_cast<kma_heap *>(dev_hdr.data());
	KMA_CUDA(cudaMemcpyAsync(tmp, h->dh, sizeof(kma_heap), cudaMemcpyDeviceToHost, st));
	KMA_CUDA(cudaStreamSynchronize(st));
	if (!kma_image_valid(h->hh, hdr, cls.data(), state.data(), home.data(), fl.data()))
		return KMA_EINVAL;
	tmp->free_head.v = hdr.free_head;
	tmp->free_tail.v = hdr.free_tail;
	tmp->ring_avail.v = hdr.ring_avail;
	tmp->err.v = hdr.err;
	for (uint32_t i = 0; i < hdr.cls_lines; i++)
		tmp->cls[i].v = cls[i];
	unsigned long long *dfl = hdr.ring ? h->hh.ring : h->hh.sb_next;
	KMA_CUDA(cudaMemcpyAsync(h->hh.sb_state, state.data(), state.size() * 4, cudaMemcpyHostToDevice, st));
	KMA_CUDA(cudaMemcpyAsync(h->hh.sb_home, home.data(), home.size() * 2, cudaMemcpyHostToDevice, st));
	KMA_CUDA(cudaMemcpyAsync(dfl, fl.data(), fl.size() * 8, cudaMemcpyHostToDevice, st));
	KMA_CUDA(cudaMemcpyAsync(h->hh.sb_base, s + hdr.off_region, h->hh.region_bytes, cudaMemcpyDefault, st));
	/* the device header last: its geometry fields are h's own, read back above */
	KMA_CUDA(cudaMemcpyAsync(h->dh, tmp, sizeof(kma_heap), cudaMemcpyHostToDevice, st));
	KMA_CUDA(cudaStreamSynchronize(st));
	return KMA_OK;
}
